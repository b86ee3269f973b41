"""Input loaders (geaxdock_gpu_b200/loaders.py) on CPU.

* On the reference's own input files (when its tree is present), every array of the complex
  and the raw and folded energy parameters equal, bit for bit, the fixtures that the
  reference's loaders and folds produced (tests/golden/make_golden.py, via oracle/refpin).
* The reference's own loader tests (src/load_test.C), restated on the same files: record and
  ensemble counts, atom/bond counts, coordinates as read and after centring, the pocket
  centre, the weight file against the parameter file.
* On small files written here, the parsing rules the reference applies: ensemble conformers
  kept only above 0.1 A RMSD and centred on their own centroid, effective points of each
  residue, one conformation per ENDMDL/TER block, both MCS line formats, unknown ligand types,
  the hydrophobicity normalisation, the peptide-plane rule from the third model on.
"""
import os

import numpy as np

from oracle import reference_root
import pytest

from geaxdock_gpu_b200 import abi, loaders
from tests.golden.fixtures import load_ref

REFERENCE = reference_root() or ""
DATA = os.path.join(REFERENCE, "data")

RUNS = {
    "1a07C1": ("1a07C1", "1a07C.pdb", "1a07C1.sdf", "1a07C1-0.8.ff", "1a07C1", 4, 0.5, 2.0),
    "1robA1": ("1robA1", "1robA.pdb", "1robA1.sdf", "1robA1-0.8.ff", "1robA1", 2, 0.5, 1.0),
}
ARRAYS = ("lig_x", "lig_y", "lig_z", "lig_center", "lig_t", "lig_c", "lig_n", "prt_x", "prt_y",
          "prt_z", "prt_t", "prt_c", "prt_ele", "prt_seq3r", "prt_hflag", "prt_hpp",
          "pocket_center", "psp", "kde_x", "kde_y", "kde_z", "kde_t", "mcs_x", "mcs_y", "mcs_z",
          "mcs_tcc")


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype.itemsize == 4 else a


@pytest.mark.parametrize("name", sorted(RUNS))
def test_reference_inputs_load_bit_exact(name):
    d, pdb, sdf, ff, cid, nt, fl, ce = RUNS[name]
    files = [os.path.join(DATA, d, f) for f in (pdb, sdf, ff)]
    paras = os.path.join(DATA, "parameters", "paras")
    if not all(os.path.exists(f) for f in files + [paras]):
        pytest.skip("the reference's input files are not present")
    z, _, _ = load_ref(name)
    cx, ep, raw = loaders.load_complex(*files, paras, cid, nt, fl, ce)
    assert np.array_equal(_bits(abi.struct_to_array(raw)), _bits(z["enepara_raw"]))
    assert np.array_equal(_bits(abi.struct_to_array(ep)), _bits(z["enepara"]))
    for k in ARRAYS:
        a, b = getattr(cx, k), z[k]
        assert a.shape == b.shape, k
        assert np.array_equal(_bits(a), _bits(b)), k
    want = np.frombuffer(z["temp"].tobytes(), dtype=abi.TEMP_DTYPE)
    assert np.array_equal(_bits(cx.temp["minus_beta"]), _bits(want["minus_beta"]))
    assert np.array_equal(cx.temp["order"], want["order"])


def _atom(serial, name, res, resnum, x, y, z):
    return "ATOM  %5d %-4s %3s A%4d    %8.3f%8.3f%8.3f  1.00  0.00           C" % (
        serial, name, res, resnum, x, y, z)


def _pdb(tmp_path, models, sep="ENDMDL"):
    """models: list of lists of (atom name, residue, resnum, x, y, z)."""
    lines = []
    for m, atoms in enumerate(models):
        lines.append("MODEL     %4d" % (m + 1))
        for i, (an, res, rn, x, y, z) in enumerate(atoms):
            name = " %-3s" % an
            lines.append(_atom(i + 1, name, res, rn, x, y, z))
        lines.append(sep)
    p = tmp_path / "p.pdb"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


def _residue(res, rn, base, side):
    out = [("N", res, rn, base, 0.0, 0.0), ("CA", res, rn, base + 1, 0.0, 0.0),
           ("C", res, rn, base + 2, 0.0, 0.0), ("O", res, rn, base + 2, 1.0, 0.0)]
    for an, x in side:
        out.append((an, res, rn, base + x, 2.0, 0.0))
    return out


def test_protein_points_and_blocks(tmp_path):
    # ALA 5, GLU 6, GLY 7, TRP 8 in two models; the second shifted by +10 in x
    def model(dx):
        atoms = []
        atoms += _residue("ALA", 5, 0.0 + dx, [("CB", 1.0)])
        atoms += _residue("GLU", 6, 10.0 + dx, [("CB", 1.0), ("CG", 2.0), ("CD", 3.0),
                                                ("OE1", 4.0)])
        atoms += _residue("GLY", 7, 20.0 + dx, [])
        atoms += _residue("TRP", 8, 30.0 + dx, [("CB", 1.0), ("CG", 2.0), ("CD1", 3.0)])
        return atoms
    prt = loaders.load_protein(_pdb(tmp_path, [model(0.0), model(100.0)]))
    # points: CA(A) A1 | CA(E) E1 E2 | CA(G) PP(E) | CA(W) PP(G) W1 W2
    assert prt.t.tolist() == [0, 2, 0, 5, 6, 0, 1, 0, 1, 26, 27]
    assert prt.r.tolist() == [0, 0, 1, 1, 1, 2, 1, 3, 2, 3, 3]
    assert prt.c.tolist() == [0, 2, 0, 2, 3, 0, 1, 0, 1, 2, 3]
    assert prt.seq3.tolist() == [5, 6, 7, 8]
    assert prt.n_conf == 2
    x = prt.x[0]
    assert x[0] == np.float32(1.0)                                   # CA of ALA
    assert x[1] == np.float32(1.0)                                   # CB of ALA
    assert x[3] == np.float32((13.0 + 14.0) / 2)                     # GLU beyond CG
    assert x[4] == np.float32((11.0 + 12.0) / 2)                     # GLU CB + CG
    # PP of GLU (residue index 1) is N(GLU) + C(ALA) + O(ALA), float sums in file order
    s = np.float32(np.float32(np.float32(2.0) + np.float32(2.0)) + np.float32(10.0))
    assert x[6] == np.float32(s / np.float32(3.0))
    assert np.allclose(prt.x[1], prt.x[0] + 100.0)


def test_protein_peptide_plane_from_third_model(tmp_path):
    def model(dx):
        return (_residue("ALA", 1, 0.0 + dx, []) + _residue("ALA", 2, 10.0 + dx, [])
                + _residue("ALA", 3, 20.0 + dx, []) + _residue("ALA", 4, 30.0 + dx, []))
    prt = loaders.load_protein(_pdb(tmp_path, [model(0.0), model(1.0), model(2.0)]))
    pp = [i for i, t in enumerate(prt.t) if t == 1]
    n_of = {1: 10.0, 2: 20.0}  # N of residues 2, 3 (index 1, 2)
    for p in pp:
        ri = int(prt.r[p])
        three = np.float32(np.float32(np.float32(n_of[ri] - 8.0) + np.float32(n_of[ri] - 8.0))
                           + np.float32(n_of[ri]))
        assert prt.x[0, p] == np.float32(three / np.float32(3.0))
        assert prt.x[2, p] == np.float32(n_of[ri] + 2.0)  # N alone (see loaders.load_protein)


def test_protein_ter_ends_a_conformation(tmp_path):
    atoms = _residue("ALA", 1, 0.0, []) + _residue("SER", 2, 5.0, [("OG", 1.0)])
    prt = loaders.load_protein(_pdb(tmp_path, [atoms], sep="TER"))
    assert prt.n_conf == 1 and prt.t.tolist() == [0, 2, 0, 23]
    assert prt.x[0, 1] == 0.0  # a point without atoms keeps 0 (nothing is stored for it)


def _sdf(tmp_path, coords, rmsds, rows, types, charges):
    lna = len(coords)
    lines = ["lig", "  x", "", "%3d%3d  0  0  0  0  0  0  0  0999 V2000" % (lna, 0)]
    for x, y, z in coords:
        lines.append("%10.4f%10.4f%10.4f C   0  0  0  0  0  0  0  0  0  0  0  0" % (x, y, z))
    lines += ["M  END", "> <MOLID>", "L1", "", "> <OB_ATOM_TYPES>", " ".join(types), "",
              "> <OB_ATOMIC_CHARGES>", " ".join("%.3f" % c for c in charges), "",
              "> <ENSEMBLE_RMSD>", " ".join("%.3f" % r for r in rmsds), "",
              "> <ENSEMBLE_COORDS>"]
    lines += [" ".join("%.4f" % v for v in row) for row in rows]
    lines += ["", "$$$$"]
    p = tmp_path / "l.sdf"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


def test_ligand_ensemble_filter_and_centring(tmp_path):
    coords = [(1.0, 2.0, 3.0), (3.0, 2.0, 1.0), (2.0, 5.0, 2.0)]
    rows = [[1, 1, 1, 2, 2, 2, 3, 3, 3], [0, 0, 0, 1, 0, 0, 0, 1, 0],
            [4, 4, 4, 4, 4, 4, 4, 4, 7]]
    lig = loaders.load_ligand(_sdf(tmp_path, coords, [0.5, 0.05, 0.1001], rows,
                                   ["C.3", "N.am", "Xx"], [0.1, -0.2, 0.3]))
    assert lig.n_conf == 3                          # the 0.05 A conformer is dropped
    assert lig.t.tolist() == [3, 13, loaders.BADKDE]
    assert lig.c.dtype == np.float32 and lig.props["MOLID"] == "L1"
    for k in range(lig.n_conf):
        for a in (lig.x[k], lig.y[k], lig.z[k]):
            assert abs(float(a.astype(np.float64).sum())) < 1e-5
    assert lig.x[1].tolist() == [-1.0, 0.0, 1.0]


def test_pocket_file(tmp_path):
    p = tmp_path / "p.ff"
    p.write_text("\n".join([
        "CENTER 1.5 -2.25 3.0",
        "KDE C.2 1.0 2.0 3.0",
        "KDE Q.q 4.0 5.0 6.0",
        "PSP 12 N.am 0.75",
        "PSP 3 Zz 9.0",
        "MCS LIG1 0.25 2 1 1.0 2.0 3.0 4 4.0 5.0 6.0",
        "MCS tmpl LIG1 0.5 1 2 7.0 8.0 9.0",
        "CENTER 10.0 20.0 30.0",
    ]) + "\n")
    pk = loaders.load_pocket(str(p), "LIG1")
    assert pk.center.tolist() == [10.0, 20.0, 30.0]   # the last CENTER line
    assert pk.kde_t.tolist() == [2, loaders.BADKDE]
    assert pk.psp[(12, 13)] == np.float32(0.75) and (3, loaders.BADKDE) in pk.psp
    assert pk.mcs_tcc.tolist() == [0.25, 0.5]
    assert pk.mcs_x[0, 1] == 1.0 and pk.mcs_z[0, 4] == 6.0 and pk.mcs_y[1, 2] == 8.0
    assert pk.mcs_x[0, 0] == np.float32(loaders.MCS_INVALID_COORD)


def test_enepara_hydrophobicity_normalised(tmp_path):
    p = tmp_path / "paras"
    lines = ["HPP %s %d" % (c, i) for i, c in enumerate(loaders.RES1)]
    lines += ["VDW CA C.3 1.5 2.5", "ELE AC 0.3", "ELE R1 -0.4", "WEI 1 2 3 4 5 6 7 8 9",
              "PLJ 1 2 3", "PEL 4 5", "KDE 0.6", "HPL Br 0.1 0.2", "HDB K1 O.2 0.5 0.6"]
    p.write_text("\n".join(lines) + "\n")
    ep = loaders.load_enepara(str(p))
    hpp = np.asarray(ep.hpp)
    assert hpp[0] == -1.0 and hpp[19] == 1.0 and np.all(np.diff(hpp) > 0)
    assert ep.vdw[0][3][0] == 1.5 and ep.ele[30] == np.float32(0.3) and ep.ele[21] == np.float32(-0.4)
    assert list(ep.w)[:9] == [1, 2, 3, 4, 5, 6, 7, 8, 9] and ep.w[9] == 0
    assert ep.kde == np.float32(0.6) and ep.hdb[12][16][1] == np.float32(0.6)


def test_unknown_residue_is_an_error(tmp_path):
    atoms = _residue("ALA", 1, 0.0, []) + [("CA", "XYZ", 2, 5.0, 0.0, 0.0)]
    with pytest.raises(loaders.LoadError):
        loaders.load_protein(_pdb(tmp_path, [atoms]))


# ------------------------------------------------------------------------------------------
# the reference's own loader tests (src/load_test.C), restated on the same files


def _data(*parts):
    p = os.path.join(DATA, *parts)
    if not os.path.exists(p):
        pytest.skip("the reference's input files are not present")
    return p


def _almost(want, got, ulps=4):
    """gtest's FloatingPoint<float>::AlmostEquals: within 4 units in the last place."""
    a, b = np.float32(want), np.float32(got)

    def key(v):
        i = int(np.array(v, np.float32).view(np.int32))
        return i if i >= 0 else -(i & 0x7FFFFFFF)
    return abs(key(a) - key(b)) <= ulps


def test_load_test_weights():
    """loadWeight/parameters (src/load_test.C:15-30): the term weights of the parameter file
    and of the separate weight file agree within 1e-4."""
    w = loaders.load_weights(_data("parameters", "08ff_opt"))
    raw = loaders.load_enepara(_data("parameters", "paras"))
    assert w.shape[0] == 9
    for i in range(w.shape[0]):
        assert abs(float(raw.w[i]) - float(w[i])) < 1e-4, i


def test_load_test_ligand_1a07C1():
    """Load_Ligands/1a07C1 (src/load_test.C:71-111): one record whose ENSEMBLE_TOTAL matches
    its coordinate rows and RMSD values, 21 conformers after the RMSD filter, conformer 0 atom
    0 x = 45.6740, conformer 2 atom 0 y = -5.2246 (as read)."""
    secs = loaders.sdf_records(_data("1a07C1", "1a07C1.sdf"))
    assert len(secs) == 1
    total = loaders.ensemble_total(secs[0])
    rmsds, rows = loaders.ensemble(secs[0])
    assert len(rows) == total and len(rmsds) == total
    lna, _ = loaders.ligand_header(secs[0])
    confs = loaders.ligand_conformers(secs[0], lna)
    assert len(confs) == 21
    assert _almost(45.6740, confs[0][0][0])
    assert _almost(-5.2246, confs[2][1][0])
    assert loaders.load_ligand(_data("1a07C1", "1a07C1.sdf")).n_conf == 21


def test_load_test_ligands_1b9v():
    """Load_Ligands/1b9vA (src/load_test.C:113-180): six records, 50 ensemble conformers with
    50 RMSD values, 23 atoms and 23 bonds; atom 1 x of the atom block -0.0184, of ensemble row
    0 2.1011, atom 1 z of row 2 -2.2202; atom 0 x after centring -3.6306739; pocket centre
    y -9.590."""
    secs = loaders.sdf_records(_data("edud", "1b9v_4.sdf"))
    assert len(secs) == 6
    sect = secs[0]
    assert loaders.ensemble_total(sect) == 50
    rmsds, rows = loaders.ensemble(sect)
    assert len(rows) == 50 and len(rmsds) == 50
    lna, lnb = loaders.ligand_header(sect)
    assert (lna, lnb) == (23, 23)
    x, y, z = loaders.atom_block(sect, lna)
    assert _almost(-0.0184, x[1])
    assert _almost(2.1011, loaders.ensemble_coords(rows[0], lna)[0][1])
    assert _almost(-2.2202, loaders.ensemble_coords(rows[2], lna)[2][1])
    assert _almost(-3.6306739, loaders.centre(x, y, z)[0][0])
    assert _almost(-9.590, loaders.pocket_center(_data("edud", "1b9v_4.ff"))[1])


def test_load_test_ligands_1e66():
    """Load_Ligands/1e66 (src/load_test.C:183-213): six records, 50 ensemble conformers,
    28 atoms and 31 bonds."""
    secs = loaders.sdf_records(_data("edud", "1e66_4.sdf"))
    assert len(secs) == 6
    assert loaders.ensemble_total(secs[0]) == 50
    rmsds, rows = loaders.ensemble(secs[0])
    assert len(rmsds) == len(rows) == 50
    assert loaders.ligand_header(secs[0]) == (28, 31)


def test_load_test_10gs():
    """Load_Ligands/10gsA00 and Load_Protein/10gsA00 (src/load_test.C:216-239): the ligand
    file loads; the protein has one conformation."""
    loaders.load_ligand(_data("10gs", "10gs_ligand.sdf"))
    loaders.pocket_center(_data("10gs", "10gsA00.ff"))
    assert loaders.load_protein(_data("10gs", "10gsA00.pdb")).n_conf == 1
