"""Input files in the reference's formats, written for the command-line tests: a parameter
file (loadEnePara's line formats), a multi-model PDB, a ligand SDF with an ensemble, and a
pocket .ff (CENTER, KDE, PSP, MCS lines)."""
import numpy as np

from geaxdock_gpu_b200 import abi, loaders


def write_paras(path, raw):
    """A parameter file holding the given raw parameters (loadEnePara's line formats)."""
    L = []
    for p, pn in enumerate(loaders.PNT):
        for l, ln in enumerate(loaders.LIG_TYPES):
            L.append("VDW %s %s %.9g %.9g" % (pn, ln, raw.vdw[p][l][0], raw.vdw[p][l][1]))
            L.append("PMF %s %s %.9g %.9g" % (pn, ln, raw.pmf[p][l][0], raw.pmf[p][l][1]))
            L.append("HDB %s %s %.9g %.9g" % (pn, ln, raw.hdb[p][l][0], raw.hdb[p][l][1]))
        L.append("ELE %s %.9g" % (pn, raw.ele[p]))
    for r, rn in enumerate(loaders.RES1):
        L.append("ELE %sC %.9g" % (rn, raw.ele[r + 30]))
        L.append("HPP %s %.9g" % (rn, raw.hpp[r]))
    for l, ln in enumerate(loaders.LIG_TYPES):
        L.append("HPL %s %.9g %.9g" % (ln, raw.hpl[l][0], raw.hpl[l][1]))
    L.append("PLJ %.9g %.9g %.9g" % tuple(raw.lj))
    L.append("PEL %.9g %.9g" % tuple(raw.el))
    L.append("KDE %.9g" % raw.kde)
    for key, arr in (("WEI", raw.w), ("NOA", raw.a_para), ("NOB", raw.b_para)):
        L.append(key + " " + " ".join("%.9g" % v for v in list(arr)[:abi.MAXWEI - 1]))
    path.write_text("\n".join(L) + "\n")


def write_complex(tmp_path, rng, n_res=40, lna=12, n_models=2):
    res = ["ALA", "LEU", "SER", "LYS", "ASP", "PHE", "GLY", "TYR", "THR", "GLU"]
    pdb = []
    for m in range(n_models):
        pdb.append("MODEL     %4d" % (m + 1))
        serial = 1
        for i in range(n_res):
            rn = res[i % len(res)]
            base = np.array([3.8 * np.cos(i * 0.6) * 3, 3.8 * np.sin(i * 0.6) * 3, 1.5 * i])
            base = base + rng.normal(0, 0.2, 3) * m
            for an, d in (("N", -1.0), ("CA", 0.0), ("C", 1.0), ("O", 1.6), ("CB", 0.8),
                          ("CG", 1.9)):
                if rn == "GLY" and an in ("CB", "CG"):
                    continue
                x, y, z = base + np.array([d, 0.3 * d, -0.2 * d])
                pdb.append("ATOM  %5d  %-3s %3s A%4d    %8.3f%8.3f%8.3f  1.00  0.00           C"
                           % (serial, an, rn, i + 1, x, y, z))
                serial += 1
        pdb.append("ENDMDL")
    (tmp_path / "p.pdb").write_text("\n".join(pdb) + "\n")
    center = np.array([0.0, 0.0, 30.0])
    types = ["C.3", "C.ar", "N.am", "O.2", "C.2", "O.3"]
    atoms = rng.normal(0, 1.5, (lna, 3)) + center
    sdf = ["lig", "  synthetic", "", "%3d%3d  0  0  0  0  0  0  0  0999 V2000" % (lna, 0)]
    for x, y, z in atoms:
        sdf.append("%10.4f%10.4f%10.4f C   0  0  0  0  0  0  0  0  0  0  0  0" % (x, y, z))
    rows = [atoms + rng.normal(0, 0.5, atoms.shape) for _ in range(4)]
    sdf += ["M  END", "> <MOLID>", "L1", "", "> <OB_ATOM_TYPES>",
            " ".join(types[i % len(types)] for i in range(lna)), "",
            "> <OB_ATOMIC_CHARGES>", " ".join("%.3f" % v for v in rng.normal(0, 0.3, lna)), "",
            "> <ENSEMBLE_RMSD>", "0.6 0.7 0.05 0.8", "", "> <ENSEMBLE_COORDS>"]
    sdf += [" ".join("%.4f" % v for v in r.ravel()) for r in rows]
    sdf += ["", "$$$$"]
    (tmp_path / "l.sdf").write_text("\n".join(sdf) + "\n")
    ff = ["CENTER %.4f %.4f %.4f" % tuple(center)]
    for i in range(60):
        p = center + rng.normal(0, 2.5, 3)
        ff.append("KDE %s %.4f %.4f %.4f" % (types[i % len(types)], *p))
    for i in range(1, n_res + 1, 3):
        ff.append("PSP %d %s %.3f" % (i, types[i % len(types)], rng.uniform(0, 1)))
    for m in range(3):
        pts = " ".join("%d %.4f %.4f %.4f" % (a, *(atoms[a - 1] + rng.normal(0, 0.3, 3)))
                       for a in (1, 4, 7))
        ff.append("MCS synth %.4f 3 %s" % (rng.uniform(0.1, 0.5), pts))
    (tmp_path / "p.ff").write_text("\n".join(ff) + "\n")
