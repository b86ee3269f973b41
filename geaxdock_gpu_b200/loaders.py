"""Input loaders: the reference's file formats into the library's complex arrays.

Restates the reference's host front end (src/load.C, src/data.C, the pre-processing folds of
src/util.C) so that a complex is built from the same files the reference reads:

  protein   PDB, one conformation per model      loadProtein       src/load.C:931-1265
  ligand    SDF with an ensemble of conformers   loadLigand        src/load.C:157-230, 330-470
  pocket    .ff: CENTER, KDE, PSP, MCS lines     loadLHM           src/load.C:1296-1450
  energy    `paras` parameter file               loadEnePara       src/load.C:1477-1660
  folds     OptimizeLigand / Protein / Psp / Kde / Mcs, CopyProteinResidue
                                                 src/util.C:264-290, 574-715
            (SetTemperature and OptimizeEnepara are the library's gd_set_temperature and
            gd_fold_enepara)

Arithmetic follows the reference's types: coordinates are parsed as C's atof does (to double,
then stored as float) and every sum, mean and centring is carried out in IEEE single
precision in the reference's order, so the arrays are the reference's bit for bit
(tests/test_loaders.py checks them against fixtures produced by the reference's own loaders).
"""
from __future__ import annotations

import re
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import abi

F32 = np.float32

MINLIGRMSD = 0.1          # src/size.h:82, ensemble conformers closer than this are dropped
BADKDE = 50               # src/size.h:94, code of an unknown ligand atom type
MCS_INVALID_COORD = 728492.0  # src/size.h:100
MAXMCS = 256              # src/size.h:79
MAXTP2 = abi.MAXTP2

# residue codes (getResCode / getResCodeOne, src/data.C:239-330)
RES3 = ["ALA", "ARG", "CYS", "PRO", "LEU", "ILE", "GLU", "HIS", "TRP", "THR", "MET", "ASP",
        "GLY", "PHE", "LYS", "GLN", "SER", "ASN", "TYR", "VAL"]
RES_CODE = {n: i for i, n in enumerate(RES3)}
RES1 = "ARCPLIEHWTMDGFKQSNYV"
RES1_CODE = {c: i for i, c in enumerate(RES1)}

# effective-point codes (getPntCode, src/data.C:380-445)
PNT = ["CA", "PP", "A1", "C1", "D1", "E1", "E2", "F1", "F2", "H1", "H2", "I1", "K1", "K2", "L1",
       "M1", "M2", "N1", "P1", "Q1", "Q2", "R1", "R2", "S1", "T1", "V1", "W1", "W2", "Y1", "Y2"]
PNT_CODE = {n: i for i, n in enumerate(PNT)}

# ligand atom types (getLigCode, src/data.C:532-587); anything else is BADKDE
LIG_TYPES = ["Br", "C.1", "C.2", "C.3", "C.ar", "C.cat", "Cl", "F", "I", "N.1", "N.2", "N.3",
             "N.4", "N.am", "N.ar", "N.pl3", "O.2", "O.3", "O.co2", "P.3", "S.2", "S.3", "S.O",
             "S.O2"]
LIG_CODE = {n: i for i, n in enumerate(LIG_TYPES)}

# side-chain effective points of each residue code: (point type, point class), in the order
# the reference pushes them (src/load.C:985-1055); glycine has none
SIDE_POINTS = {
    0: [(2, 2)], 1: [(21, 2), (22, 3)], 2: [(3, 2)], 3: [(18, 2)], 4: [(14, 2)], 5: [(11, 2)],
    6: [(5, 2), (6, 3)], 7: [(9, 2), (10, 3)], 8: [(26, 2), (27, 3)], 9: [(24, 2)],
    10: [(15, 2), (16, 3)], 11: [(4, 2)], 12: [], 13: [(7, 2), (8, 3)], 14: [(12, 2), (13, 3)],
    15: [(19, 2), (20, 3)], 16: [(23, 2)], 17: [(17, 2)], 18: [(28, 2), (29, 3)],
    19: [(25, 2)],
}
# which atoms of the residue make up a point of each type (src/load.C:1095-1141)
_BACKBONE = {" N  ", " CA ", " C  ", " O  "}
_ONE_BEAD = {2, 3, 4, 11, 14, 17, 18, 23, 24, 25}       # every side-chain atom
_DISTAL = {5, 7, 9, 12, 15, 19, 21, 26, 28}             # side chain beyond CG
_PROXIMAL = {6, 8, 10, 13, 16, 20, 22, 27, 29}          # CB and CG


class LoadError(ValueError):
    """A file the reference would reject (it prints a message and exits)."""


_NUM = re.compile(r"[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)",
                  re.IGNORECASE)
_INT = re.compile(r"[+-]?\d+")


def c_atof(s: str) -> float:
    """C atof: leading white space skipped, the longest numeric prefix, 0.0 when there is none."""
    m = _NUM.match(s.lstrip(" \t\n\r\f\v"))
    return float(m.group(0)) if m else 0.0


def c_atoi(s: str) -> int:
    m = _INT.match(s.lstrip(" \t\n\r\f\v"))
    return int(m.group(0)) if m else 0


def _f(s: str) -> np.float32:
    """atof stored into a float (double -> nearest float)."""
    return F32(c_atof(s))


def _is_float(s: str) -> bool:
    """is_float (src/load.C:1288-1294): the whole token, without leading white space, is a
    number as istream >> float reads it."""
    if not s or s[0].isspace():
        return False
    m = _NUM.fullmatch(s)
    return m is not None and not s.lower().lstrip("+-").startswith(("inf", "nan"))


def _lines(path: str) -> List[str]:
    """getline semantics: lines without their '\\n' (a final line without one is kept)."""
    try:
        with open(path, "r", errors="replace", newline="") as f:
            text = f.read()
    except OSError as e:
        raise LoadError("cannot open %s: %s" % (path, e))
    out = text.split("\n")
    if out and out[-1] == "":
        out.pop()
    return out


# ------------------------------------------------------------------------------------------
# energy parameters


def load_enepara(path: str) -> abi.EneParaRaw:
    """loadEnePara (src/load.C:1477-1660): the raw parameter set, hydrophobicity scale
    normalised to [-1, 1]."""
    ep = abi.EneParaRaw()
    for line in _lines(path):
        if len(line) <= 3:
            continue
        key = line[:3]
        tok = line.split()
        if key == "VDW":
            p, l = PNT_CODE.get(tok[1]), LIG_CODE.get(tok[2], BADKDE)
            if p is None:
                raise LoadError("unknown effective point %r" % tok[1])
            if l < MAXTP2:  # the reference writes past the row for unknown types
                ep.vdw[p][l][0] = _f(tok[3])
                ep.vdw[p][l][1] = _f(tok[4])
        elif key in ("WEI", "NOA", "NOB"):
            if len(tok) != abi.MAXWEI:
                raise LoadError("%s line needs %d fields" % (key, abi.MAXWEI))
            dst = {"WEI": ep.w, "NOA": ep.a_para, "NOB": ep.b_para}[key]
            for i in range(len(tok) - 1):
                dst[i] = _f(tok[i + 1])
        elif key == "PLJ":
            for i in range(3):
                ep.lj[i] = _f(tok[i + 1])
        elif key == "ELE":
            name = tok[1]
            if name[1:2] != "C":
                p = PNT_CODE.get(name)
                if p is None:
                    raise LoadError("unknown effective point %r" % name)
                ep.ele[p] = _f(tok[2])
            else:
                r = RES1_CODE.get(name[:1])
                if r is None:
                    raise LoadError("unknown residue %r" % name[:1])
                ep.ele[r + 30] = _f(tok[2])
        elif key == "PEL":
            for i in range(2):
                ep.el[i] = _f(tok[i + 1])
        elif key == "PMF":
            p, l = PNT_CODE.get(tok[1]), LIG_CODE.get(tok[2], BADKDE)
            if p is None:
                raise LoadError("unknown effective point %r" % tok[1])
            if l < MAXTP2:  # the reference writes past the row for unknown types
                ep.pmf[p][l][0] = _f(tok[3])
                ep.pmf[p][l][1] = _f(tok[4])
        elif key == "HPP":
            r = RES1_CODE.get(tok[1])
            if r is None:
                raise LoadError("unknown residue %r" % tok[1])
            ep.hpp[r] = _f(tok[2])
        elif key == "HPL":
            l = LIG_CODE.get(tok[1], BADKDE)
            if l < MAXTP2:
                ep.hpl[l][0] = _f(tok[2])
                ep.hpl[l][1] = _f(tok[3])
        elif key == "HDB":
            p, l = PNT_CODE.get(tok[1]), LIG_CODE.get(tok[2], BADKDE)
            if p is None:
                raise LoadError("unknown effective point %r" % tok[1])
            if l < MAXTP2:  # the reference writes past the row for unknown types
                ep.hdb[p][l][0] = _f(tok[3])
                ep.hdb[p][l][1] = _f(tok[4])
        elif key == "KDE":
            ep.kde = _f(tok[1])
    # min-max normalisation of the hydrophobicity scale: float differences and quotient, the
    # affine map in double (the literals are doubles), stored as float and clamped
    lo, hi = F32(1e6), F32(-1e6)
    hpp = [F32(ep.hpp[i]) for i in range(abi.MAXTP4)]
    for v in hpp:
        lo = v if v < lo else lo
        hi = v if v > hi else hi
    for i, v in enumerate(hpp):
        q = F32(F32(v - lo) / F32(hi - lo))
        n = F32(float(q) * 2.0 - 1.0)
        n = F32(-1.0) if n < -1.0 else (F32(1.0) if n > 1.0 else n)
        ep.hpp[i] = n
    return ep


# ------------------------------------------------------------------------------------------
# protein


@dataclass
class Protein:
    """Effective points of every conformation (Protein0, src/dock.h)."""
    r: np.ndarray      # [pnp] residue index of the point
    t: np.ndarray      # [pnp] point type
    d: np.ndarray      # [pnp] residue code
    c: np.ndarray      # [pnp] point class
    seq3: np.ndarray   # [pnr] residue serial numbers
    x: np.ndarray      # [n_conf, pnp]
    y: np.ndarray
    z: np.ndarray

    @property
    def pnp(self):
        return self.t.shape[0]

    @property
    def n_conf(self):
        return self.x.shape[0]


def load_weights(path: str) -> np.ndarray:
    """loadWeight (src/load.C:1762-1794): one term weight per line, the number at the start of
    its first 30 characters (0 where there is none)."""
    out = []
    for line in _lines(path):
        tok = line[:30].split()
        v = np.float32(0.0)
        if tok:
            m = re.match(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?", tok[0])
            if m:
                v = np.float32(float(m.group(0)))
        out.append(v)
    return np.asarray(out, F32)


def _pdb_points(lines: Sequence[str]):
    """The point list of the first model (src/load.C:965-1060)."""
    r, t, d, c, seq3 = [], [], [], [], []
    for line in lines:
        if len(line) > 53:
            if line[:6] == "ATOM  " and line[12:16] == " CA ":
                name = line[17:20]
                code = RES_CODE.get(name)
                if code is None:
                    raise LoadError("unknown residue %r" % name)
                pnr = len(seq3)
                seq3.append(c_atoi(line[22:26]))
                r.append(pnr); t.append(0); d.append(code); c.append(0)
                if pnr > 1:
                    r.append(pnr - 1); t.append(1); d.append(code); c.append(1)
                for pt, pc in SIDE_POINTS[code]:
                    r.append(pnr); t.append(pt); d.append(code); c.append(pc)
        elif line[:6] == "ENDMDL":
            break
    i32 = lambda a: np.asarray(a, np.int32)
    return i32(r), i32(t), i32(d), i32(c), i32(seq3)


def _point_takes(pt: int, atom: str) -> bool:
    if pt == 0:
        return atom == " CA "
    if pt in _ONE_BEAD:
        return atom not in _BACKBONE
    if pt in _DISTAL:
        return atom not in _BACKBONE and atom not in (" CB ", " CG ")
    if pt in _PROXIMAL:
        return atom in (" CB ", " CG ")
    return False


def load_protein(path: str) -> Protein:
    """loadProtein (src/load.C:931-1265): each effective point is the float mean of its atoms
    (CA; side-chain beads; the peptide plane N(i) + C(i-1) + O(i-1)), one conformation per
    block ended by an ENDMDL or TER line."""
    lines = _lines(path)
    r, t, d, c, seq3 = _pdb_points(lines)
    pnr = seq3.shape[0]
    pnp = t.shape[0]
    # atoms by residue serial, in file order, with the block (conformation) they belong to
    by_serial: Dict[int, List[Tuple[int, int, str, np.float32, np.float32, np.float32]]] = {}
    block = 0
    n_blocks = 0
    for li, line in enumerate(lines):
        if len(line) > 53:
            if line[:6] == "ATOM  ":
                s = c_atoi(line[22:26])
                by_serial.setdefault(s, []).append(
                    (li, block, line[12:16], _f(line[30:38]), _f(line[38:46]), _f(line[46:54])))
        elif line[:6] == "ENDMDL" or line[:3] == "TER":
            block += 1
            n_blocks = max(n_blocks, block)
    if n_blocks == 0:
        raise LoadError("%s: no ENDMDL or TER line ends a conformation" % path)
    x = np.zeros((n_blocks, pnp), F32)
    y = np.zeros((n_blocks, pnp), F32)
    z = np.zeros((n_blocks, pnp), F32)
    for p in range(pnp):
        pt, rp = int(t[p]), int(r[p])
        s3 = int(seq3[rp])
        atoms = [a for a in by_serial.get(s3, ()) if _point_takes(pt, a[2])]
        if pt == 1 and 0 < rp < pnr - 1:
            # The reference looks the previous residue's serial up in the record of the
            # conformation before the one being read (src/load.C:1143-1146), which holds the
            # point list only for conformation 0; from the third conformation on it reads a
            # zeroed record, i.e. serial 0. The peptide-plane point of those conformations is
            # therefore N(i) plus C / O of a residue numbered 0 (usually none).
            s6 = int(seq3[rp - 1])
            atoms = [a for a in by_serial.get(s3, ()) if a[2] == " N  "]
            atoms += [a for a in by_serial.get(s6, ()) if a[2] in (" C  ", " O  ") and a[1] < 2]
            atoms += [a for a in by_serial.get(0, ()) if a[2] in (" C  ", " O  ") and a[1] >= 2]
            atoms.sort(key=lambda a: a[0])
        sx = [F32(0.0)] * n_blocks
        sy = [F32(0.0)] * n_blocks
        sz = [F32(0.0)] * n_blocks
        sn = [F32(0.0)] * n_blocks
        for (_, b, _, ax, ay, az) in atoms:
            if b >= n_blocks:  # after the last ENDMDL / TER: never stored
                continue
            sx[b] = F32(sx[b] + ax)
            sy[b] = F32(sy[b] + ay)
            sz[b] = F32(sz[b] + az)
            sn[b] = F32(sn[b] + F32(1.0))
        for b in range(n_blocks):
            if sn[b] > 0:
                x[b, p] = F32(sx[b] / sn[b])
                y[b, p] = F32(sy[b] / sn[b])
                z[b, p] = F32(sz[b] / sn[b])
    return Protein(r=r, t=t, d=d, c=c, seq3=seq3, x=x, y=y, z=z)


# ------------------------------------------------------------------------------------------
# ligand


@dataclass
class Ligand:
    """The ligand's conformers (Ligand0, src/dock.h), centred on their own centroid."""
    t: np.ndarray   # [lna] atom type codes
    c: np.ndarray   # [lna] partial charges
    n: np.ndarray   # [lna] atom numbers
    x: np.ndarray   # [n_conf, lna]
    y: np.ndarray
    z: np.ndarray
    props: Dict[str, str]

    @property
    def lna(self):
        return self.t.shape[0]

    @property
    def n_conf(self):
        return self.x.shape[0]


def _sdf_sections(lines: Sequence[str]) -> List[List[str]]:
    secs, cur = [], []
    for line in lines:
        cur.append(line)
        if line == "$$$$":
            secs.append(cur)
            cur = []
    return secs


def sdf_records(path: str) -> List[List[str]]:
    """readLigandSections (src/load.C:428-446): the file's records, each the lines up to and
    including its `$$$$`."""
    return _sdf_sections(_lines(path))


def ligand_header(sect: Sequence[str]) -> Tuple[int, int]:
    """writeLigProperty's counts (src/load.C:388-426): atoms and bonds from the counts line."""
    if len(sect) < 4:
        raise LoadError("truncated SDF header")
    return c_atoi(sect[3][0:3]), c_atoi(sect[3][3:6])


def atom_block(sect: Sequence[str], lna: int):
    """writeDefaultLigAtomCoord (src/load.C:302-320): the atom block's coordinates as read
    (columns 1-30)."""
    if lna < 1 or 4 + lna > len(sect):
        raise LoadError("bad atom count %d" % lna)
    return (np.asarray([_f(sect[4 + i][0:10]) for i in range(lna)], F32),
            np.asarray([_f(sect[4 + i][10:20]) for i in range(lna)], F32),
            np.asarray([_f(sect[4 + i][20:30]) for i in range(lna)], F32))


def ensemble(sect: Sequence[str]) -> Tuple[List[float], List[str]]:
    """getLigEnsembleRmsd / getLigEnsembleCoords (src/load.C:108-156): the ENSEMBLE_RMSD values
    (the lines after the tag while they start with a digit) and the ENSEMBLE_COORDS rows (the
    lines after the tag up to an empty one)."""
    rmsds: List[float] = []
    coords: List[str] = []
    for i, line in enumerate(sect):
        if "ENSEMBLE_RMSD" in line:
            j = i + 1
            while j < len(sect) and sect[j][:1].isdigit():
                rmsds += [c_atof(tok) for tok in sect[j].split()]
                j += 1
        if "ENSEMBLE_COORDS" in line:
            j = i + 1
            while j < len(sect) and sect[j] != "":
                coords.append(sect[j])
                j += 1
    return rmsds, coords


def ensemble_coords(row: str, lna: int):
    """writeEnsAtomCoord (src/load.C:284-300): one ENSEMBLE_COORDS row as x y z triples
    (missing atoms at 0)."""
    v = [_f(tok) for tok in row.split()]
    if len(v) % 3:
        raise LoadError("an ENSEMBLE_COORDS row is not x y z triples")
    xs = np.zeros(lna, F32); ys = np.zeros(lna, F32); zs = np.zeros(lna, F32)
    for k in range(min(len(v) // 3, lna)):
        xs[k], ys[k], zs[k] = v[3 * k], v[3 * k + 1], v[3 * k + 2]
    return xs, ys, zs


def centre(x: np.ndarray, y: np.ndarray, z: np.ndarray):
    """moveLigand2ItsCenterFrame (src/load.C:239-260): float sums, float means, subtract."""
    lna = x.shape[0]
    sx = sy = sz = F32(0.0)
    for i in range(lna):
        sx = F32(sx + x[i]); sy = F32(sy + y[i]); sz = F32(sz + z[i])
    cx, cy, cz = F32(sx / F32(lna)), F32(sy / F32(lna)), F32(sz / F32(lna))
    return (np.asarray([F32(v - cx) for v in x], F32), np.asarray([F32(v - cy) for v in y], F32),
            np.asarray([F32(v - cz) for v in z], F32))


def ensemble_total(sect: Sequence[str]) -> int:
    """getLigEnsembleTotal (src/load.C:262-279): the integer on the line after the last
    ENSEMBLE_TOTAL tag (a record without one is an error, where the reference exits)."""
    tot = -1
    for i, line in enumerate(sect):
        if "ENSEMBLE_TOTAL" in line:
            tot = c_atoi(sect[i + 1] if i + 1 < len(sect) else "")
    if tot == -1:
        raise LoadError("no ENSEMBLE_TOTAL")
    return tot


def pocket_center(path: str) -> np.ndarray:
    """loadPocketCenter (src/load.C:1326-1343): x y z of the last line holding CENTER."""
    center_line = None
    for line in _lines(path):
        if "CENTER" in line:
            center_line = line
    if center_line is None:
        raise LoadError("%s: no CENTER line" % path)
    tok = center_line.split()
    if len(tok) < 4:
        raise LoadError("%s: CENTER line with fewer than three values" % path)
    return np.asarray([_f(tok[1]), _f(tok[2]), _f(tok[3])], F32)


def ligand_conformers(sect: Sequence[str], lna: int) -> List[Tuple[np.ndarray, ...]]:
    """loadOneLigand's conformers as read, before centring (src/load.C:200-227): the atom
    block, then every ENSEMBLE_COORDS row whose ENSEMBLE_RMSD is above 0.1 A."""
    confs = [atom_block(sect, lna)]
    rmsds, coords = ensemble(sect)
    if len(rmsds) != len(coords):
        raise LoadError("%d ENSEMBLE_RMSD values for %d ENSEMBLE_COORDS rows" %
                        (len(rmsds), len(coords)))
    for rm, row in zip(rmsds, coords):
        # rmsd values are compared as floats against the double threshold
        if float(F32(rm)) > MINLIGRMSD:
            confs.append(ensemble_coords(row, lna))
    return confs


def load_ligand(path: str) -> Ligand:
    """loadLigand / loadOneLigand (src/load.C:157-230): the first SDF record; conformer 0 is
    the atom block, the others are the ENSEMBLE_COORDS rows whose ENSEMBLE_RMSD is above
    0.1 A; every conformer is centred on its own centroid."""
    secs = sdf_records(path)
    if not secs:
        raise LoadError("%s: no SDF record ($$$$)" % path)
    sect = secs[0]
    try:
        lna, lnb = ligand_header(sect)
        if lna < 1 or 4 + lna > len(sect):
            raise LoadError("bad atom count %d" % lna)
    except LoadError as ex:
        raise LoadError("%s: %s" % (path, ex))
    start = 4 + lna + lnb
    types: List[int] = []
    charges: List[np.float32] = []
    props: Dict[str, str] = {}
    for i in range(start, len(sect)):
        line = sect[i]
        nxt = sect[i + 1] if i + 1 < len(sect) else ""
        if "OB_ATOM_TYPES" in line:
            types = [LIG_CODE.get(tok, BADKDE) for tok in nxt.split()]
        elif "OB_ATOMIC_CHARGES" in line or "OB_CHARGES" in line:
            charges = [_f(tok) for tok in nxt.split()]
        for key in ("MOLID", "SMILES_CANONICAL", "OB_MW", "OB_logP", "OB_PSA", "OB_MR",
                    "MCT_HBD", "MCT_HBA"):
            if key in line:
                props[key] = nxt
    if len(types) < lna or len(charges) < lna:
        raise LoadError("%s: OB_ATOM_TYPES / OB_ATOMIC_CHARGES shorter than %d atoms" %
                        (path, lna))
    try:
        confs = ligand_conformers(sect, lna)
    except LoadError as ex:
        raise LoadError("%s: %s" % (path, ex))
    cx = [centre(*cf) for cf in confs]
    return Ligand(t=np.asarray(types[:lna], np.int32), c=np.asarray(charges[:lna], F32),
                  n=np.arange(lna, dtype=np.int32),
                  x=np.stack([a for a, _, _ in cx]), y=np.stack([b for _, b, _ in cx]),
                  z=np.stack([q for _, _, q in cx]), props=props)


# ------------------------------------------------------------------------------------------
# pocket file (.ff)


@dataclass
class Pocket:
    center: np.ndarray                  # [3] CENTER
    kde_t: np.ndarray                   # [pnk]
    kde_x: np.ndarray
    kde_y: np.ndarray
    kde_z: np.ndarray
    psp: Dict[Tuple[int, int], np.float32]  # (residue serial, ligand type) -> value
    mcs_tcc: np.ndarray                 # [pos]
    mcs_x: np.ndarray                   # [pos, MAXMCS]
    mcs_y: np.ndarray
    mcs_z: np.ndarray


def load_pocket(path: str, ligand_id: str) -> Pocket:
    """loadPocketCenter + loadLHM (src/load.C:1270-1450): the last CENTER line; KDE points;
    PSP entries; MCS restraints (`MCS <id> <tcc> <n> (atom x y z)*n` when the id is the
    ligand's, else one more leading field), atoms without a restraint at 728492."""
    lines = _lines(path)
    center_line = None
    for line in lines:
        if "CENTER" in line:
            center_line = line
    if center_line is None:
        raise LoadError("%s: no CENTER line" % path)
    tok = center_line.split()
    center = np.asarray([_f(tok[1]), _f(tok[2]), _f(tok[3])], F32)
    kt, kx, ky, kz = [], [], [], []
    psp: Dict[Tuple[int, int], np.float32] = {}
    tcc, mx, my, mz = [], [], [], []
    for line in lines:
        if len(line) <= 3:
            continue
        key = line[:3]
        d = line.split()
        if key == "KDE":
            kt.append(LIG_CODE.get(d[1], BADKDE))
            kx.append(_f(d[2])); ky.append(_f(d[3])); kz.append(_f(d[4]))
        elif key == "PSP":
            psp[(c_atoi(d[1]), LIG_CODE.get(d[2], BADKDE))] = _f(d[3])
        elif key == "MCS":
            d = d[:MAXMCS]
            own = len(d) > 2 and d[1] == ligand_id and _is_float(d[2])
            o = 4 if own else 5
            tcc.append(_f(d[2] if own else (d[3] if len(d) > 3 else "")))
            total = c_atoi(d[3] if own else (d[4] if len(d) > 4 else ""))
            ax = np.full(MAXMCS, MCS_INVALID_COORD, F32)
            ay = ax.copy(); az = ax.copy()
            for ia in range(total):
                g = lambda k: d[o + ia * 4 + k] if o + ia * 4 + k < len(d) else ""
                idx = c_atoi(g(0))
                if not 0 <= idx < MAXMCS:
                    raise LoadError("%s: MCS atom index %d outside 0..%d" % (path, idx, MAXMCS - 1))
                ax[idx], ay[idx], az[idx] = _f(g(1)), _f(g(2)), _f(g(3))
            mx.append(ax); my.append(ay); mz.append(az)
    f32 = lambda a: np.asarray(a, F32)
    return Pocket(center=center, kde_t=np.asarray(kt, np.int32), kde_x=f32(kx), kde_y=f32(ky),
                  kde_z=f32(kz), psp=psp, mcs_tcc=f32(tcc),
                  mcs_x=np.asarray(mx, F32).reshape(-1, MAXMCS),
                  mcs_y=np.asarray(my, F32).reshape(-1, MAXMCS),
                  mcs_z=np.asarray(mz, F32).reshape(-1, MAXMCS))


# ------------------------------------------------------------------------------------------
# folds into the library's arrays


def complex_arrays(prt: Protein, lig: Ligand, pocket: Pocket, raw: abi.EneParaRaw,
                   temp: np.ndarray) -> abi.ComplexArrays:
    """OptimizeLigand / OptimizeProtein (CopyProteinResidue) / OptimizePsp / OptimizeKde /
    OptimizeMcs (src/util.C:264-290, 574-715) into the library's complex arrays."""
    n_lig, lna = lig.n_conf, lig.lna
    lig_center = np.tile(pocket.center, (n_lig, 1)).astype(F32)
    t, d, c, r = prt.t, prt.d, prt.c, prt.r
    ele_tab = np.asarray(raw.ele, F32)
    hpp_tab = np.asarray(raw.hpp, F32)
    dt = np.where(t == 0, d + 30, t)
    ele = np.tile(ele_tab[dt], (prt.n_conf, 1))
    seq3r = np.tile(prt.seq3[r], (prt.n_conf, 1)).astype(np.int32)
    hflag = np.tile(((c == 0) & (d == 12)) | (c == 2), (prt.n_conf, 1)).astype(np.int32)
    hpp = np.tile(hpp_tab[d], (prt.n_conf, 1))
    ld = int(seq3r.max()) + 1 if seq3r.size else 1
    psp = np.zeros((MAXTP2, ld), F32)
    for (s, lt), v in pocket.psp.items():
        if 0 <= lt < MAXTP2 and 0 <= s < ld:
            psp[lt, s] = v
    return abi.ComplexArrays(
        lig_x=lig.x, lig_y=lig.y, lig_z=lig.z, lig_center=lig_center,
        lig_t=np.tile(lig.t, (n_lig, 1)), lig_c=np.tile(lig.c, (n_lig, 1)),
        lig_n=np.tile(lig.n, (n_lig, 1)),
        prt_x=prt.x, prt_y=prt.y, prt_z=prt.z, prt_t=np.tile(t, (prt.n_conf, 1)),
        prt_c=np.tile(c, (prt.n_conf, 1)), prt_ele=ele, prt_seq3r=seq3r, prt_hflag=hflag,
        prt_hpp=hpp, pocket_center=pocket.center, psp=psp,
        kde_x=pocket.kde_x, kde_y=pocket.kde_y, kde_z=pocket.kde_z, kde_t=pocket.kde_t,
        mcs_x=pocket.mcs_x, mcs_y=pocket.mcs_y, mcs_z=pocket.mcs_z, mcs_tcc=pocket.mcs_tcc,
        temp=temp)


def load_complex(pdb: str, sdf: str, ff: str, paras: str, ligand_id: str, n_tmp: int,
                 floor_temp: float, ceiling_temp: float):
    """The reference's load-and-fold sequence (src/dock.C:97-181): returns
    (ComplexArrays, folded EnePara, raw EneParaRaw)."""
    from .engine import fold_enepara, set_temperature
    raw = load_enepara(paras)
    prt = load_protein(pdb)
    lig = load_ligand(sdf)
    pocket = load_pocket(ff, ligand_id)
    temp = set_temperature(n_tmp, floor_temp, ceiling_temp)
    return complex_arrays(prt, lig, pocket, raw, temp), fold_enepara(raw), raw
