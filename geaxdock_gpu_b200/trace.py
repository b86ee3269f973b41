"""The reference's `trace` program on this library:

    python -m geaxdock_gpu_b200.trace -p prt.pdb -l lig.sdf -s pocket.ff -para paras \\
        -id <complex id> -tr trajectory.out -lc <output prefix> [-device 0]

Same options and output as src/trace.C:18-136 with the hand parser of src/util.C:107-262:
load the complex, read the trajectory rows (read2D, src/load.C:80-105: every line whose first
character is a digit, whitespace-separated numbers), and for row k place ligand conformer
int(row[1]) with the move vector row[2:8] (PlaceLigand, src/util.C:457-502; here on the GPU
through gd_place_ligand, the transform the Monte Carlo kernel applies) and write
`<prefix>_<k>.sdf`: the ligand file with the coordinate lines of its first molecule (file
lines 4 .. 3 + lna) replaced by `%10.4f%10.4f%10.4f` of the placed atom and the rest of the
line from column 30 on (replaceLigandCoords, src/util.C:504-545). The protein index row[0]
plays no part, as in the reference.

Error behaviour follows the reference: a missing -p, -l or -s prints the reference's message
and exits 1; an unreadable trajectory prints "Error opening file <path>" and writes nothing;
an unreadable ligand file exits 1. Where the reference reads out of bounds (a row with fewer
than eight numbers, a ligand conformer index outside the ensemble, an atom line shorter than
30 characters) this tool reports the row or line and exits 1. Option of this implementation:
-device (the GPU to place on). Options the reference parses but trace does not use (-na, -nb,
-opt, -ns, -nc, -d, -t, -r, ...) are accepted and ignored.
"""
from __future__ import annotations

import os
import sys
from typing import List

import numpy as np

from . import abi, engine, loaders


class TraceError(Exception):
    pass


# flags of src/util.C:107-262 that take a value
_VALUE_FLAGS = {"-id", "-p", "-l", "-s", "-opt", "-na", "-nb", "-para", "-ns", "-nc",
                "-floor_temp", "-ceiling_temp", "-nt", "-d", "-tr", "-lc", "-t", "-r", "-device"}


def parse(argv: List[str]) -> dict:
    """The hand parser's scan (src/util.C:137-240): each flag takes the next word; later
    occurrences win; unknown words are skipped."""
    a = {"-para": "gpudocksm.ff", "-id": "", "-lc": "", "-tr": "", "-nt": "1",
         "-floor_temp": "0.3", "-ceiling_temp": "0.3", "-device": "0"}
    for i, w in enumerate(argv):
        if w in _VALUE_FLAGS and i + 1 < len(argv):
            a[w] = argv[i + 1]
    return a


def read_trace(path: str) -> List[List[float]]:
    """read2D (src/load.C:80-105): the rows of `path` whose first character is a digit, each
    the leading run of numbers of the line. An unreadable file gives no rows (the reference
    prints the error and carries on)."""
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        print("Error opening file %s" % path)
        return []
    print("reading near native traces from %s" % path)
    rows = []
    for line in text.split("\n"):
        if line[:1].isdigit():
            row = []
            for tok in line.split():
                try:
                    row.append(float(np.float32(tok)))
                except ValueError:
                    break
            rows.append(row)
    return rows


def sdf_lines(path: str) -> List[str]:
    """The ligand file as getline reads it: split at newlines, no trailing empty line."""
    try:
        with open(path, newline="") as f:
            text = f.read()
    except OSError:
        raise TraceError("cannot open ligand file\nCannot open %s" % path)
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    return lines


def replace_ligand_coords(lines: List[str], xyz: np.ndarray) -> List[str]:
    """replaceLigandCoords (src/util.C:504-545): file lines 4 .. 3 + lna take the placed atoms
    (xyz [lna, 3]) as `%10.4f%10.4f%10.4f` followed by the old line from column 30."""
    lna = xyz.shape[0]
    out = list(lines)
    for a in range(lna):
        n = 4 + a
        if n >= len(out):
            break
        old = out[n]
        if len(old) < 30:
            raise TraceError("ligand file line %d is shorter than 30 characters" % (n + 1))
        x, y, z = (float(v) for v in xyz[a])
        out[n] = "%10.4f%10.4f%10.4f" % (x, y, z) + old[30:]
    return out


def run(a: dict) -> int:
    for flag, msg in (("-p", "Provide target protein structure"),
                      ("-l", "Provide compound library in SD format"),
                      ("-s", "Provide LHM potentials")):
        if flag not in a:
            print(msg)
            return 1
    cx, ff, _ = loaders.load_complex(a["-p"], a["-l"], a["-s"], a["-para"], a["-id"],
                                     int(a["-nt"]), float(a["-floor_temp"]),
                                     float(a["-ceiling_temp"]))
    rows = read_trace(a["-tr"])
    template = sdf_lines(a["-l"])
    if not rows:
        return 0
    for k, r in enumerate(rows):
        if len(r) < 8:
            raise TraceError("trajectory row %d has %d numbers, 8 needed" % (k, len(r)))
        lc = int(r[1])
        if not 0 <= lc < cx.n_lig:
            raise TraceError("trajectory row %d: ligand conformer %d outside [0, %d)"
                             % (k, lc, cx.n_lig))
    lig_conf = np.array([int(r[1]) for r in rows])
    mm = np.array([r[2:8] for r in rows], np.float32)
    placed = np.zeros((len(rows), cx.lna, 3), np.float32)
    with engine.Engine(ff, [cx], abi.mc_params(), device=int(a["-device"])) as e:
        for lc in np.unique(lig_conf):
            sel = np.nonzero(lig_conf == lc)[0]
            placed[sel] = e.place_ligand(0, int(lc), mm[sel])
    prefix = a["-lc"]
    for k in range(len(rows)):
        ofn = prefix + "_" + str(k) + ".sdf"
        with open(ofn, "w") as f:
            for line in replace_ligand_coords(template, placed[k]):
                f.write(line + "\n")
        print("write the new ligand conformation to %s" % ofn)
    return 0


def main(argv=None) -> int:
    a = parse(sys.argv[1:] if argv is None else list(argv))
    try:
        return run(a)
    except (loaders.LoadError, TraceError) as ex:
        print("trace: %s" % ex, file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
