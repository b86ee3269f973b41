"""Convert the reference's sample trajectory of 1a07C1 into the committed fixture
tests/golden/trajectory_1a07C1.npz, with the reference's own trace program run on every 13th
row of it:

  python tests/golden/make_trajectory.py [--reference /path/to/geaxdock_gpu]

data/trajectory.out is the text that printLigandTrajectories (src/util.C:2041-2056) writes for
accepted steps: one row per step, `PrtIdx LigIdx v1..v6 cms ener`, with the move vector,
the contact fraction and the weighted total energy each printed with %f. The rows are stored
unchanged as float64 (every printed value is exact in float64 to its six decimals).

`trace_rows` / `trace_xyz`: oracle/_ref/refpin --trace (the reference's read2D, PlaceLigand and
replaceLigandCoords, src/trace.C:90-122, built from its sources by oracle/refpin/Makefile) on
those rows; the placed atoms as the SDF lines print them (%10.4f), stored in units of 1e-4.
"""
import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import reference_root  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())
    a = ap.parse_args()
    src = os.path.join(a.reference, "data", "trajectory.out")
    with open(src) as f:
        head = f.readline().split()
        assert head == ["PrtIdx", "LigIdx", "v1", "v2", "v3", "v4", "v5", "v6", "cms", "ener"], head
        rows = np.array([[float(v) for v in line.split()] for line in f if line.strip()], np.float64)
    repo = os.path.dirname(os.path.dirname(HERE))
    subprocess.run(["make", "-s", "-C", os.path.join(repo, "oracle"), "refpin",
                    "REFERENCE=" + a.reference], check=True)
    ref = os.path.join(repo, "oracle", "_ref")
    pick = np.arange(0, rows.shape[0], 13)
    sel = os.path.join(ref, "trace_rows.txt")
    with open(sel, "w") as f:
        for i in pick:
            f.write("%d %d " % (rows[i, 0], rows[i, 1]) +
                    " ".join("%f" % v for v in rows[i, 2:]) + "\n")
    out = os.path.join(ref, "trace_1a07C1.txt")
    d = os.path.join(a.reference, "data", "1a07C1")
    subprocess.run([os.path.join(ref, "refpin"), "--pdb", os.path.join(d, "1a07C.pdb"),
                    "--sdf", os.path.join(d, "1a07C1.sdf"), "--ff", os.path.join(d, "1a07C1-0.8.ff"),
                    "--paras", os.path.join(a.reference, "data", "parameters", "paras"),
                    "--id", "1a07C1", "--nt", "1", "--trace", sel, "--out", out],
                   check=True, stdout=subprocess.DEVNULL)
    blocks = open(out).read().split(">>>> row ")[1:]
    assert len(blocks) == pick.shape[0], (len(blocks), pick.shape[0])
    lna = int(blocks[0].split("\n")[4][0:3])
    xyz = np.zeros((len(blocks), lna, 3), np.int32)
    for k, b in enumerate(blocks):
        lines = b.split("\n")[1:]
        for j in range(lna):
            ln = lines[4 + j]
            xyz[k, j] = [round(float(ln[c:c + 10]) * 1e4) for c in (0, 10, 20)]
    dst = os.path.join(HERE, "trajectory_1a07C1.npz")
    np.savez_compressed(dst, rows=rows, trace_rows=pick.astype(np.int32), trace_xyz=xyz)
    print(rows.shape[0], "rows,", os.path.getsize(dst), "bytes", file=sys.stderr)


if __name__ == "__main__":
    main()
