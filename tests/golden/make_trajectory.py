"""Convert the reference's sample trajectory of 1a07C1 into the committed fixture
tests/golden/trajectory_1a07C1.npz:

  python tests/golden/make_trajectory.py [--reference /path/to/geaxdock_gpu]

data/trajectory.out is the text that printLigandTrajectories (src/util.C:2041-2056) writes for
accepted steps: one row per step, `PrtIdx LigIdx v1..v6 cms ener`, with the move vector,
the contact fraction and the weighted total energy each printed with %f. The rows are stored
unchanged as float64 (every printed value is exact in float64 to its six decimals).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    a = ap.parse_args()
    src = os.path.join(a.reference, "data", "trajectory.out")
    with open(src) as f:
        head = f.readline().split()
        assert head == ["PrtIdx", "LigIdx", "v1", "v2", "v3", "v4", "v5", "v6", "cms", "ener"], head
        rows = np.array([[float(v) for v in line.split()] for line in f if line.strip()], np.float64)
    dst = os.path.join(HERE, "trajectory_1a07C1.npz")
    np.savez_compressed(dst, rows=rows)
    print(rows.shape[0], "rows,", os.path.getsize(dst), "bytes", file=sys.stderr)


if __name__ == "__main__":
    main()
