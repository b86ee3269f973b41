"""Golden output of the reference's printStates (src/util.C:1504-1545), the trajectory table of
the `dock` program, for tests/golden/states_ref.npz:

  python tests/golden/make_states.py [--reference /path/to/geaxdock_gpu]

Builds oracle/_ref/refpin (the reference's sources compiled for the CPU, see oracle/refpin/),
writes 300 seeded records in the LigRecordSingleStep layout (values of every magnitude the
table meets, with signed zeros, values that round to zero from below and 4-decimal rounding
ties), lets the reference's printStates write the table, and stores records and table.
"""
import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from geaxdock_gpu_b200 import abi  # noqa: E402
from oracle import reference_root


def records(n=300, seed=9):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, abi.RECORD_DTYPE)
    r["replica"]["idx_rep"] = rng.integers(0, 7000, n)
    r["replica"]["idx_prt"] = rng.integers(0, 11, n)
    r["replica"]["idx_tmp"] = rng.integers(0, 20, n)
    r["replica"]["idx_lig"] = rng.integers(0, 31, n)
    mag = 10.0 ** rng.integers(-6, 5, (n, 10))
    r["energy"]["e"] = (rng.normal(0, 1, (n, 10)) * mag).astype(np.float32)
    r["energy"]["cms"] = rng.uniform(0, 1, n).astype(np.float32)
    r["energy"]["rmsd"] = rng.uniform(0, 30, n).astype(np.float32)
    r["movematrix"] = (rng.normal(0, 1, (n, 6)) * 10.0 ** rng.integers(-5, 3, (n, 6))).astype(
        np.float32)
    r["step"] = rng.integers(0, 20000, n)
    special = np.array([0.0, -0.0, -0.00004, 0.00005, -0.00005, 0.12345, 2.5e-5, -1e-9,
                        12345.6789, -3.14159], np.float32)
    r["energy"]["e"][:10] = special[None, :]
    r["movematrix"][10:20] = special[:6][None, :]
    r["energy"]["cms"][20:30] = special[:10]
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())
    a = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "refpin",
                    "REFERENCE=" + a.reference], check=True)
    ref = os.path.join(REPO, "oracle", "_ref")
    rec = records()
    src = os.path.join(ref, "states_in.bin")
    out = os.path.join(ref, "states_out.txt")
    rec.tofile(src)
    subprocess.run([os.path.join(ref, "refpin"), "--states", src, "--out", out], check=True,
                   stdout=subprocess.DEVNULL)
    with open(out, "rb") as f:
        text = f.read()
    dst = os.path.join(HERE, "states_ref.npz")
    np.savez_compressed(dst, records=np.frombuffer(rec.tobytes(), np.uint8),
                        table=np.frombuffer(text, np.uint8))
    print(rec.shape[0], "records,", os.path.getsize(dst), "bytes", file=sys.stderr)


if __name__ == "__main__":
    main()
