"""Generate the golden fixtures under tests/golden/ from the reference's own code.

Builds oracle/_ref/refpin (the reference's loaders, host folds, kernel source and k-means
module compiled for the CPU; see oracle/refpin/) and runs it on the reference's real complexes
and on the k-means module's sample data. Each run writes a .gdfx container that this script
converts to a compressed .npz:

  python tests/golden/make_golden.py [--reference /path/to/geaxdock_gpu]

Needs the reference tree; the committed .npz files are what the tests read.
"""
import argparse
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from oracle import reference_root  # noqa: E402

RUNS = {
    # name: (data dir, pdb, sdf, ff, id, n_tmp, floor, ceil, n_exchanges, n_poses)
    "1a07C1": ("1a07C1", "1a07C.pdb", "1a07C1.sdf", "1a07C1-0.8.ff", "1a07C1", 4, 0.5, 2.0, 3, 64),
    "1robA1": ("1robA1", "1robA.pdb", "1robA1.sdf", "1robA1-0.8.ff", "1robA1", 2, 0.5, 1.0, 1, 48),
}


def read_gdfx(path):
    out = {}
    with open(path, "rb") as f:
        assert f.read(6) == b"GDFX1\n"
        while True:
            h = f.read(4)
            if not h:
                break
            n = struct.unpack("<I", h)[0]
            name = f.read(n).decode()
            dt = f.read(1).decode()
            nd = struct.unpack("<I", f.read(4))[0]
            dims = struct.unpack("<%dQ" % nd, f.read(8 * nd))
            dtype = {"f": np.float32, "i": np.int32, "d": np.float64, "b": np.uint8}[dt]
            cnt = int(np.prod(dims)) if dims else 1
            out[name] = np.frombuffer(f.read(cnt * np.dtype(dtype).itemsize), dtype=dtype).reshape(dims)
    return out


# cluster_test's run (src/cluster_test.C:23-66) on the vendored k-means module's text data:
# name -> (data file under src/modules/kmeans-master/Image_data, clusters)
KMEANS = {"edge100": ("edge100.txt", 10), "color100": ("color100.txt", 10),
          "texture100": ("texture100.txt", 10)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())
    a = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "refpin",
                    "REFERENCE=" + a.reference], check=True)
    binp = os.path.join(REPO, "oracle", "_ref", "refpin")
    data = os.path.join(a.reference, "data")
    for name, (d, pdb, sdf, ff, cid, nt, fl, ce, nex, npo) in RUNS.items():
        tmp = os.path.join(REPO, "oracle", "_ref", name + ".gdfx")
        cmd = [binp, "--pdb", os.path.join(data, d, pdb), "--sdf", os.path.join(data, d, sdf),
               "--ff", os.path.join(data, d, ff), "--paras", os.path.join(data, "parameters", "paras"),
               "--id", cid, "--nt", str(nt), "--floor", str(fl), "--ceil", str(ce), "--nc", "10",
               "--nex", str(nex), "--seed", "42", "--poses", str(npo), "--out", tmp]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        arrs = read_gdfx(tmp)
        dst = os.path.join(HERE, "ref_%s.npz" % name)
        np.savez_compressed(dst, **arrs)
        print(name, os.path.getsize(dst), "bytes", file=sys.stderr)
    km = {}
    for name, (fname, k) in KMEANS.items():
        tmp = os.path.join(REPO, "oracle", "_ref", "kmeans_%s.gdfx" % name)
        src = os.path.join(a.reference, "src", "modules", "kmeans-master", "Image_data", fname)
        subprocess.run([binp, "--kmeans", src, "--k", str(k), "--out", tmp], check=True,
                       stdout=subprocess.DEVNULL)
        for key, v in read_gdfx(tmp).items():
            km["%s_%s" % (name, key)] = v
    dst = os.path.join(HERE, "kmeans_ref.npz")
    np.savez_compressed(dst, **km)
    print("kmeans", os.path.getsize(dst), "bytes", file=sys.stderr)


if __name__ == "__main__":
    main()
