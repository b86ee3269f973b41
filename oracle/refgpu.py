"""The reference's own GPU implementation timed on this machine's GPU: a witness beside the
benchmark (benchmark infrastructure, not part of the product).

    python -m oracle.refgpu [--dump 50] [--config 1]

oracle/_ref/refgpu_gd<GD> (oracle/refgpu/Makefile) is the reference's Run with its kernels built
for sm_100a at grid sizes of 1, 2 and 4 blocks of 64 x 8 threads per SM. Each is run on the
config-1 system (the product's arrays, written as a container by oracle/refbench.py, folded by
the oracle's OptimizeEnepara restatement so the product library is not loaded), with dump
windows of --dump steps; Run loops over windows until its records reach steps_per_dump x n_rep
and reports the time of its own kernel launches (McLog t0). Prints one JSON line: each grid
size's replica-steps/s by that time, and the best.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def binaries():
    return sorted(glob.glob(os.path.join(HERE, "_ref", "refgpu_gd*")),
                  key=lambda p: int(p.rsplit("gd", 1)[1]))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dump", type=int, default=50)
    ap.add_argument("--config", type=int, default=1)
    a = ap.parse_args(argv)
    from geaxdock_gpu_b200 import abi, system
    from oracle import pyoracle as po, refbench
    import numpy as np
    z = np.load(os.path.join(REPO, "tests", "golden", "ref_1a07C1.npz"))
    w = system.config(a.config, abi.enepara_raw_from_array(z["enepara_raw"]), seed=42,
                      fold=po.fold_enepara)
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.move_kind = abi.MOVE_UNIFORM  # the reference's Move_d draws U(-1, 1) x scale
    tmp = tempfile.mkdtemp(prefix="refgpu")
    path = os.path.join(tmp, "complex.gdfx")
    refbench.complex_container(path, cx, ff, params)
    runs = []
    for b in binaries():
        r = subprocess.run([b, "--bench", path, "--dump", str(a.dump)], capture_output=True,
                           text=True, timeout=900)
        if r.returncode != 0:
            raise RuntimeError("%s failed: %s" % (b, (r.stderr or r.stdout)[-500:]))
        runs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    best = max(runs, key=lambda x: x["replica_steps_per_s"]) if runs else None
    print(json.dumps({"reference_gpu": {
        "workload": "config%d: %d replicas (P=%d x %d conf, L=%d x %d conf, T=%d), the "
                    "reference's uniform moves at the configured scales" %
                    (a.config, cx.n_rep, cx.pnp, cx.n_prt, cx.lna, cx.n_lig, cx.n_tmp),
        "unit": "replica-steps/s (steps_total x n_rep / the reference's own launch time t0)",
        "runs": runs, "best": best}}), flush=True)


if __name__ == "__main__":
    main()
