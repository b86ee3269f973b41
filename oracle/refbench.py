"""CPU timing of the reference's own Monte Carlo step code (test / benchmark infrastructure).

`oracle/_ref/refpin --bench` (built by oracle/refpin/Makefile from the reference's sources,
which it compiles for the CPU) runs the reference's MonteCarlo_d step functions (Move_d,
CalcEnergy_d, CalcMcc_d, Accept_d, RecordLigand_d; src/kernel_cuda_l1_montecarlo.cu:95-117) on
one thread for a replica range of a complex handed over as the product's arrays in the
harness's named-array container. The reference's device code keeps its state in globals, so
the host cores are used by one process per core, each on its own replica range.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
import time
from typing import Dict, Optional

import numpy as np

from geaxdock_gpu_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REFPIN = os.path.join(HERE, "_ref", "refpin")


def available() -> bool:
    return os.path.exists(REFPIN) and os.access(REFPIN, os.X_OK)


def write_gdfx(path: str, arrays: Dict[str, np.ndarray]):
    with open(path, "wb") as f:
        f.write(b"GDFX1\n")
        for name, a in arrays.items():
            a = np.ascontiguousarray(a)
            if a.dtype.kind == "f":
                a, code = a.astype(np.float32), b"f"
            else:
                a, code = a.astype(np.int32), b"i"
            nb = name.encode()
            f.write(struct.pack("<I", len(nb)) + nb + code + struct.pack("<I", a.ndim))
            for d in a.shape:
                f.write(struct.pack("<Q", d))
            f.write(a.tobytes())


def complex_container(path: str, cx: abi.ComplexArrays, ff: abi.EnePara, params: abi.McParams):
    """The complex, the folded force field, the temperatures, the move scales and kind."""
    sizes = np.array([cx.n_lig, cx.n_prt, cx.n_tmp, cx.lna, cx.pnp, cx.pnk, cx.pos, 0], np.int32)
    arrays = {"sizes": sizes}
    for name in ("lig_x", "lig_y", "lig_z", "lig_center", "lig_t", "lig_c", "lig_n", "prt_x",
                 "prt_y", "prt_z", "prt_t", "prt_c", "prt_ele", "prt_seq3r", "prt_hflag",
                 "prt_hpp", "pocket_center", "psp", "kde_x", "kde_y", "kde_z", "kde_t", "mcs_x",
                 "mcs_y", "mcs_z", "mcs_tcc"):
        arrays[name] = getattr(cx, name)
    arrays["temp"] = np.frombuffer(np.ascontiguousarray(cx.temp).tobytes(), np.float32)
    arrays["enepara"] = np.frombuffer(bytes(ff), np.float32)
    arrays["move_scale"] = np.array([params.move_scale[i] for i in range(6)], np.float32)
    arrays["move_kind"] = np.array([params.move_kind], np.int32)
    write_gdfx(path, arrays)


def run(cx: abi.ComplexArrays, ff: abi.EnePara, params: abi.McParams, n_rep: int, steps: int,
        procs: int = 0, seed: int = 42, workdir: Optional[str] = None) -> Dict:
    """Runs replicas [0, n_rep) for `steps` steps on `procs` processes in parallel; returns
    replica-steps, the wall time of the slowest process and the accepted moves."""
    procs = procs or os.cpu_count() or 1
    procs = max(1, min(procs, n_rep))
    tmp = workdir or tempfile.mkdtemp(prefix="refbench")
    path = os.path.join(tmp, "complex.gdfx")
    complex_container(path, cx, ff, params)
    cuts = [n_rep * i // procs for i in range(procs + 1)]
    t0 = time.perf_counter()
    ps = [subprocess.Popen([REFPIN, "--bench", path, "--r0", str(cuts[i]), "--r1", str(cuts[i + 1]),
                            "--steps", str(steps), "--seed", str(seed)],
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
          for i in range(procs)]
    outs = [p.communicate() for p in ps]
    wall = time.perf_counter() - t0
    total, acc, inner = 0, 0, 0.0
    for p, (o, e) in zip(ps, outs):
        if p.returncode != 0:
            raise RuntimeError("refpin --bench failed: %s" % e.strip()[-300:])
        n, sec, a = o.split()
        total += int(n)
        acc += int(a)
        inner = max(inner, float(sec))
    return {"replica_steps": total, "seconds": inner, "wall": wall, "accepted": acc,
            "processes": procs}
