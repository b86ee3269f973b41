"""The reference's Run (src/run.h:8-19) as the drop-in geaxdock_gpu_b200/run_gpu/run_gpu.cpp.

run_gpu_check is the reference's own docking flow up to its Run call (its loaders and host
folds compiled from its sources, src/dock.C:97-191) linked with the drop-in Run and the
library. On the GPU, the records that Run returns for input files written in the reference's
formats must equal, bit for bit, the records of the library's Python mirror (Engine.run, the
same launcher loop) on the same files loaded by this package's loaders, for the same seed.
Without the built binary (it needs the reference tree to build) the tests skip.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, loaders
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref
from tests.inputs import write_complex, write_paras

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(os.path.dirname(HERE), "geaxdock_gpu_b200", "run_gpu", "_build")
CHECK = os.path.join(BUILD, "run_gpu_check")

needs_binary = pytest.mark.skipif(not os.access(CHECK, os.X_OK),
                                  reason="run_gpu_check not built (needs the reference tree)")


def _inputs(tmp_path, seed):
    write_complex(tmp_path, np.random.default_rng(seed))
    z, _, _ = load_ref("1a07C1")
    write_paras(tmp_path / "paras", abi.enepara_raw_from_array(z["enepara_raw"]))
    return ["--pdb", str(tmp_path / "p.pdb"), "--sdf", str(tmp_path / "l.sdf"),
            "--ff", str(tmp_path / "p.ff"), "--para", str(tmp_path / "paras"), "--id", "synth"]


def _read_records(path):
    raw = np.fromfile(path, dtype=np.uint8)
    n_rep = int(raw[:4].view(np.int32)[0])
    count = raw[4:4 + 4 * n_rep].view(np.int32)
    rows = raw[4 + 4 * n_rep:].view(abi.RECORD_DTYPE)
    assert rows.shape[0] == count.sum()
    return count, rows


@needs_binary
def test_run_drop_in_links_against_the_library():
    """Run is defined by run_gpu.o and the driver resolves the library it was linked with."""
    nm = subprocess.run(["nm", "-C", os.path.join(BUILD, "run_gpu.o")], capture_output=True,
                        text=True, check=True).stdout
    assert any(" T Run(" in ln for ln in nm.splitlines()), nm[-2000:]
    ldd = subprocess.run(["ldd", CHECK], capture_output=True, text=True, check=True).stdout
    line = [ln for ln in ldd.splitlines() if "libgeauxdock_b200" in ln]
    assert line and "not found" not in line[0], ldd


@needs_binary
@pytest.mark.skipif(have_gpu(), reason="checks the no-device error path")
def test_run_drop_in_reports_a_missing_device(tmp_path):
    r = subprocess.run([CHECK] + _inputs(tmp_path, 4) + ["--nt", "2", "--out",
                       str(tmp_path / "rec.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "gd_create failed" in r.stderr


@pytest.mark.gpu
@needs_binary
def test_run_drop_in_records_equal_the_engine(tmp_path):
    args = _inputs(tmp_path, 8)
    nt, floor_t, ceil_t, nc, ts, rs, seed = 3, 0.3, 0.9, 10, 0.2, 0.1, 77
    env = dict(os.environ, GD_SEED=str(seed), GD_DEVICE="0")
    r = subprocess.run([CHECK] + args + ["--nt", str(nt), "--floor_temp", str(floor_t),
                                         "--ceiling_temp", str(ceil_t), "--nc", str(nc),
                                         "-t", str(ts), "-r", str(rs),
                                         "--out", str(tmp_path / "rec.bin")],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    log = json.loads(r.stdout.strip().splitlines()[-1])
    count, rows = _read_records(str(tmp_path / "rec.bin"))

    cx, ff, _ = loaders.load_complex(str(tmp_path / "p.pdb"), str(tmp_path / "l.sdf"),
                                     str(tmp_path / "p.ff"), str(tmp_path / "paras"), "synth",
                                     nt, floor_t, ceil_t)
    assert log["n_rep"] == cx.n_rep == count.shape[0]
    params = abi.mc_params(steps_per_exchange=nc, steps_per_dump=abi.STEPS_PER_DUMP,
                           move_scale=(ts, ts, ts, rs, rs, rs), move_kind=abi.MOVE_UNIFORM,
                           record=1, seed=seed)
    with engine.Engine(ff, [cx], params) as eng:
        # the reference's IS_EXCHANGE toggle is off (src/toggle.h), so Run does not exchange
        want = eng.run(abi.STEPS_PER_DUMP * cx.n_rep, exchange=False)
        steps_total = eng.steps_total
    assert log["steps_total"] == steps_total
    got_count = np.array([len(want[i]) for i in range(cx.n_rep)])
    assert np.array_equal(count, got_count)
    want_rows = np.concatenate([np.array(want[i], dtype=abi.RECORD_DTYPE)
                                for i in range(cx.n_rep) if len(want[i])])
    assert rows.tobytes() == want_rows.tobytes()
    assert abs(log["ar"] - count.sum() / (cx.n_rep * steps_total)) < 1e-6
