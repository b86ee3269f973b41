"""The allocation-free pose-energy entry point, gd_eval_energy_noalloc.

Callers that cannot allocate device memory when they need energies (a framework that owns the
whole device pool, a callback or real-time context where cudaMalloc is not allowed) pass
device buffers they already own; the entry point's own scratch lives in a fixed device array
of the library. These checks call it through the C ABI several times in a row, against the
regular gd_eval_energy on the same poses (the same kernel on the same poses, so the results
must agree bit for bit), at the size limit and past it, and check that a call leaves the
device's free memory unchanged. The file is named to be collected last, so that a run stopping
at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine
from tests.golden.fixtures import load_ref

pytestmark = pytest.mark.gpu

MAX_POSES = 16384  # GD_NOALLOC_MAX_POSES in include/geauxdock_b200.h


def _noalloc_fn():
    fn = engine.lib().gd_eval_energy_noalloc
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _poses(rng, n):
    return np.concatenate([rng.normal(0, 1.0, (n, 3)), rng.uniform(-3.1, 3.1, (n, 3))],
                          axis=1).astype(np.float32)


def test_noalloc_matches_eval_energy_on_two_calls():
    import torch

    fn = _noalloc_fn()
    z, cx, ff = load_ref("1a07C1")
    rng = np.random.default_rng(11)
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        for call, (ip, il, n) in enumerate([(0, 3, 37), (2, 11, 300), (1, 5, MAX_POSES)]):
            mm = _poses(rng, n)
            want = eng.eval_energy(0, ip, il, mm)
            # device buffers owned by the caller (allocated here, not by the entry point)
            d_mm = torch.from_numpy(mm).to("cuda")
            d_out = torch.full((n * 12,), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            rc = fn(eng.h, 0, ip, il, d_mm.data_ptr(), n, d_out.data_ptr())
            assert rc == abi.GD_OK, engine.lib().gd_last_error_string()
            eng.sync()
            got = d_out.cpu().numpy().view(abi.ENERGY_DTYPE)
            assert got.tobytes() == want.tobytes(), "call %d (%d poses)" % (call, n)


def test_noalloc_call_leaves_free_device_memory_unchanged():
    import torch

    fn = _noalloc_fn()
    z, cx, ff = load_ref("1a07C1")
    n = 1000
    mm = _poses(np.random.default_rng(3), n)
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        d_mm = torch.from_numpy(mm).to("cuda")
        d_out = torch.zeros(n * 12, dtype=torch.float32, device="cuda")
        first = torch.zeros_like(d_out)
        assert fn(eng.h, 0, 0, 0, d_mm.data_ptr(), n, first.data_ptr()) == abi.GD_OK
        eng.sync()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        assert fn(eng.h, 0, 0, 0, d_mm.data_ptr(), n, d_out.data_ptr()) == abi.GD_OK
        eng.sync()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
        assert torch.equal(first, d_out)


def test_noalloc_rejects_too_many_poses():
    import torch

    fn = _noalloc_fn()
    z, cx, ff = load_ref("1a07C1")
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        d = torch.zeros(16, dtype=torch.float32, device="cuda")
        rc = fn(eng.h, 0, 0, 0, d.data_ptr(), MAX_POSES + 1, d.data_ptr())
        assert rc == abi.GD_ERR_CAPACITY
        assert b"allocation-free" in engine.lib().gd_last_error_string()
        assert fn(eng.h, 0, 0, 0, d.data_ptr(), -1, d.data_ptr()) == abi.GD_ERR_INVALID
        assert fn(eng.h, 0, 0, 0, d.data_ptr(), 0, d.data_ptr()) == abi.GD_OK
