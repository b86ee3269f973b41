"""Context memory: gd_create's buffers come from a per-device pool that keeps freed memory for
the next context (gd_destroy does not unmap it), and gd_release_memory gives it back."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import engine, system
from tests.golden.fixtures import load_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def raw():
    from geaxdock_gpu_b200 import abi
    z, _, _ = load_ref("1a07C1")
    return abi.enepara_raw_from_array(z["enepara_raw"])


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_pool_keeps_memory_and_release_returns_it(raw):
    w = system.config(0, raw)
    cx, ff = w.complexes[0], w.ff
    engine.release_memory(0)
    base = _free_bytes()
    with engine.Engine(ff, [cx], w.params) as eng:
        eng.mc_init()
        eng.mc_run(0, 0)
        eng.sync()
        first = eng.etotal().copy()
        held = base - _free_bytes()
    assert held > 0
    # destroyed: the pool still holds the buffers
    assert base - _free_bytes() >= held // 2
    # a second context reuses them and computes the same chains
    with engine.Engine(ff, [cx], w.params) as eng:
        eng.mc_init()
        eng.mc_run(0, 0)
        eng.sync()
        assert np.array_equal(eng.etotal().view(np.uint32), first.view(np.uint32))
    engine.release_memory(0)
    assert base - _free_bytes() < held // 2
