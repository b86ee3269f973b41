"""Record streaming (gd_records_stream): the host buffer filled while the run proceeds equals,
after each flush, the records downloaded at that point (gd_get_records_raw), through plain
steps, the fused loop, a records reset, delayed-acceptance collect steps, and a stream started
before gd_mc_init."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a B200")]


def _same(e, buf, nxt):
    steps, n2 = e.records()
    assert np.array_equal(nxt, n2)
    for r in range(e.n_rep):
        assert buf[r, :nxt[r]].tobytes() == steps[r, :nxt[r]].tobytes(), r


@pytest.fixture(scope="module")
def cx_ff():
    z, cx, ff = load_ref("1a07C1")
    return cx, ff


def test_stream_matches_downloads(cx_ff):
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, seed=3)
    with engine.Engine(ff, [cx], params) as e:
        e.mc_init()
        buf = e.stream_records(201)
        for it in range(5):
            e.mc_run(0, it * 10)
            e.exchange(int(not (it % 2)))
        b, nxt = e.stream_flush()
        assert b is buf and nxt.max() > 1
        _same(e, buf, nxt)
        e.run_fused(50, 50, exchange=True)
        _same(e, *e.stream_flush())
        e.reset_records()
        for it in range(3):
            e.mc_run(200, it * 10)
        _same(e, *e.stream_flush())
        e.stream_stop()
        e.mc_run(200, 30)
        steps, n2 = e.records()
        assert n2.max() > 0


def test_stream_before_init_and_small_cap(cx_ff):
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, seed=4)
    with engine.Engine(ff, [cx], params) as e:
        buf = e.stream_records(25)
        e.mc_init()
        for it in range(4):
            e.mc_run(0, it * 10)
        b, nxt = e.stream_flush()
        steps, n2 = e.records()
        assert np.array_equal(nxt, n2)
        for r in range(e.n_rep):
            m = min(25, nxt[r])
            assert b[r, :m].tobytes() == steps[r, :m].tobytes()


def test_stream_delayed_acceptance_collect(cx_ff):
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=400, seed=5,
                           move_kind=abi.MOVE_GAUSSIAN)
    with engine.Engine(ff, [cx], params) as e:
        e.mc_init()
        sur = engine.Surrogate(e, hidden=128, batch=256, sample_cap=1 << 14)
        buf = e.stream_records(401)
        sur.collect(0, 40, exchange=True)
        sur.train(5)
        sur.run(40, 40, exchange=True)
        _same(e, *e.stream_flush())


def test_stream_started_mid_window(cx_ff):
    """A stream started after records exist copies those rows with its first snapshot, then
    the rows of every later call; a second stream on the same context restarts from row 0."""
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, seed=6)
    with engine.Engine(ff, [cx], params) as e:
        e.mc_init()
        for it in range(3):
            e.mc_run(0, it * 10)
        buf = e.stream_records(201)
        for it in range(3, 6):
            e.mc_run(0, it * 10)
        b, nxt = e.stream_flush()
        assert b is buf and nxt.max() > 30
        _same(e, buf, nxt)
        buf2 = e.stream_records(201)
        e.run_fused(60, 20, exchange=True)
        b2, nxt2 = e.stream_flush()
        assert b2 is buf2
        _same(e, buf2, nxt2)


def test_stream_partial_reset(cx_ff):
    """Resetting the records of some replicas restarts only their copies: the host array
    still equals the device records afterwards."""
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, seed=7)
    with engine.Engine(ff, [cx], params) as e:
        e.mc_init()
        buf = e.stream_records(201)
        for it in range(3):
            e.mc_run(0, it * 10)
        half = e.n_rep // 2
        e.reset_records(0, half - 1)
        for it in range(3, 5):
            e.mc_run(0, it * 10)
        b, nxt = e.stream_flush()
        assert b is buf and nxt[:half].max() <= 20 and nxt[half:].max() >= nxt[:half].max()
        _same(e, buf, nxt)


def test_async_window_download_is_the_download_at_that_point(cx_ff):
    """gd_get_records_async snapshots the window in stream order: the reset and the steps queued
    after it do not change what arrives, which equals a synchronous download taken at the same
    point of an identical run; the runs go on identically."""
    cx, ff = cx_ff
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=100, seed=5)
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        for e in (a, b):
            e.mc_init()
            for it in range(10):
                e.mc_run(0, it * 10)
                e.exchange(int(not (it % 2)))
        want, wnxt = a.records()
        out = np.empty(b.n_rep * b.cap, abi.RECORD_DTYPE)
        nxt = np.empty(b.n_rep, np.int32)
        b.records_async(out, nxt)
        for e in (a, b):
            e.reset_records()
            for it in range(3):
                e.mc_run(100, it * 10)
                e.exchange(int(not (it % 2)))
        got, gnxt = b.records_wait()
        assert np.array_equal(gnxt, wnxt) and wnxt.max() > 1
        assert got.shape == want.shape
        for r in range(b.n_rep):
            assert got[r, :wnxt[r]].tobytes() == want[r, :wnxt[r]].tobytes(), r
        assert a.state().tobytes() == b.state().tobytes()
        # the next window, asynchronously again into the same arrays
        b.records_async(out, nxt)
        w2, n2 = a.records()
        g2, m2 = b.records_wait()
        assert np.array_equal(m2, n2)
        for r in range(b.n_rep):
            assert g2[r, :n2[r]].tobytes() == w2[r, :n2[r]].tobytes(), r
