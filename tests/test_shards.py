"""Replica shards on two ranks (gloo, CPU): the partition is agreed by every rank, covers each
complex exactly once with its batch index as RNG stream id, splits by whole exchange groups,
and the timing reduction is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from geaxdock_gpu_b200 import shard


def test_assign_complexes_balances_and_covers():
    costs = [50, 10, 40, 30, 20, 60, 5]
    parts = shard.assign_complexes(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert shard.assign_complexes(costs, 3) == parts  # deterministic


def test_protein_conformer_split_is_group_aligned():
    for n_prt in (1, 4, 11):
        for world in (1, 2, 3, 8):
            cuts = [shard.split_protein_conformers(n_prt, world, r) for r in range(world)]
            assert cuts[0][0] == 0 and cuts[-1][1] == n_prt
            for (a0, a1), (b0, b1) in zip(cuts, cuts[1:]):
                assert a1 == b0 and a0 <= a1
            sizes = [b - a for a, b in cuts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        parts = shard.assign_complexes(costs, world)
        mine = parts[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = shard.max_over_ranks(1.5 + rank, dist)
        q.put((rank, mine, gathered, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards_and_max_time():
    costs = [7, 3, 9, 1, 4, 4, 8]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    all_idx = sorted(i for _, mine, _, _ in out for i in mine)
    assert all_idx == list(range(len(costs)))
    for rank, mine, gathered, t in out:
        assert gathered == [o[1] for o in out]
        assert t == 1.5 + (world - 1)


def test_shard_batch_keeps_batch_index_as_stream():
    class Cx:
        def __init__(self, n_rep, lna, pnp):
            self.n_rep, self.lna, self.pnp = n_rep, lna, pnp
    batch = [Cx(512, 10 + i, 1200 + 100 * i) for i in range(6)]
    seen = []
    for rank in range(2):
        cxs, streams = shard.shard_batch(batch, 2, rank)
        assert [batch[s] for s in streams] == cxs
        seen += streams
    assert sorted(seen) == list(range(6))


def _mc_shard_worker(rank, world, port, q):
    """One rank: its shard of a small ragged batch through the oracle's FP32 Monte Carlo
    restatement (each complex with its batch index as RNG stream), states gathered on rank 0."""
    import datetime

    import numpy as np
    import torch.distributed as dist

    from geaxdock_gpu_b200 import abi, system
    from oracle import pyoracle as po
    from tests.golden.fixtures import load_ref
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        z, _, _ = load_ref("1a07C1")
        w = system.config(2, abi.enepara_raw_from_array(z["enepara_raw"]), n_ligands=5,
                          fold=po.fold_enepara)
        batch = [c.subset(n_lig=2, n_prt=1, n_tmp=4) for c in w.complexes]
        params = w.params
        params.record = 0
        mine, streams = shard.shard_batch(batch, world, rank)
        out = {}
        for cx, sid in zip(mine, streams):
            mc = po.MC(w.ff, cx, params, stream=sid, precision=32)
            mc.init()
            for e in range(2):
                mc.run(0, 10 * e, 10, 1)
                mc.exchange(int(not (e % 2)))
            g = mc.get()
            out[sid] = (g["mm_old"].tobytes(), g["e_old"].tobytes(), g["replica"].tobytes())
        gathered = [None] * world
        dist.all_gather_object(gathered, out)
        q.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_batch_and_reproduce_the_single_run():
    """A ragged batch split by shard_batch over two ranks: every complex runs on exactly one
    rank with its batch index as RNG stream, and the union of the ranks' final states equals
    the single-rank run of the whole batch bit for bit."""
    from geaxdock_gpu_b200 import abi, system
    from oracle import pyoracle as po
    from tests.golden.fixtures import load_ref
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mc_shard_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    union = {}
    for part in res[0][1]:
        assert not set(part) & set(union)
        union.update(part)
    assert res[0][1] == res[1][1]
    z, _, _ = load_ref("1a07C1")
    w = system.config(2, abi.enepara_raw_from_array(z["enepara_raw"]), n_ligands=5,
                      fold=po.fold_enepara)
    batch = [c.subset(n_lig=2, n_prt=1, n_tmp=4) for c in w.complexes]
    params = w.params
    params.record = 0
    assert sorted(union) == list(range(len(batch)))
    for sid, cx in enumerate(batch):
        mc = po.MC(w.ff, cx, params, stream=sid, precision=32)
        mc.init()
        for e in range(2):
            mc.run(0, 10 * e, 10, 1)
            mc.exchange(int(not (e % 2)))
        g = mc.get()
        assert union[sid] == (g["mm_old"].tobytes(), g["e_old"].tobytes(),
                              g["replica"].tobytes()), sid
