"""Post-Monte-Carlo clustering on the GPU against the CPU oracle (oracle/kmeans.py), bit for
bit: memberships, representatives, cluster sizes and pass counts of the batched k-means, and
the whole post_mc (per-replica k = 50, pooled k = 500) on the records of a short run."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, postmc
from oracle import kmeans as ok
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a B200")]


def _energies(rng, n, dup=0):
    e = (rng.normal(0, 1, (n, 9)) * rng.uniform(0.1, 3.0, 9)).astype(np.float32)
    if dup and n > dup:
        e[-dup:] = e[:dup]  # exact duplicates: ties in every distance
    return e


def _check_segments(sizes, k, seed, rng):
    objs = [_energies(rng, n, dup=min(5, n // 4)) for n in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    ks = [k] * len(sizes)
    mem, med, size, passes, base = postmc.kmeans(np.concatenate(objs), off, ks, seed)
    for s, o in enumerate(objs):
        m_o, r_o, z_o, p_o = ok.cluster_by_kmeans(o, k, seed, s)
        cnt = min(k, sizes[s])
        assert np.array_equal(mem[off[s]:off[s + 1]], m_o), s
        got_r = med[base[s]:base[s] + cnt]
        assert np.array_equal(np.where(got_r >= 0, got_r - off[s], -1), r_o), s
        assert np.array_equal(size[base[s]:base[s] + cnt], z_o), s
        assert passes[s] == p_o, s


def test_kmeans_matches_oracle_ragged_segments():
    _check_segments([5, 50, 51, 300, 2001, 1, 777], 50, seed=11, rng=np.random.default_rng(1))


def test_kmeans_matches_oracle_large_k():
    """9,000 objects: above the size where members are listed by a radix sort"""
    _check_segments([9000], 500, seed=3, rng=np.random.default_rng(2))


def test_kmeans_batch_properties_at_scale():
    """2,000 segments of 2,001 objects (the per-replica stage at scale): every representative
    is a member of its cluster, sizes add up, a sample of segments equals the oracle."""
    rng = np.random.default_rng(3)
    n_seg, n = 2000, 2001
    obj = _energies(rng, n_seg * n)
    off = (np.arange(n_seg + 1) * n).astype(np.int32)
    mem, med, size, passes, base = postmc.kmeans(obj, off, [50] * n_seg, seed=5)
    assert np.all(size.reshape(n_seg, 50).sum(1) == n)
    ok_r = med >= 0
    cl = np.repeat(np.arange(n_seg), 50)
    assert np.all(mem[med[ok_r]] == (np.arange(n_seg * 50) - base[cl])[ok_r])
    for s in (0, 977, 1999):
        m_o, r_o, z_o, p_o = ok.cluster_by_kmeans(obj[off[s]:off[s + 1]], 50, 5, s)
        assert np.array_equal(mem[off[s]:off[s + 1]], m_o)
        assert passes[s] == p_o


def test_post_mc_matches_oracle_on_run_records():
    z, cx, ff = load_ref("1a07C1")
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, seed=9)
    with engine.Engine(ff, [cx], params) as e:
        e.mc_init()
        for it in range(20):
            e.mc_run(0, it * 10)
            e.exchange(int(not (it % 2)))
        steps, nxt = e.records()
    recs = [steps[i, :nxt[i]] for i in range(cx.n_rep)]
    got_r, got_z = postmc.post_mc(recs, seed=21)
    want_r, want_z = ok.post_mc(recs, seed=21)
    assert got_r.shape == want_r.shape and got_r.tobytes() == want_r.tobytes()
    assert np.array_equal(got_z, want_z)
    st_r, st_z = postmc.post_mc_steps(steps, nxt, seed=21)
    assert st_r.tobytes() == want_r.tobytes() and np.array_equal(st_z, want_z)


def test_post_mc_edge_cases():
    """Replicas without records, replicas with fewer records than clusters, and no records
    at all."""
    rng = np.random.default_rng(8)
    recs = []
    for n in (0, 3, 0, 120, 49, 50):
        r = np.zeros(n, abi.RECORD_DTYPE)
        r["energy"]["e"] = rng.normal(0, 1, (n, 10)).astype(np.float32)
        r["step"] = np.arange(n)
        recs.append(r)
    got_r, got_z = postmc.post_mc(recs, seed=4)
    want_r, want_z = ok.post_mc(recs, seed=4)
    assert got_r.tobytes() == want_r.tobytes() and np.array_equal(got_z, want_z)
    e_r, e_z = postmc.post_mc([np.zeros(0, abi.RECORD_DTYPE)] * 3, seed=4)
    assert e_r.shape == (0,) and e_z.shape == (0,)


def test_gpu_kmeans_is_the_references_seq_kmeans():
    """The library's k-means on the reference's own k-means run (src/seq_kmeans.c on the
    k-means module's 9-coordinate sample, 10 clusters, threshold 0.001; fixture from
    tests/golden/make_golden.py), the objects laid out so that the seeded shuffle restores the
    file's order: the reference's membership, cluster sizes and pass count."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "kmeans_ref.npz"))
    obj, ref = z["color100_objects"], z["color100_membership"]
    n = obj.shape[0]
    for seed in (0, 5):
        perm = postmc.permutation(seed, 0, n)
        objp = np.empty_like(obj)
        objp[perm] = obj
        mem, med, size, passes, base = postmc.kmeans(objp, [0, n], [10], seed)
        assert np.array_equal(mem[perm], ref)
        assert size.tolist() == np.bincount(ref, minlength=10).tolist()
        assert int(passes[0]) == int(z["color100_loops"][0])
