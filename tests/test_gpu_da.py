"""Delayed acceptance on the GPU: exactness against the plain Monte Carlo path.

* collect mode (every proposal passes, samples stored) is the plain trajectory, bit for bit;
* with the surrogate stage switched off, the delayed-acceptance step is the plain step, bit
  for bit (S_new = S_cur, same proposal and final uniform);
* with the stage on, every decision is replayed on the CPU from the Philox draws, the traced
  surrogate energies and the exact energies (checked against the FP64 oracle): stage 1 is
  u1 < exp(mb (S_new - S_cur)), stage 2 is u2 < exp(mb ((E_new - E_old) - (S_new - S_cur)));
* per-temperature energy distributions of delayed acceptance and plain Monte Carlo from the
  same equilibrated start are indistinguishable (two-sample KS per temperature, the family of
  20 tests at level 0.01);
* the fallback controller switches a complex whose stage-2 acceptance is below the threshold
  back to plain Monte Carlo.
"""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, system
from oracle import pyoracle as po
from tests.conftest import have_gpu
from tests.golden.fixtures import load_ref
from tests.tolerance import scales

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a B200")]


@pytest.fixture(scope="module")
def raw():
    z, _, _ = load_ref("1a07C1")
    return abi.enepara_raw_from_array(z["enepara_raw"])


def _small(raw, **kw):
    w = system.config(0, raw)
    p = w.params
    p.steps_per_dump = 400
    for k, v in kw.items():
        if k == "move_scale":
            for i in range(6):
                p.move_scale[i] = v[i]
        else:
            setattr(p, k, v)
    return w


def _same_records(a, b):
    ra, na = a.records()
    rb, nb = b.records()
    assert np.array_equal(na, nb)
    for r in range(na.size):
        assert ra[r, :na[r]].tobytes() == rb[r, :nb[r]].tobytes(), r


def test_collect_is_the_plain_trajectory(raw):
    w = _small(raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        a.mc_init()
        b.mc_init()
        a.run_fused(0, 60, exchange=True)
        sur = engine.Surrogate(b, hidden=128, batch=256, sample_cap=1 << 16)
        sur.collect(0, 60, exchange=True)
        a.sync()
        b.sync()
        assert a.state().tobytes() == b.state().tobytes()
        _same_records(a, b)
        assert sur.info()["n_samples"] == 60 * cx.n_rep
        st = sur.stats()[0]
        assert st["plain"] == 60 * cx.n_rep and st["proposed"] == 0
        assert st["plain_accepted"] == int(b.state()["n_accept"].sum())


def test_concurrent_chains_collect_is_plain(raw):
    """Collect steps on a ragged batch split into 3 concurrent chains equal the plain fused
    loop on one chain."""
    w = system.config(2, raw, n_ligands=6)
    params = w.params
    params.steps_per_dump = 40
    with engine.Engine(w.ff, w.complexes, params) as a, \
            engine.Engine(w.ff, w.complexes, params) as b:
        a.set_concurrency(1, 1)
        b.set_concurrency(1, 3)
        for e in (a, b):
            e.set_tile(4, 256)
            e.mc_init()
        a.run_fused(0, 20, exchange=True)
        sur = engine.Surrogate(b, hidden=128, batch=256, sample_cap=1 << 16)
        sur.collect(0, 20, exchange=True)
        a.sync()
        b.sync()
        assert a.state().tobytes() == b.state().tobytes()
        _same_records(a, b)


@pytest.mark.parametrize("unroll", [0, 4])
def test_stage_off_is_the_plain_step(raw, unroll):
    """unroll 4: a tile with four point pairs in flight (the unsplit exact stage runs two)."""
    w = _small(raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        if unroll:
            for e in (a, b):
                t = e.tile()
                e.set_tile(t[0], t[1], unroll)
        a.mc_init()
        b.mc_init()
        a.run_fused(0, 60, exchange=True)
        sur = engine.Surrogate(b, hidden=128, batch=256, sample_cap=1 << 16, fallback_accept=0.0)
        sur.collect(0, 60, exchange=True)
        sur.train(20)
        assert sur.stats()[0]["active"] == 1
        sur.set_active(0, False)
        a.run_fused(60, 60, exchange=True)
        sur.run(60, 60, exchange=True)
        a.sync()
        b.sync()
        assert a.state().tobytes() == b.state().tobytes()
        _same_records(a, b)


def _stage1_uniform(seed, stream, replica, step):
    w = po.philox(int(replica), int(step), int(stream), 1, seed & 0xFFFFFFFF, seed >> 32)[3]
    return np.float32((w >> 8) * 2.0 ** -24)


@pytest.mark.parametrize("split,unroll", [(0, 0), (3, 0), (3, 4)])
def test_decisions_replay(raw, split, unroll):
    """split 3: the exact stage walks each protein segment with 3 lanes per atom; unroll 4:
    with four point pairs in flight (the exact stage keeps the tile's unroll when split)."""
    scale = (0.6, 0.6, 0.6, 0.3, 0.3, 0.3)  # larger moves: both stages reject
    w = _small(raw, move_scale=scale)
    cx, ff, params = w.complexes[0], w.ff, w.params
    s0, n = 100, 30
    with engine.Engine(ff, [cx], params) as eng:
        if unroll:
            t = eng.tile()
            eng.set_tile(t[0], t[1], unroll)
        eng.mc_init()
        sur = engine.Surrogate(eng, hidden=128, batch=512, sample_cap=1 << 16,
                               fallback_accept=0.0, split=split)
        sur.collect(0, s0, exchange=True)
        losses = sur.train(150)
        assert losses[-1] < losses[0]
        st0 = eng.state()
        sur.trace_enable(s0, n)
        sur.run(s0, n, exchange=False)
        eng.sync()
        s_tr, e_tr, f_tr = sur.trace()
        st1 = eng.state()
    assert set(np.unique(f_tr)) <= {0, 1, 2}
    assert (f_tr == 0).any() and (f_tr == 1).any() and (f_tr == 2).any()
    refmap = po.ref_map(ff, cx)
    mm = st0["movematrix_old"].copy()
    e_old = st0["energy_old"]["e"][:, 9].copy()
    s_cur = np.full(cx.n_rep, np.nan, np.float32)  # known once a replica accepted a move
    idx_tmp = st0["replica"]["idx_tmp"]
    mbs = np.asarray(cx.temp["minus_beta"], np.float32)
    checked_e = 0
    worst = np.zeros(10)
    for k in range(n):
        step = s0 + k
        reps = np.arange(cx.n_rep, dtype=np.uint32)
        delta, u2 = po.draw_steps(params.seed, params.move_kind, list(params.move_scale), reps,
                                  np.full(cx.n_rep, step, np.uint32))
        for r in range(cx.n_rep):
            mb = mbs[idx_tmp[r]]
            mmn = (mm[r] + delta[r]).astype(np.float32)
            f = f_tr[r, k]
            sn = s_tr[r, k]
            if not np.isnan(s_cur[r]):
                u1 = _stage1_uniform(params.seed, 0, r, step)
                d1 = np.float32(np.float32(sn - s_cur[r]) * mb)
                assert (f > 0) == bool(u1 < po.expf(d1)), (r, k)
            if f == 0:
                assert np.isnan(e_tr[r, k])
                continue
            en = np.float32(e_tr[r, k])
            if r % 9 == 0:
                p, l = r // (cx.n_tmp * cx.n_lig), r % cx.n_lig
                o = po.pose_energy(ff, cx, int(p), int(l), mmn, refmap, 64)
                worst[9] = max(worst[9], abs(float(en) - o["e"][9]) / scales(o, ff)[9])
                checked_e += 1
            sc = s_cur[r] if not np.isnan(s_cur[r]) else sn
            d2 = np.float32(np.float32(np.float32(en - e_old[r]) - np.float32(sn - sc)) * mb)
            acc = bool(u2[r] < po.expf(d2))
            if not np.isnan(s_cur[r]):
                assert acc == (f == 2), (r, k)
            if f == 2:
                mm[r] = mmn
                e_old[r] = en
                s_cur[r] = sn
    assert checked_e > 20
    assert worst[9] < 1e-5, worst[9]
    assert np.array_equal(st1["movematrix_old"].view(np.uint32), mm.view(np.uint32))
    assert np.array_equal(st1["energy_old"]["e"][:, 9], e_old)
    assert np.array_equal(st1["n_accept"] - st0["n_accept"], (f_tr == 2).sum(axis=1))


def test_energy_distributions_match_plain(raw):
    """Config-1 system, configured moves: 2,000 plain burn-in steps (the surrogate's training
    samples), then plain and delayed-acceptance runs of 1,000 steps each from the same state.
    The 341 (protein, ligand conformer) chains at one temperature are independent, so the
    final snapshot gives independent samples per temperature."""
    from scipy import stats
    w = system.config(1, raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.record = 0
    burn, span = 2000, 1000
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        b.mc_init()
        sur = engine.Surrogate(b, sample_cap=16 << 20, fallback_accept=0.0)
        sur.collect(0, burn, exchange=True)
        losses = sur.train(1000)
        assert losses[-50:].mean() < 0.05 * losses[:10].mean()
        b.sync()
        a.mc_init()
        a.set_state(b.state())
        a.run_fused(burn, span, exchange=True)
        sur.run(burn, span, exchange=True)
        sa, sb = a.state(), b.state()
        st = sur.stats()[0]
    assert st["proposed"] == span * cx.n_rep and st["active"] == 1
    assert st["rmse"] < 0.5
    ea, eb = sa["energy_old"]["e"][:, 9], sb["energy_old"]["e"][:, 9]
    ta, tb = sa["replica"]["idx_tmp"], sb["replica"]["idx_tmp"]
    ps = [stats.ks_2samp(ea[ta == t], eb[tb == t]).pvalue for t in range(cx.n_tmp)]
    # 20 KS tests at p > 0.01 each fail somewhere ~18 % of the time for identical processes;
    # the family is held at level 0.01 (Bonferroni) and at most two temperatures may sit
    # below 0.01 (their expected number under equality is 0.2)
    assert min(ps) > 0.01 / cx.n_tmp, ps
    assert sum(p <= 0.01 for p in ps) <= 2, ps


def test_fallback_to_plain(raw):
    w = _small(raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    with engine.Engine(ff, [cx], params) as eng:
        eng.mc_init()
        sur = engine.Surrogate(eng, hidden=128, batch=64, sample_cap=1 << 14,
                               fallback_accept=0.999, fallback_window=500)
        sur.collect(0, 20, exchange=True)
        sur.train(1)  # barely trained: stage-2 acceptance below 0.999
        sur.run(20, 20, exchange=True)
        st = sur.stats()[0]
        assert st["active"] == 0
        assert st["proposed"] == 20 * cx.n_rep
        sur.run(40, 20, exchange=True)
        st2 = sur.stats()[0]
        assert st2["proposed"] == st["proposed"]
        assert st2["plain"] == st["plain"] + 20 * cx.n_rep
        assert st["rmse"] > 0 and st["n_err"] == st["passed"]


def test_trained_surrogate_gains_over_plain_and_untrained(raw):
    """What the trained network gains, on the config-0 system at 20x the configured moves
    (2 A / 1 rad): from one equilibrated state, plain Monte Carlo, delayed acceptance with an
    untrained network (its random initial weights, normalised like a trained one) and delayed
    acceptance with the network trained on the burn-in's exact energies each run 300 steps.
    The cost of an accepted move is the number of exact energy evaluations spent per accepted
    move: every proposal for plain Monte Carlo, the stage-1 survivors for delayed acceptance.
    The trained network must spend fewer than both others, by at least a third, and pass its
    survivors through stage 2 at least 90 % of the time."""
    w = _small(raw, move_scale=(2.0, 2.0, 2.0, 1.0, 1.0, 1.0))
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.record = 0
    burn, span = 2000, 300
    R = cx.n_rep
    with engine.Engine(ff, [cx], params) as plain, \
            engine.Engine(ff, [cx], params) as good, \
            engine.Engine(ff, [cx], params) as blind:
        good.mc_init()
        sg = engine.Surrogate(good, hidden=256, batch=2048, sample_cap=1 << 20,
                              fallback_accept=0.0)
        sg.collect(0, burn, exchange=True)
        losses = sg.train(1500)
        assert losses[-50:].mean() < 0.1 * losses[:10].mean()
        start = good.state()
        blind.mc_init()
        sb = engine.Surrogate(blind, hidden=256, batch=2048, sample_cap=1 << 16,
                              fallback_accept=0.0)
        sb.collect(0, 20, exchange=True)   # samples only set the output normalisation
        sb.train(0)                        # stage on with the untrained network
        blind.set_state(start)
        plain.mc_init()
        plain.set_state(start)
        for e in (plain, good, blind):
            e.sync()
        st0 = {k: s.stats()[0] for k, s in (("good", sg), ("blind", sb))}
        plain.run_fused(burn, span, exchange=True)
        sg.run(burn, span, exchange=True)
        sb.run(burn, span, exchange=True)
        plain_acc = int((plain.state()["n_accept"] - start["n_accept"]).sum())
        st1 = {k: s.stats()[0] for k, s in (("good", sg), ("blind", sb))}
    d = {k: {f: st1[k][f] - st0[k][f] for f in ("proposed", "passed", "accepted")}
         for k in st1}
    assert d["good"]["proposed"] == d["blind"]["proposed"] == span * R
    cost_plain = span * R / max(1, plain_acc)
    cost_good = d["good"]["passed"] / max(1, d["good"]["accepted"])
    cost_blind = d["blind"]["passed"] / max(1, d["blind"]["accepted"])
    stage2_good = d["good"]["accepted"] / max(1, d["good"]["passed"])
    print("exact evaluations per accepted move: plain %.3f, untrained %.3f, trained %.3f; "
          "trained stage-2 acceptance %.3f, acceptance plain %.3f / trained %.3f"
          % (cost_plain, cost_blind, cost_good, stage2_good, plain_acc / (span * R),
             d["good"]["accepted"] / (span * R)))
    assert stage2_good >= 0.9
    assert cost_good < (2.0 / 3.0) * cost_plain
    assert cost_good < (2.0 / 3.0) * cost_blind


def test_decisions_replay_ragged_batch(raw):
    """Delayed acceptance with the stage on over a ragged config-2 batch (6 ligands of uneven
    size on uneven pockets, one network for the batch): every stage-1 and stage-2 decision of
    every replica is replayed on the CPU from the Philox draws of its complex's stream, the
    traced surrogate energies and the exact energies; a sample of the exact energies is
    checked against the FP64 oracle."""
    w = system.config(2, raw, n_ligands=6)
    params = w.params
    params.steps_per_dump = 400
    for i in range(6):
        params.move_scale[i] *= 8.0
    s0, n = 60, 12
    with engine.Engine(w.ff, w.complexes, params) as eng:
        eng.set_tile(4, 256)
        eng.mc_init()
        sur = engine.Surrogate(eng, hidden=128, batch=1024, sample_cap=1 << 20,
                               fallback_accept=0.0)
        sur.collect(0, s0, exchange=True)
        losses = sur.train(200)
        assert losses[-1] < losses[0]
        st0 = eng.state()
        sur.trace_enable(s0, n)
        sur.run(s0, n, exchange=False)
        eng.sync()
        s_tr, e_tr, f_tr = sur.trace()
        st1 = eng.state()
        offs = list(eng.offsets)
    assert (f_tr == 0).any() and (f_tr == 1).any() and (f_tr == 2).any()
    mm_all = st0["movematrix_old"].copy()
    eo_all = st0["energy_old"]["e"][:, 9].copy()
    checked, worst = 0, 0.0
    for ci, cx in enumerate(w.complexes):
        sl = slice(offs[ci], offs[ci] + cx.n_rep)
        mm, e_old = mm_all[sl], eo_all[sl]
        ft, st_, et = f_tr[sl], s_tr[sl], e_tr[sl]
        s_cur = np.full(cx.n_rep, np.nan, np.float32)
        idx_tmp = st0["replica"]["idx_tmp"][sl]
        mbs = np.asarray(cx.temp["minus_beta"], np.float32)
        refmap = po.ref_map(w.ff, cx)
        reps = np.arange(cx.n_rep, dtype=np.uint32)
        for k in range(n):
            step = s0 + k
            delta, u2 = po.draw_steps(params.seed, params.move_kind, list(params.move_scale),
                                      reps, np.full(cx.n_rep, step, np.uint32), stream=ci)
            for r in range(cx.n_rep):
                mb = mbs[idx_tmp[r]]
                mmn = (mm[r] + delta[r]).astype(np.float32)
                f, sn = ft[r, k], st_[r, k]
                if not np.isnan(s_cur[r]):
                    u1 = _stage1_uniform(params.seed, ci, r, step)
                    d1 = np.float32(np.float32(sn - s_cur[r]) * mb)
                    assert (f > 0) == bool(u1 < po.expf(d1)), (ci, r, k)
                if f == 0:
                    continue
                en = np.float32(et[r, k])
                if r % 101 == 0:
                    p, l = r // (cx.n_tmp * cx.n_lig), r % cx.n_lig
                    o = po.pose_energy(w.ff, cx, int(p), int(l), mmn, refmap, 64)
                    worst = max(worst, abs(float(en) - o["e"][9]) / scales(o, w.ff)[9])
                    checked += 1
                sc = s_cur[r] if not np.isnan(s_cur[r]) else sn
                d2 = np.float32(np.float32(np.float32(en - e_old[r]) - np.float32(sn - sc)) * mb)
                if not np.isnan(s_cur[r]):
                    assert bool(u2[r] < po.expf(d2)) == (f == 2), (ci, r, k)
                if f == 2:
                    mm[r] = mmn
                    e_old[r] = en
                    s_cur[r] = sn
        mm_all[sl], eo_all[sl] = mm, e_old
    assert checked > 20 and worst < 1e-5, (checked, worst)
    assert np.array_equal(st1["movematrix_old"].view(np.uint32), mm_all.view(np.uint32))
    assert np.array_equal(st1["energy_old"]["e"][:, 9], eo_all)


def test_training_steps_replayed_from_a_graph_are_deterministic(raw):
    """gd_sur_train runs its first Adam step eagerly and replays the rest from a CUDA graph
    whose per-step values (batch-draw iteration, loss slot, Adam step count) live on the
    device. Without the embedding (whose gradient is an atomic scatter) training is
    deterministic: two engines trained on the same samples give the same loss history, every
    slot written, and a second call continues the draws and Adam's step count."""
    w = _small(raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    hist = []
    for _ in range(2):
        with engine.Engine(ff, [cx], params) as e:
            e.mc_init()
            sur = engine.Surrogate(e, hidden=128, batch=512, sample_cap=1 << 16, embedding=0,
                                   fallback_accept=0.0)
            sur.collect(0, 40, exchange=True)
            l1 = sur.train(25)
            l2 = sur.train(25)
            hist.append(np.concatenate([l1, l2]))
            x = np.zeros((4, 6), np.float32)
            x[:, 0] = np.arange(4) * 0.3
            hist.append(sur.predict(0, 0, 1, x))
    assert np.array_equal(hist[0], hist[2])
    assert np.array_equal(hist[1], hist[3])
    losses = hist[0]
    assert np.all(np.isfinite(losses)) and np.all(losses > 0)
    assert losses[40:].mean() < losses[:5].mean()
    assert len(set(losses.tolist())) > 40  # every step wrote its own slot


def test_collect_is_the_plain_trajectory_with_two_replicas_per_thread(raw):
    """A context whose plain tile holds two replicas per thread (the autotuner may pick it)
    still runs the delayed-acceptance pipeline, whose kernels hold one replica per lane: its
    collect steps are the plain trajectory bit for bit."""
    w = _small(raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        for e in (a, b):
            e.set_tile(6, 512, 1, 1, 0, 2)
            e.mc_init()
        a.run_fused(0, 40, exchange=True)
        sur = engine.Surrogate(b, hidden=128, batch=256, sample_cap=1 << 16)
        sur.collect(0, 40, exchange=True)
        a.sync()
        b.sync()
        assert a.state().tobytes() == b.state().tobytes()
        _same_records(a, b)
