"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances: energies per term within 1e-5 relative to the FP64 oracle on the same FP32 placed
coordinates, with the conditioning-aware scale of tests/tolerance.py; contact counts (cms)
exact up to FP32 rounding of the MCC formula; accept / exchange decisions and replica
permutations bit-exact given the same Philox stream.
"""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, system
from oracle import pyoracle as po
from tests.golden.fixtures import load_ref
from tests.tolerance import plain_rel_errors, rel_errors, report, scales

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def raw():
    z, _, _ = load_ref("1a07C1")
    return abi.enepara_raw_from_array(z["enepara_raw"])


def _energy_check(eng, ff, cx, ci, ip, il, mm, refmap, plain=None):
    """Worst sum-of-magnitudes error per term of eng's energies of poses mm; the worst plain
    relative error per term is folded into `plain` when given."""
    got = eng.eval_energy(ci, ip, il, mm)
    worst = np.zeros(10)
    for i in range(mm.shape[0]):
        o = po.pose_energy(ff, cx, ip, il, mm[i], refmap, 64)
        worst = np.maximum(worst, rel_errors(got["e"][i], o, ff))
        if plain is not None:
            np.maximum(plain, plain_rel_errors(got["e"][i], o), out=plain)
        assert abs(got["cms"][i] - o["cms"]) <= 2e-6, (i, got["cms"][i], o["cms"])
        assert abs(got["rmsd"][i] - o["rmsd"]) <= 1e-5 * max(1.0, o["rmsd"])
    return worst


@pytest.mark.parametrize("name", ["1a07C1", "1robA1"])
def test_eval_energy_reference_complexes(name):
    z, cx, ff = load_ref(name)
    rm = z["ref_matrix"].astype(np.uint8)
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        sumabs, plain = np.zeros(10), np.zeros(10)
        for ip in range(min(cx.n_prt, 3)):
            sel = np.nonzero(z["pose_idx"][:, 0] == ip)[0]
            for il in np.unique(z["pose_idx"][sel, 1])[:4]:
                mm = z["pose_mm"][sel[z["pose_idx"][sel, 1] == il]]
                worst = _energy_check(eng, ff, cx, 0, ip, int(il), mm, rm, plain)
                sumabs = np.maximum(sumabs, worst)
                assert worst.max() <= TOL, (ip, il, worst)
    report("GPU gd_eval_energy, %s" % name, sumabs, plain)


@pytest.mark.parametrize("cfg", [0, 1])
def test_eval_energy_synthetic(raw, cfg):
    w = system.config(cfg, raw)
    cx, ff = w.complexes[0], w.ff
    rm = po.ref_map(ff, cx)
    rng = np.random.default_rng(5)
    mm = np.concatenate([rng.normal(0, 1.5, (24, 3)), rng.uniform(-3.2, 3.2, (24, 3))], 1)
    sumabs, plain = np.zeros(10), np.zeros(10)
    with engine.Engine(ff, [cx], w.params) as eng:
        for ip in range(min(cx.n_prt, 2)):
            worst = _energy_check(eng, ff, cx, 0, ip, 1, mm.astype(np.float32), rm, plain)
            sumabs = np.maximum(sumabs, worst)
            assert worst.max() <= TOL, worst
    report("GPU gd_eval_energy, config %d" % cfg, sumabs, plain)


@pytest.mark.parametrize("chunk", [64, 512, 4096])
def test_chunk_pipeline_gives_same_energies(raw, chunk):
    """Streaming (chunks < points) and resident protein tiles agree term by term."""
    w = system.config(1, raw)
    cx, ff = w.complexes[0], w.ff
    rm = po.ref_map(ff, cx)
    mm = np.random.default_rng(9).normal(0, 0.5, (16, 6)).astype(np.float32)
    with engine.Engine(ff, [cx], w.params) as eng:
        k = eng.tile()[0]
        eng.set_tile(k, chunk)
        worst = _energy_check(eng, ff, cx, 0, 3, 2, mm, rm)
        assert worst.max() <= TOL


def test_unroll_depths_give_identical_energies(raw):
    """One, two or four point pairs in flight per lane: the accumulators take the pairs in the
    same order, so the energies are bit-identical, and within the tolerance of the oracle."""
    w = system.config(1, raw)
    cx, ff = w.complexes[0], w.ff
    rm = po.ref_map(ff, cx)
    mm = np.random.default_rng(21).normal(0, 0.8, (12, 6)).astype(np.float32)
    got = {}
    with engine.Engine(ff, [cx], w.params) as eng:
        k = eng.tile()[0]
        for u in (1, 2, 4):
            eng.set_tile(k, 1024, u)
            assert eng.tile()[2] == u
            got[u] = eng.eval_energy(0, 5, 7, mm)
        worst = _energy_check(eng, ff, cx, 0, 5, 7, mm, rm)
    for u in (1, 4):
        assert got[u].tobytes() == got[2].tobytes(), u
    assert worst.max() <= TOL, worst


def test_far_pair_form_does_not_depend_on_warp_mates(raw):
    """Within each point segment the pair loop switches to the far form of the pair body at a
    slot set by the largest distance of the warp's atoms from the pocket centre. The far form
    gives the full form's result bit for bit, so a pose's energies do not depend on the poses
    that share its warps: one pose per CTA, six per CTA, the poses in another order, and a pose
    moved 15 A out of the pocket beside the others all give the same bytes."""
    w = system.config(1, raw)
    cx, ff = w.complexes[0], w.ff
    rng = np.random.default_rng(33)
    mm = rng.normal(0, 0.6, (12, 6)).astype(np.float32)
    mm[5, :3] = [15.0, -4.0, 6.0]
    perm = rng.permutation(12)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(12)
    runs = []
    with engine.Engine(ff, [cx], w.params) as eng:
        for k in (1, 6):
            eng.set_tile(k, 1024)
            runs.append(eng.eval_energy(0, 2, 4, mm))
            runs.append(eng.eval_energy(0, 2, 4, mm[perm])[inv])
        worst = _energy_check(eng, ff, cx, 0, 2, 4, mm, po.ref_map(ff, cx))
    for r in runs[1:]:
        assert r.tobytes() == runs[0].tobytes()
    assert worst.max() <= TOL, worst


def _init_and_compare(eng, ff, cx, w_params):
    eng.mc_init()
    eng.sync()
    st = eng.state()
    rm = po.ref_map(ff, cx)
    for r in range(0, cx.n_rep, max(1, cx.n_rep // 16)):
        p = r // (cx.n_tmp * cx.n_lig)
        l = r % cx.n_lig
        o = po.pose_energy(ff, cx, p, l, np.zeros(6, np.float32), rm, 64)
        assert rel_errors(st["energy_old"]["e"][r], o, ff).max() <= TOL
    steps, nxt = eng.records()
    assert np.all(nxt == 1)
    assert np.all(steps[:, 0]["step"] == 0)
    return st


def _replay(eng, cx, params, n_dumps_steps, trace_e, trace_acc, st0, exch_log):
    """Bit-exact replay of Metropolis decisions and exchanges from the device's own energies."""
    n_rep = cx.n_rep
    spe = params.steps_per_exchange
    e_old = st0["energy_old"]["e"][:, 9].copy()
    mm = st0["movematrix_old"].copy()
    idx_tmp = st0["replica"]["idx_tmp"].copy()
    mb_tab = cx.temp["minus_beta"]
    reps = np.arange(n_rep, dtype=np.uint32)
    for s in range(n_dumps_steps):
        delta, u = po.draw_steps(params.seed, params.move_kind, np.array(params.move_scale[:]),
                                 reps, np.full(n_rep, s, np.uint32))
        mmn = (mm + delta).astype(np.float32)
        acc = po.metropolis(trace_e[:, s], e_old, mb_tab[idx_tmp], u)
        assert np.array_equal(acc, trace_acc[:, s]), ("step", s, np.nonzero(acc != trace_acc[:, s]))
        m = acc.astype(bool)
        mm[m] = mmn[m]
        e_old[m] = trace_e[m, s]
        if (s + 1) % spe == 0:
            e = (s + 1) // spe - 1
            before, etot, after = exch_log[e]
            assert np.array_equal(before, idx_tmp)
            assert np.array_equal(etot, e_old)
            rep = np.zeros(n_rep, abi.REPLICA_DTYPE)
            rep["idx_tmp"] = idx_tmp
            po.exchange_apply(cx, params.seed, e, int(not (e % 2)), rep, e_old)
            assert np.array_equal(rep["idx_tmp"], after)
            idx_tmp = after
    return mm, e_old


@pytest.mark.parametrize("move_kind", [abi.MOVE_UNIFORM, abi.MOVE_GAUSSIAN])
def test_trajectory_replay_bit_exact(raw, move_kind):
    z, cx, ff = load_ref("1a07C1")
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=200, move_kind=move_kind,
                           move_scale=(0.2, 0.2, 0.2, 0.1, 0.1, 0.1), seed=1234)
    n_steps = 60
    with engine.Engine(ff, [cx], params) as eng:
        st0 = _init_and_compare(eng, ff, cx, params)
        eng.trace_enable(n_steps)
        log = []
        for e in range(n_steps // 10):
            eng.mc_run(0, e * 10)
            before = eng.replicas()["idx_tmp"].copy()
            et = eng.etotal()
            eng.exchange(int(not (e % 2)))
            log.append((before, et, eng.replicas()["idx_tmp"].copy()))
        eng.sync()
        te, ta = eng.trace()
        mm, e_old = _replay(eng, cx, params, n_steps, te, ta, st0, log)
        st = eng.state()
        assert np.array_equal(st["movematrix_old"].view(np.uint32), mm.view(np.uint32))
        assert np.array_equal(st["energy_old"]["e"][:, 9], e_old)
        assert np.array_equal(st["n_accept"], ta.sum(axis=1))
        # records: one per accepted step after the step-0 record, with their step numbers
        steps, nxt = eng.records()
        assert np.array_equal(nxt, 1 + ta.sum(axis=1))
        for r in range(0, cx.n_rep, 17):
            want = np.nonzero(ta[r])[0]
            assert np.array_equal(steps[r, 1:nxt[r]]["step"], want)
        # acceptance must be neither 0 nor 1 for the replay to mean something
        assert 0.05 < ta.mean() < 0.98


def test_fused_window_in_pieces_equals_one_call(raw):
    """The exchange inside the fused kernel takes mode_t from the interval's step within its
    dump window, so a window run as one call, in 10-step calls or in uneven pieces gives the
    same chains, and equals the stepwise loop across a window boundary (3 intervals per
    window: the alternation restarts at each window, as in the reference's launcher)."""
    w = system.config(0, raw)
    cx, ff = w.complexes[0], w.ff
    params = w.params
    params.steps_per_dump = 30
    engs = [engine.Engine(ff, [cx], params) for _ in range(4)]
    try:
        for e in engs:
            e.mc_init()
        a, b, c, d = engs
        for e in range(6):  # two dump windows of three intervals
            s1, s2 = (e // 3) * 30, (e % 3) * 10
            a.mc_run(s1, s2)
            a.exchange(int(not ((s2 // 10) % 2)))
        b.run_fused(0, 30, exchange=True)
        b.run_fused(30, 30, exchange=True)
        for s in range(0, 60, 10):
            c.run_fused(s, 10, exchange=True)
        d.run_fused(0, 20, exchange=True)
        d.run_fused(20, 30, exchange=True)
        d.run_fused(50, 10, exchange=True)
        want = a.state().tobytes()
        for e in (b, c, d):
            assert e.state().tobytes() == want
    finally:
        for e in engs:
            e.close()


def test_fused_graph_equals_stepwise(raw):
    w = system.config(0, raw)
    cx, ff = w.complexes[0], w.ff
    params = w.params
    params.steps_per_dump = 200
    with engine.Engine(ff, [cx], params) as a, engine.Engine(ff, [cx], params) as b:
        a.mc_init()
        b.mc_init()
        for e in range(6):
            a.mc_run(0, e * 10)
            a.exchange(int(not (e % 2)))
        b.run_fused(0, 60, exchange=True)
        a.sync()
        b.sync()
        sa, sb = a.state(), b.state()
        assert np.array_equal(sa.view(np.uint8), sb.view(np.uint8))
        ra, na = a.records()
        rb, nb = b.records()
        assert np.array_equal(na, nb)
        # a second replay of the cached graph continues the same chain
        for e in range(6, 12):
            a.mc_run(0, e * 10)
            a.exchange(int(not (e % 2)))
        b.run_fused(60, 60, exchange=True)
        a.sync()
        b.sync()
        assert np.array_equal(a.state().view(np.uint8), b.state().view(np.uint8))


@pytest.mark.parametrize("split,k", [(2, 3), (3, 2), (7, 1)])
def test_protein_split_energies(raw, split, k):
    """Lanes per atom > 1 (each walks part of every protein segment): every term still within
    1e-5 of the FP64 oracle, contact counts exact."""
    z, cx, ff = load_ref("1a07C1")
    refmap = po.ref_map(ff, cx)
    rng = np.random.default_rng(11 + split)
    with engine.Engine(ff, [cx], abi.mc_params(steps_per_dump=10)) as eng:
        eng.set_tile(k, 128, 0, split)
        assert eng.tile()[3] == split
        eng.mc_init()
        for ip, il in ((0, 0), (2, 5)):
            mm = np.zeros((7, 6), np.float32)
            mm[:, :3] = rng.normal(0, 1.0, (7, 3))
            mm[:, 3:] = rng.normal(0, 0.5, (7, 3))
            worst = _energy_check(eng, ff, cx, 0, ip, il, mm, refmap)
            assert worst.max() <= TOL, worst


@pytest.mark.parametrize("chains", [3, 5])
def test_concurrent_chains_give_the_same_chains(raw, chains):
    """The fused graph split into concurrent chains (streams) reproduces the single-chain run
    bit for bit, records included."""
    w = system.config(2, raw, n_ligands=6)
    params = w.params
    params.steps_per_dump = 40
    with engine.Engine(w.ff, w.complexes, params) as a, \
            engine.Engine(w.ff, w.complexes, params) as b:
        a.set_concurrency(1, 1)
        b.set_concurrency(chains, chains)
        for e in (a, b):
            e.set_tile(4, 256)
            e.mc_init()
            e.run_fused(0, 20, exchange=True)
            e.run_fused(20, 20, exchange=True)
            e.sync()
        assert a.state().tobytes() == b.state().tobytes()
        ra, na = a.records()
        rb, nb = b.records()
        assert np.array_equal(na, nb)
        assert ra.tobytes() == rb.tobytes()


def test_fill_tile_gives_each_complex_its_own_replica_count(raw):
    """threads > 0: every complex of a ragged batch gets as many replicas as fill the CTA; the
    chains equal those of a uniform tile (the replica count per CTA does not enter the
    arithmetic)."""
    w = system.config(2, raw, n_ligands=6)
    params = w.params
    params.steps_per_dump = 40
    with engine.Engine(w.ff, w.complexes, params) as a, \
            engine.Engine(w.ff, w.complexes, params) as b:
        a.set_tile(2, 256)
        b.set_tile(0, 256, 0, 1, 256)
        ks = [b.replicas_per_cta(i) for i in range(len(w.complexes))]
        for i, cx in enumerate(w.complexes):
            assert ks[i] == min(cx.n_tmp * cx.n_lig, 256 // cx.lna), (i, ks[i], cx.lna)
        assert b.tile() == (0, 256, 2, 1, 256, 1)
        for e in (a, b):
            e.mc_init()
            e.run_fused(0, 20, exchange=True)
            e.sync()
        assert a.state().tobytes() == b.state().tobytes()


def test_batch_equals_alone(raw):
    """Config-2 style batch (uneven ligands and pockets): each complex's trajectory in the
    batch is bit-identical to running it alone with the same stream id and tile."""
    w = system.config(2, raw, n_ligands=6)
    params = w.params
    params.steps_per_dump = 40
    with engine.Engine(w.ff, w.complexes, params) as eng:
        eng.set_tile(4, 256)
        eng.mc_init()
        eng.run_fused(0, 20, exchange=True)
        eng.sync()
        st = eng.state()
        for k in (0, 3, 5):
            cx = w.complexes[k]
            off = eng.offsets[k]
            with engine.Engine(w.ff, [cx], params) as one:
                one.set_rng_stream(0, k)
                one.set_tile(4, 256)
                one.mc_init()
                one.run_fused(0, 20, exchange=True)
                one.sync()
                s1 = one.state()
                mine = st[off:off + cx.n_rep]
                assert np.array_equal(s1["movematrix_old"], mine["movematrix_old"])
                for fld in ("e", "cms", "rmsd"):
                    assert np.array_equal(s1["energy_old"][fld], mine["energy_old"][fld]), fld
                assert np.array_equal(s1["replica"]["idx_tmp"], mine["replica"]["idx_tmp"])
                assert np.array_equal(s1["n_accept"], mine["n_accept"])


def test_cpu_baseline_statistics_match(raw):
    """Same Philox stream on the FP32 OpenMP CPU restatement: per-temperature energy samples
    are indistinguishable (two-sample KS p > 0.01) and most decisions coincide."""
    from scipy import stats
    w = system.config(0, raw)
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.record = 0
    n_ex = 20
    cpu = po.MC(ff, cx, params, stream=0, precision=32)
    cpu.init()
    with engine.Engine(ff, [cx], params) as eng:
        eng.mc_init()
        g_e, c_e, g_t, c_t = [], [], [], []
        for e in range(n_ex):
            eng.mc_run(0, e * 10)
            cpu.run(0, e * 10, 10)
            if e >= 5:
                gs, cs_ = eng.state(), cpu.get()
                g_e.append(gs["energy_old"]["e"][:, 9].copy())
                c_e.append(cs_["e_old"]["e"][:, 9].copy())
                g_t.append(gs["replica"]["idx_tmp"].copy())
                c_t.append(cs_["replica"]["idx_tmp"].copy())
            eng.exchange(int(not (e % 2)))
            cpu.exchange(int(not (e % 2)))
        eng.sync()
        ge, ce = np.array(g_e), np.array(c_e)
        gt, ct = np.array(g_t), np.array(c_t)
        for t in range(cx.n_tmp):
            a, b = ge[gt == t], ce[ct == t]
            assert stats.ks_2samp(a, b).pvalue > 0.01, t
        st, cs_ = eng.state(), cpu.get()
        same = np.mean(st["n_accept"] == cs_["n_accept"])
        assert same > 0.9, same


def test_record_overflow_is_reported(raw):
    z, cx, ff = load_ref("1a07C1")
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=3, move_scale=(0, 0, 0, 0, 0, 0))
    with engine.Engine(ff, [cx], params) as eng:
        eng.mc_init()
        eng.mc_run(0, 0)  # zero moves are always accepted: 10 records > capacity 4
        with pytest.raises(engine.GDError) as e:
            eng.sync()
        assert e.value.code == abi.GD_ERR_RECORD_FULL
        steps, nxt = eng.records()
        assert np.all(nxt == 4)


def test_bounded_wait_times_out_without_fault(raw):
    """A wait that runs out ends the kernel with GD_ERR_TIMEOUT; the context stays usable."""
    w = system.config(1, raw)
    cx, ff = w.complexes[0], w.ff
    params = w.params
    params.record = 0
    with engine.Engine(ff, [cx], params) as eng:
        k = eng.tile()[0]
        eng.set_tile(k, 64)  # streaming tiles: many waits
        eng.mc_init()
        eng.sync()
        eng.set_wait_timeout(0)
        eng.mc_run(0, 0)
        with pytest.raises(engine.GDError) as e:
            eng.sync()
        assert e.value.code == abi.GD_ERR_TIMEOUT
        eng.set_wait_timeout(2_000_000_000)
        eng.mc_init()
        eng.mc_run(0, 0)
        eng.sync()
        assert np.all(np.isfinite(eng.etotal()))


def test_autotune_picks_a_tile_and_keeps_the_chains(raw, tmp_path):
    from geaxdock_gpu_b200 import autotune
    w = system.config(0, raw)
    cx, ff = w.complexes[0], w.ff
    with engine.Engine(ff, [cx], w.params) as eng:
        eng.mc_init()
        eng.mc_run(0, 0)
        eng.sync()
        before = eng.state()
        res = autotune.tune(eng, cache_path=str(tmp_path / "cache.json"), repeats=1)
        assert not res["cached"]
        k, ch, u, sp, thr, pk = eng.tile()
        assert [k, ch, u, sp, pk] == res["tile"][:4] + res["tile"][5:] and sp == 1
        assert all(m > 0 or m == -1 for m in res["ms"].values())
        after = eng.state()
        assert np.array_equal(before.view(np.uint8), after.view(np.uint8))
        # the chains continue under the new tile exactly as a fresh run would
        eng.mc_run(0, 10)
        eng.sync()
        again = autotune.tune(eng, cache_path=str(tmp_path / "cache.json"))
        assert again["cached"] and again["tile"] == res["tile"]


def test_eval_energy_reproduces_reference_trajectory():
    """The library's energy kernel on every accepted step of the reference's own sample
    trajectory of 1a07C1 (data/trajectory.out, printed with %f by printLigandTrajectories,
    src/util.C:2041-2056): weighted total within 1e-5 and cms within 2e-6 of the printed
    values, the bounds the FP64 oracle meets on the same rows."""
    from tests.golden.fixtures import load_trajectory
    rows = load_trajectory()
    z, cx, ff = load_ref("1a07C1")
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        for ip, il in {(int(a), int(b)) for a, b in rows[:, :2]}:
            sel = (rows[:, 0] == ip) & (rows[:, 1] == il)
            got = eng.eval_energy(0, ip, il, rows[sel, 2:8].astype(np.float32))
            de = np.abs(got["e"][:, 9].astype(np.float64) - rows[sel, 9])
            dc = np.abs(got["cms"].astype(np.float64) - rows[sel, 8])
            assert de.max() <= 1e-5, (ip, il, int(de.argmax()), de.max())
            assert dc.max() <= 2e-6, (ip, il, int(dc.argmax()), dc.max())


def test_eval_energy_soft_core_poses():
    """Poses that put one ligand atom 0.4-1.9 A from a protein point, inside the soft core of
    the electrostatic term (r < 1 / el1), where the kernel adds the near-field terms after
    each segment's pair loop: every term within 1e-5 of the FP64 oracle."""
    z, cx, ff = load_ref("1a07C1")
    rm = z["ref_matrix"].astype(np.uint8)
    rng = np.random.default_rng(12)
    L, P = cx.lna, cx.pnp
    mm = np.zeros((24, 6), np.float32)
    for i in range(mm.shape[0]):
        l, p = int(rng.integers(L)), int(rng.integers(P))
        d = rng.normal(size=3)
        d *= rng.uniform(0.4, 1.9) / np.linalg.norm(d)
        orig = np.array([cx.lig_x[0, l], cx.lig_y[0, l], cx.lig_z[0, l]], np.float64)
        target = np.array([cx.prt_x[0, p], cx.prt_y[0, p], cx.prt_z[0, p]], np.float64) + d
        mm[i, :3] = target - orig - cx.lig_center[0]
    near = 1.0 / ff.el1
    for i in range(mm.shape[0]):
        xyz, _ = po.place_f64(cx, 0, mm[i])
        dmin = min(np.min((xyz[0][:, None] - cx.prt_x[0][None]) ** 2
                          + (xyz[1][:, None] - cx.prt_y[0][None]) ** 2
                          + (xyz[2][:, None] - cx.prt_z[0][None]) ** 2) ** 0.5, 9.0)
        assert dmin < near, (i, dmin)
    with engine.Engine(ff, [cx], abi.mc_params()) as eng:
        worst = _energy_check(eng, ff, cx, 0, 0, 0, mm, rm)
    assert worst.max() <= TOL, worst


def _extreme_batch(raw):
    """Config-2 complexes at the shape extremes: ligands of 10 and 64 atoms (8 conformers)
    against pockets of 1,200 and 6,000 points (4 conformers), 16 temperatures each."""
    rng = np.random.default_rng(2024)
    ff = system.forcefield(raw, 42)
    cxs = []
    for j, P in enumerate((1200, 6000)):
        center = np.array([100.0 * j, 0.0, 0.0])
        prot = system.make_protein(rng, ff, P, 4, center)
        for L in (10, 64):
            cxs.append(system.make_complex(rng, ff, L=L, n_lig=8, P=P, n_prt=4, n_tmp=16,
                                           protein=prot, pocket=center))
    return ff, cxs


@pytest.mark.parametrize("chunk", [512, 2048])
def test_config2_extreme_shapes_against_oracle(raw, chunk):
    """Energies of the batched kernel at config 2's extremes (L 10 / 64, P 1,200 / 6,000) in
    one context with the fill tile of 256 threads (25 replicas per CTA at L = 10, 4 at
    L = 64) and protein chunks smaller than every pocket (streamed): every term, cms and rmsd
    of given poses (gd_eval_energy) and of the initial poses (gd_mc_init) against the FP64
    oracle. Both error metrics are printed and the sum-of-magnitudes one is asserted: the
    synthetic totals here cancel by up to 130x (sum of |w_i e_i| over |e_9|), so a plain 1e-5
    on them would ask for 8e-8 of the summed magnitudes, below FP32 pair arithmetic."""
    ff, cxs = _extreme_batch(raw)
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=10, seed=7)
    rng = np.random.default_rng(chunk)
    sumabs, plain = np.zeros(10), np.zeros(10)
    with engine.Engine(ff, cxs, params) as eng:
        eng.set_tile(0, chunk, 0, 1, 256)
        ks = [eng.replicas_per_cta(i) for i in range(len(cxs))]
        assert ks == [25, 4, 25, 4], ks
        for ci, cx in enumerate(cxs):
            rm = po.ref_map(ff, cx)
            for ip, il in ((0, 0), (3, 5)):
                mm = np.zeros((10, 6), np.float32)
                mm[:, :3] = rng.normal(0, 1.5, (10, 3))
                mm[:, 3:] = rng.uniform(-3.1, 3.1, (10, 3))
                w = _energy_check(eng, ff, cx, ci, ip, il, mm, rm, plain)
                sumabs = np.maximum(sumabs, w)
        eng.mc_init()
        eng.sync()
        st = eng.state()
        for ci, cx in enumerate(cxs):
            rm = po.ref_map(ff, cx)
            off = eng.offsets[ci]
            for r in range(0, cx.n_rep, 37):
                p, l = r // (cx.n_tmp * cx.n_lig), r % cx.n_lig
                o = po.pose_energy(ff, cx, p, l, np.zeros(6, np.float32), rm, 64)
                got = st["energy_old"][off + r]
                sumabs = np.maximum(sumabs, rel_errors(got["e"], o, ff))
                np.maximum(plain, plain_rel_errors(got["e"], o), out=plain)
                assert abs(got["cms"] - o["cms"]) <= 2e-6
                assert abs(got["rmsd"] - o["rmsd"]) <= 1e-5 * max(1.0, o["rmsd"])
    report("config-2 extremes, chunk %d" % chunk, sumabs, plain)
    assert sumabs.max() <= TOL, sumabs


@pytest.mark.parametrize("cfg", [0, 2])
def test_two_replicas_per_lane_is_bit_identical(raw, cfg):
    """Two replicas per thread (the same atom of two slots sharing each point's loads) gives
    the chains, records and pose energies of one replica per lane bit for bit: config 0 with an
    odd replica count per CTA (the last thread's second slot empty), and a ragged config-2
    batch in fill mode."""
    if cfg == 0:
        w = system.config(0, raw)
        tiles = ((5, 512, 1, 1, 0, 1), (5, 512, 1, 1, 0, 2), (5, 512, 2, 1, 0, 2))
    else:
        w = system.config(2, raw, n_ligands=6)
        tiles = ((0, 256, 1, 1, 256, 1), (0, 256, 1, 1, 256, 2), (0, 256, 2, 1, 256, 2))
    params = w.params
    params.steps_per_dump = 40
    states, recs, energies = [], [], []
    mm = np.random.default_rng(3).normal(0, 1.0, (9, 6)).astype(np.float32)
    for t in tiles:
        with engine.Engine(w.ff, w.complexes, params) as e:
            e.set_tile(*t)
            assert e.tile()[5] == t[5]
            e.mc_init()
            e.run_fused(0, 20, exchange=True)
            e.mc_run(20, 0)
            e.exchange(1)
            e.sync()
            states.append(e.state().tobytes())
            r, n = e.records()
            recs.append((r.tobytes(), n.tobytes()))
            ci = len(w.complexes) - 1
            ip = min(1, w.complexes[ci].n_prt - 1)
            energies.append(e.eval_energy(ci, ip, 2, mm).tobytes())
    for i in (1, 2):
        assert states[i] == states[0], tiles[i]
        assert recs[i] == recs[0], tiles[i]
        assert energies[i] == energies[0], tiles[i]


def test_two_replicas_per_lane_rejects_what_it_cannot_take(raw):
    z, cx, ff = load_ref("1a07C1")
    with engine.Engine(ff, [cx], abi.mc_params()) as e:
        with pytest.raises(engine.GDError):
            e.set_tile(2, 256, 1, 2, 0, 2)  # split 2
        e.set_tile(6, 256, 1, 1, 0, 2)
        assert e.tile()[5] == 2 and e.replicas_per_cta(0) == 6


def test_largest_and_smallest_complexes_against_oracle(raw):
    """The capacities the C ABI accepts, batched in one context: a ligand of GD_MAXLIG = 100
    atoms against GD_MAXPRO = 10,000 protein points at GD_MAXTMP = 40 temperatures with 3,000
    KDE points and 20 MCS positions, next to a one-atom ligand against a one-point protein.
    Every term, cms and rmsd of given poses and of the initial poses against the FP64 oracle,
    with the default tile and with the 256-lane fill tile; ten Monte Carlo steps stay finite."""
    rng = np.random.default_rng(77)
    ff = system.forcefield(raw, 42)
    big = system.make_complex(rng, ff, L=abi.MAXLIG, n_lig=2, P=abi.MAXPRO, n_prt=1,
                              n_tmp=abi.MAXTMP, K=3000, M=20)
    small = system.make_complex(rng, ff, L=1, n_lig=2, P=1, n_prt=1, n_tmp=3, K=5, M=2,
                                pocket=np.array([200.0, 0.0, 0.0]))
    for m in range(small.pos):  # every MCS position restrains the single atom
        small.mcs_x[m, 1], small.mcs_y[m, 1], small.mcs_z[m, 1] = 200.5, 0.3, -0.2
    cxs = [big, small]
    params = abi.mc_params(steps_per_exchange=10, steps_per_dump=20, seed=3)
    sumabs = np.zeros(10)
    for tile in ((0, 512, 2, 1, 0, 1), (0, 512, 1, 1, 256, 1)):
        with engine.Engine(ff, cxs, params) as eng:
            if tile[4] == 0:
                eng.set_tile(2, 512, 2)
            else:
                eng.set_tile(*tile)
            for ci, cx in enumerate(cxs):
                rm = po.ref_map(ff, cx)
                mm = np.zeros((6, 6), np.float32)
                mm[:, :3] = rng.normal(0, 1.0, (6, 3))
                mm[:, 3:] = rng.uniform(-3.1, 3.1, (6, 3))
                for il in range(cx.n_lig):
                    sumabs = np.maximum(sumabs, _energy_check(eng, ff, cx, ci, 0, il, mm, rm))
            eng.mc_init()
            eng.sync()
            st = eng.state()
            for ci, cx in enumerate(cxs):
                rm = po.ref_map(ff, cx)
                for r in range(0, cx.n_rep, 7):
                    o = po.pose_energy(ff, cx, 0, r % cx.n_lig, np.zeros(6, np.float32), rm, 64)
                    got = st["energy_old"][eng.offsets[ci] + r]
                    sumabs = np.maximum(sumabs, rel_errors(got["e"], o, ff))
                    assert abs(got["cms"] - o["cms"]) <= 2e-6
            eng.run_fused(0, 10, exchange=True)
            eng.sync()
            assert np.all(np.isfinite(eng.etotal()))
    assert sumabs.max() <= TOL, sumabs


def test_energies_of_the_references_own_placed_coordinates():
    """gd_eval_energy_xyz on the coordinates the reference's own Move_d produced (the pin
    fixtures' pose_xyz / pose_center, src/kernel_cuda_l2_move.cu run on the CPU): every term
    within 1e-5 of the FP64 oracle on the same coordinates, and the total within 2e-5 of the
    reference's own FP32 CalcEnergy_d on them (whose own error is up to 7.3e-6 by the same
    metric); and placing poses with gd_place_ligand then evaluating the coordinates gives
    gd_eval_energy's results bit for bit."""
    for name in ("1a07C1", "1robA1"):
        z, cx, ff = load_ref(name)
        rm = z["ref_matrix"].astype(np.uint8)
        with engine.Engine(ff, [cx], abi.mc_params()) as eng:
            worst, vs_ref = np.zeros(10), 0.0
            for i in range(z["pose_mm"].shape[0]):
                ip, il = (int(v) for v in z["pose_idx"][i])
                xyz = np.ascontiguousarray(z["pose_xyz"][i].T)  # [lna, 3]
                got = eng.eval_energy_xyz(0, ip, il, xyz[None], z["pose_center"][i][None])[0]
                o = po.energy_eval(ff, cx, ip, il, z["pose_xyz"][i][0], z["pose_xyz"][i][1],
                                   z["pose_xyz"][i][2], z["pose_center"][i], rm, 64)
                worst = np.maximum(worst, rel_errors(got["e"], o, ff))
                assert abs(got["cms"] - o["cms"]) <= 2e-6
                vs_ref = max(vs_ref, abs(float(got["e"][9]) - float(z["pose_energy"][i][9]))
                             / scales(o, ff)[9])
            assert worst.max() <= TOL, (name, worst)
            assert vs_ref <= 2e-5, (name, vs_ref)
            ip, il = 1, 3
            mm = np.random.default_rng(4).normal(0, 1.0, (17, 6)).astype(np.float32)
            xyz = eng.place_ligand(0, il, mm)
            ctr = (mm[:, :3] + cx.lig_center[il][None, :].astype(np.float32)).astype(np.float32)
            a = eng.eval_energy(0, ip, il, mm)
            b = eng.eval_energy_xyz(0, ip, il, xyz, ctr)
            assert a.tobytes() == b.tobytes(), name
