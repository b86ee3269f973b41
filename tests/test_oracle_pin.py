"""The oracle against the reference's own code (fixtures from tests/golden/make_golden.py).

The fixtures hold, for the reference's real complexes 1a07C1 and 1robA1, the output of the
reference's CalcEnergy_d / CalcMcc_d / InitRefMatrix_d / Move_d / Accept_d /
ExchangeReplicas_d source compiled for the CPU and driven with the shared Philox stream.
"""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi
from oracle import pyoracle as po
from tests.golden.fixtures import load_ref
from tests.tolerance import plain_rel_errors, rel_errors, report

NAMES = ["1a07C1", "1robA1"]


@pytest.fixture(scope="module", params=NAMES)
def ref(request):
    return load_ref(request.param)


def test_sizes_of_1a07C1_match_reference_loader():
    z, cx, _ = load_ref("1a07C1")
    # reference src/load_test.C pins 21 conformers for 1a07C1; lna 34, pnp 344 from its loader
    assert (cx.n_lig, cx.lna, cx.n_prt, cx.pnp, cx.pnk, cx.pos) == (21, 34, 3, 344, 454, 11)


def test_contact_reference_matches_InitRefMatrix(ref):
    z, cx, ff = ref
    rm = po.ref_map(ff, cx)
    assert np.array_equal(rm, z["ref_matrix"].astype(np.uint8))


def test_fold_enepara_matches_OptimizeEnepara(ref):
    z, cx, ff = ref
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    folded = abi.struct_to_array(po.fold_enepara(raw))
    assert np.array_equal(folded.view(np.uint32), z["enepara"].view(np.uint32))


def test_set_temperature_matches_SetTemperature(ref):
    z, cx, ff = ref
    want = np.frombuffer(z["temp"].tobytes(), dtype=abi.TEMP_DTYPE)
    n = want.shape[0]
    floor_t = 0.5
    ceil_t = {4: 2.0, 2: 1.0}[n]
    got = po.set_temperature(n, floor_t, ceil_t)
    assert np.array_equal(got["minus_beta"].view(np.uint32), want["minus_beta"].view(np.uint32))
    assert np.array_equal(got["order"], want["order"])


def test_placement_matches_Move_d(ref):
    z, cx, ff = ref
    for i in range(z["pose_mm"].shape[0]):
        il = int(z["pose_idx"][i, 1])
        xyz, c = po.place_f32(cx, il, z["pose_mm"][i])
        # same Z-Y-X Euler transform; sin/cos implementations differ by an ulp or two
        assert np.max(np.abs(xyz - z["pose_xyz"][i])) <= 3e-5
        assert np.max(np.abs(c - z["pose_center"][i])) == 0.0


def test_energy_function_matches_CalcEnergy_d(ref):
    """FP64 oracle vs the reference's FP32 CalcEnergy_d on the reference's own coordinates."""
    z, cx, ff = ref
    rm = z["ref_matrix"].astype(np.uint8)
    worst = np.zeros(10)
    for i in range(z["pose_mm"].shape[0]):
        ip, il = (int(v) for v in z["pose_idx"][i])
        xyz = z["pose_xyz"][i]
        o = po.energy_eval(ff, cx, ip, il, xyz[0], xyz[1], xyz[2], z["pose_center"][i], rm, 64)
        worst = np.maximum(worst, rel_errors(z["pose_energy"][i][:10], o, ff))
        assert abs(o["cms"] - z["pose_energy"][i][10]) <= 1e-6
    # the reference computes in FP32: its own rounding is the bound here
    assert worst.max() <= 2e-5, worst


def test_reference_fp32_energies_scored_both_ways(ref):
    """The reference's own FP32 CalcEnergy_d against the FP64 oracle, by both metrics: every
    term within 1e-5 of the sum of magnitudes and the weighted total within 1e-5 plain, while
    the plain per-term error of the cancelled sums exceeds 1e-5 (ele on 1a07C1 reaches 3.4e-3,
    vdw on 1robA1 1.6e-4): the plain per-term form of "1e-5 relative to FP64" is not met by
    the reference's FP32 arithmetic itself."""
    z, cx, ff = ref
    rm = z["ref_matrix"].astype(np.uint8)
    sumabs, plain = np.zeros(10), np.zeros(10)
    for i in range(z["pose_mm"].shape[0]):
        ip, il = (int(v) for v in z["pose_idx"][i])
        xyz = z["pose_xyz"][i]
        o = po.energy_eval(ff, cx, ip, il, xyz[0], xyz[1], xyz[2], z["pose_center"][i], rm, 64)
        sumabs = np.maximum(sumabs, rel_errors(z["pose_energy"][i][:10], o, ff))
        plain = np.maximum(plain, plain_rel_errors(z["pose_energy"][i][:10], o))
    report("reference FP32 CalcEnergy_d, %d poses" % z["pose_mm"].shape[0], sumabs, plain)
    assert sumabs.max() <= 1e-5, sumabs
    assert plain[9] <= 1e-5, plain
    assert plain[:9].max() > 1e-5, plain


def test_init_energies_match_MonteCarlo_Init_d(ref):
    z, cx, ff = ref
    rm = z["ref_matrix"].astype(np.uint8)
    n_rep = cx.n_rep
    worst = 0.0
    for r in range(0, n_rep, max(1, n_rep // 40)):
        p = r // (cx.n_tmp * cx.n_lig)
        l = r % cx.n_lig
        o = po.pose_energy(ff, cx, p, l, np.zeros(6, np.float32), rm, 64)
        worst = max(worst, rel_errors(z["init_energy"][r][:10], o, ff).max())
        assert abs(o["cms"] - z["init_energy"][r][10]) <= 1e-6
    assert worst <= 1e-4, worst


def test_trajectory_proposals_and_decisions_match_MonteCarlo_d(ref):
    """Same Philox draws -> bit-identical proposals; Metropolis decisions identical on the
    reference's own energies; energies of the proposals within FP32 rounding."""
    z, cx, ff = ref
    rm = z["ref_matrix"].astype(np.uint8)
    n_rep, n_steps = z["traj_u"].shape
    scale = z["move_scale"]
    seed = int(z["run_params"][2])
    reps = np.repeat(np.arange(n_rep), n_steps).astype(np.uint32)
    steps = np.tile(np.arange(n_steps), n_rep).astype(np.uint32)
    delta, u = po.draw_steps(seed, abi.MOVE_UNIFORM, scale, reps, steps)
    mm_old = z["traj_mm_old"].reshape(-1, 6)
    prop = (mm_old + delta).astype(np.float32)
    assert np.array_equal(prop.view(np.uint32), z["traj_mm_new"].reshape(-1, 6).view(np.uint32))
    assert np.array_equal(u, z["traj_u"].reshape(-1))
    # decisions: replay Accept_d with the reference's energies and temperatures
    e_new = z["traj_energy"][:, :, 9].reshape(-1)
    acc_ref = z["traj_accept"].reshape(-1)
    nex = int(z["run_params"][1])
    nc = int(z["run_params"][0])
    temps = np.frombuffer(z["temp"].tobytes(), dtype=abi.TEMP_DTYPE)
    e_old = np.zeros_like(e_new)
    mb = np.zeros_like(e_new)
    for r in range(n_rep):
        cur = z["init_energy"][r][9]
        for s in range(n_steps):
            e = s // nc
            idx_tmp = z["xch_after"][e - 1][r] if e > 0 else (r // cx.n_lig) % cx.n_tmp
            k = r * n_steps + s
            e_old[k] = cur
            mb[k] = temps["minus_beta"][idx_tmp]
            if acc_ref[k]:
                cur = e_new[k]
    got = po.metropolis(e_new, e_old, mb, u)
    assert np.array_equal(got, acc_ref)
    # energies of a sample of proposals
    worst = 0.0
    for k in range(0, n_rep * n_steps, max(1, n_rep * n_steps // 60)):
        r = k // n_steps
        p = r // (cx.n_tmp * cx.n_lig)
        l = r % cx.n_lig
        o = po.pose_energy(ff, cx, p, l, prop[k], rm, 64)
        worst = max(worst, rel_errors(z["traj_energy"].reshape(-1, 12)[k][:10], o, ff).max())
    assert worst <= 1e-4, worst


def test_exchange_matches_ExchangeReplicas_d(ref):
    z, cx, ff = ref
    seed = int(z["run_params"][2])
    nc = int(z["run_params"][0])
    nex = z["xch_etotal"].shape[0]
    n_rep = cx.n_rep
    acs = np.zeros(n_rep, np.int32)
    for e in range(nex):
        rep = np.zeros(n_rep, abi.REPLICA_DTYPE)
        rep["idx_tmp"] = z["xch_before"][e]
        mode_t = int(not ((e * nc // nc) % 2))
        po.exchange_apply(cx, seed, e, mode_t, rep, z["xch_etotal"][e], acs)
        assert np.array_equal(rep["idx_tmp"], z["xch_after"][e])
        # the reference counts into acs_temp_exchg[slot position] (a per-slot index, not a
        # replica index); summing ours over (protein, ligand) groups gives its array
        nt, nl = cx.n_tmp, cx.n_lig
        folded = acs.reshape(cx.n_prt, nt, nl).sum(axis=(0, 2))
        assert np.array_equal(folded, z["xch_acs_ref"][e][:nt])
        assert not z["xch_acs_ref"][e][nt:].any()


# ---------------- RNG and math primitives ----------------

def test_philox4x32_10_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    assert po.philox(0, 0, 0, 0, 0, 0) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert po.philox(0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF) == \
        [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert po.philox(0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def _ulps(got, want):
    got = np.float32(got)
    return abs(float(got) - want) / float(np.spacing(np.float32(abs(want)) if want else np.float32(1e-45)))


def test_expf_accuracy():
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-87.0, 88.0, 4000), rng.uniform(-2, 2, 2000)])
    worst = max(_ulps(po.expf(float(x)), np.exp(np.float64(np.float32(x)))) for x in xs)
    assert worst <= 2.0, worst
    assert po.expf(-100.0) == 0.0 and po.expf(100.0) == float("inf")


def test_logf_accuracy():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(1e-7, 1.0, 4000), 2.0 ** -np.arange(0, 24)])
    for x in xs:
        want = np.log(np.float64(np.float32(x)))
        assert abs(po.logf(float(x)) - want) <= 4e-7 * max(1.0, abs(want))


def test_sincosf_accuracy():
    rng = np.random.default_rng(3)
    for x in np.concatenate([rng.uniform(-50, 50, 3000), rng.uniform(-1, 1, 1000)]):
        xf = np.float64(np.float32(x))
        s, c = po.sincosf(float(x))
        assert abs(s - np.sin(xf)) <= 2.5e-7 and abs(c - np.cos(xf)) <= 2.5e-7


def test_gaussian_moves_are_standard_normal():
    from scipy import stats
    n = 20000
    delta, u = po.draw_steps(7, abi.MOVE_GAUSSIAN, np.ones(6, np.float32), np.arange(n), np.zeros(n))
    for i in range(6):
        assert stats.kstest(delta[:, i], "norm").pvalue > 1e-3
    assert stats.kstest(u, "uniform").pvalue > 1e-3
    d2, _ = po.draw_steps(7, abi.MOVE_UNIFORM, np.ones(6, np.float32), np.arange(n), np.zeros(n))
    assert np.all(np.abs(d2) < 1.0) and abs(d2.mean()) < 0.02


def test_fp32_baseline_agrees_with_fp64(ref):
    z, cx, ff = ref
    rm = z["ref_matrix"].astype(np.uint8)
    for i in range(0, z["pose_mm"].shape[0], 8):
        ip, il = (int(v) for v in z["pose_idx"][i])
        o64 = po.pose_energy(ff, cx, ip, il, z["pose_mm"][i], rm, 64)
        o32 = po.pose_energy(ff, cx, ip, il, z["pose_mm"][i], rm, 32)
        assert rel_errors(o32["e"], o64, ff).max() <= 2e-5


# The reference's sample trajectory prints each value with %f (6 decimals, +-5e-7) after an
# FP32 evaluation on the GPU: the weighted total is held to 1e-5, the contact fraction to 2e-6.
TRAJ_E_TOL = 1e-5
TRAJ_CMS_TOL = 2e-6


def test_oracle_reproduces_reference_trajectory():
    """Every accepted step of data/trajectory.out (1a07C1, written by printLigandTrajectories,
    src/util.C:2041-2056) re-evaluated from its protein/ligand index and move vector with the
    reference's own parameter file and .ff: the weighted total and cms come back to the
    printed precision, which pins the loaders, the parameter fold and CalcEnergy_d together
    on data the reference produced itself."""
    from tests.golden.fixtures import load_trajectory
    rows = load_trajectory()
    z, cx, ff = load_ref("1a07C1")
    rm = po.ref_map(ff, cx)
    assert rows.shape == (2666, 10)
    de = np.zeros(rows.shape[0])
    dc = np.zeros(rows.shape[0])
    for i, r in enumerate(rows):
        o = po.pose_energy(ff, cx, int(r[0]), int(r[1]), r[2:8].astype(np.float32), rm, 64)
        de[i] = abs(o["e"][9] - r[9])
        dc[i] = abs(o["cms"] - r[8])
    assert de.max() <= TRAJ_E_TOL, (int(de.argmax()), de.max())
    assert dc.max() <= TRAJ_CMS_TOL, (int(dc.argmax()), dc.max())


def test_oracle_placement_is_the_reference_trace():
    """The reference's trace program (read2D, PlaceLigand, replaceLigandCoords; src/trace.C:90-122,
    run by tests/golden/make_trajectory.py through oracle/_ref/refpin on every 13th row of
    data/trajectory.out): the oracle places every atom of those rows within the SDF lines'
    printed precision (5e-5 rounding, 1.1e-4 allowed) in FP64 and in FP32."""
    from tests.golden.fixtures import load_trajectory_trace
    rows, pick, ref = load_trajectory_trace()
    z, cx, ff = load_ref("1a07C1")
    assert ref.shape == (pick.shape[0], cx.lna, 3)
    for k, i in enumerate(pick):
        lc, mm = int(rows[i, 1]), rows[i, 2:8].astype(np.float32)
        for place in (po.place_f64, po.place_f32):
            xyz, _ = place(cx, lc, mm)
            assert np.max(np.abs(np.asarray(xyz, np.float64).T - ref[k])) <= 1.1e-4, (k, place)
