"""Throughput of the replica-exchange Monte Carlo docking path (MC replica-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: config 1 (P = 3,000 protein points x 11 conformers, L = 40 ligand atoms x 31
conformers, 20 temperatures: 6,820 replicas; Gaussian moves; exchange every 10 steps), seeded
synthetic data. One bench step = one exchange interval: 10 MC steps of every replica + one
temperature exchange, one launch of gd_mc_run_fused (the exchange runs inside the Monte Carlo
kernel). K timed steps after W warm-up steps.

ours:      device time from CUDA events recorded on the library's own stream around each
           step, L2 flushed between steps (outside the events), max over ranks; `e2e` is a
           whole run through the C ABI from host buffers (gd_create uploads, init, K steps,
           record download per dump window) timed on the host, on every rank (the slowest
           rank's time); `cpu_baseline` is the reference's own step code
           on the host cores (as the reference arm) on a bounded sample (rank 0, N = 1).
reference: the reference's own MonteCarlo_d step functions (Move_d, CalcEnergy_d, CalcMcc_d,
           Accept_d, RecordLigand_d) compiled for the CPU from its sources (oracle/_ref/refpin),
           one process per host core, a bounded replica sample per step, same metric; the
           oracle's FP32 OpenMP restatement when that build is absent.
Multi-GPU (torchrun): the job is one batch of N config-1 complexes (complex i drawn with seed
42 + i, RNG stream i), split across ranks by shard.shard_batch's assignment (one complex per GPU);
exchange never crosses complexes, so there is no data-path collective: weak scaling.
delayed_acceptance (N = 1): the config-3 workload on the config-1 system (2,000 burn-in steps of
           training samples, one epoch of Adam, then K intervals of delayed-acceptance and of
           plain steps from the same state, device-timed), at the configured moves and at 20x
           and 60x larger moves; surrogate RMSE, stage acceptances, per-temperature KS p-values.
batched_screen (N = 1): config 2 (2,048 uneven ligands x 8 uneven pockets, 1,048,576 replicas)
           in one context, one persistent launch per 10-step interval, autotuned tile.
delayed_acceptance.sampling_efficiency (N = 1): effective samples per second (integrated
           autocorrelation time of every chain's energy) of plain Monte Carlo and of delayed
           acceptance, each at its best move scale of x1 / x5 / x20 / x40 / x60 / x100.
screen_delayed_acceptance (N = 1): config 4, delayed acceptance on that screen with one network
           per pocket, against the plain batched run from the same state, at the configured and
           at 20x larger moves; best-pose energy and RMSD agreement per ligand.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC replica-steps/s (plain batched REMC; delayed acceptance under delayed_acceptance)"
UNIT = "replica-steps/s"


def load_raw():
    from geaxdock_gpu_b200 import abi
    z = np.load(os.path.join(ROOT, "tests", "golden", "ref_1a07C1.npz"))
    return abi.enepara_raw_from_array(z["enepara_raw"])


def workload(seed, fold=None):
    from geaxdock_gpu_b200 import system
    return system.config(1, load_raw(), seed=seed, fold=fold)


def bench_config(world):
    """The workload object both arms print (the same system, moves and step at every N)."""
    return {"workload": "config1: P=3000 x 11 conf, L=40 x 31 conf, T=20, 6820 replicas per "
                        "GPU, gaussian moves 0.1 A / 0.05 rad, exchange/10",
            "step": "10 MC steps of every replica + 1 exchange",
            "l2": "flushed between steps (256 MB write)",
            "parallelism": ("one batch of N config-1 complexes split by shard_batch, one "
                            "complex per GPU, no collective") if world > 1 else "1 GPU"}


def product_library_mapped():
    """True when this process has the product's CUDA library mapped (Linux /proc maps)."""
    try:
        with open("/proc/self/maps") as f:
            return any("libgeauxdock_b200" in ln for ln in f)
    except OSError:
        return False


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
                power.append(float(p[3]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_median": statistics.median(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def algorithmic_flops_per_replica_step(eng, w, n_sample=24):
    """FLOPs per replica-step by the counting convention: 36 per ligand-protein pair, plus
    hpc 12 / hdb 8 / psp 1 per conditional hit, KDE 11 per matched pair, MCS 9 per valid atom,
    with the hit counts measured by the oracle on a sample of the current poses."""
    from oracle import pyoracle as po
    cx, ff = w.complexes[0], w.ff
    st = eng.state()
    rm = po.ref_map(ff, cx)
    rng = np.random.default_rng(0)
    tot = 0.0
    picks = rng.choice(cx.n_rep, n_sample, replace=False)
    for r in picks:
        p = r // (cx.n_tmp * cx.n_lig)
        l = r % cx.n_lig
        o = po.pose_energy(ff, cx, int(p), int(l), st["movematrix_old"][r], rm, 64)
        tot += (36.0 * cx.lna * cx.pnp + 12.0 * o["hits_hpc"] + 8.0 * o["hits_hdb"] +
                1.0 * o["hits_psp"] + 11.0 * o["hits_kde"] + 9.0 * o["hits_mcs"])
    return tot / n_sample


def cpu_baseline_sample(w, seconds=12.0, nthreads=0):
    """The reference's own MonteCarlo_d step code compiled for the CPU (oracle/_ref/refpin, one
    process per host core) on a bounded replica sample of the same workload; the oracle's FP32
    OpenMP restatement when that build is absent."""
    from oracle import pyoracle as po, refbench
    cx, ff = w.complexes[0], w.ff
    params = type(w.params).from_buffer_copy(w.params)
    params.record = 0
    nt = nthreads or po.max_threads()
    if refbench.available():
        probe = refbench.run(cx, ff, params, n_rep=nt, steps=1, procs=nt)
        rate = probe["replica_steps"] / max(probe["seconds"], 1e-3)
        n_rep = int(min(cx.n_rep, max(nt, nt * round(seconds * rate / 10 / nt))))
        r = refbench.run(cx, ff, params, n_rep=n_rep, steps=10, procs=nt)
        return {"value": r["replica_steps"] / r["seconds"], "unit": UNIT, "cores": r["processes"],
                "kind": "reference",
                "sample": "%d replicas x 10 MC steps of the config-1 system through the reference's "
                          "MonteCarlo_d step functions (oracle/_ref/refpin), one process per core, "
                          "slowest process %.1f s" % (n_rep, r["seconds"])}
    mc = po.MC(ff, cx, params, stream=0, precision=32)
    mc.init()
    t0 = time.perf_counter()
    mc.run_range(0, nt, 0, 0, 1, nt)  # probe: one step on nt replicas
    rate = nt / max(time.perf_counter() - t0, 1e-3)  # replica-steps/s
    n_rep = int(min(cx.n_rep, max(nt, nt * round(seconds * rate / 10 / nt))))
    t0 = time.perf_counter()
    mc.run_range(0, n_rep, 0, 1, 10, nt)
    dt = time.perf_counter() - t0
    return {"value": n_rep * 10 / dt, "unit": UNIT, "cores": nt, "kind": "port",
            "sample": "%d replicas x 10 MC steps of the config-1 system (%.1f s)" % (n_rep, dt)}


def run_reference(args, rank, world):
    """The reference arm: the reference's own MonteCarlo_d step code on the host cores
    (oracle/_ref/refpin, one process per core; the oracle's FP32 OpenMP port when that build is
    absent), each bench step a bounded replica sample x 10 MC steps of the config-1 system with
    the configured Gaussian moves. The force field is folded by the oracle's OptimizeEnepara
    restatement (bit-identical to the reference's and the library's folds), so this process
    never loads the product's library; it checks that before printing."""
    if rank != 0:
        return
    from oracle import pyoracle as po, refbench
    w = workload(42, fold=po.fold_enepara)
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.record = 0
    nt = po.max_threads()
    use_ref = refbench.available()
    if use_ref:
        probe = refbench.run(cx, ff, params, n_rep=nt, steps=1, procs=nt)
        rate = probe["replica_steps"] / max(probe["seconds"], 1e-3)
        n_rep = int(min(cx.n_rep, max(nt, nt * int(0.8 * rate / 10 / nt))))

        def one_step(s2):
            r = refbench.run(cx, ff, params, n_rep=n_rep, steps=10, procs=nt, seed=42 + s2)
            return r["seconds"], r["replica_steps"]
    else:
        mc = po.MC(ff, cx, params, stream=0, precision=32)
        mc.init()
        t0 = time.perf_counter()
        mc.run_range(0, nt, 0, 0, 1, nt)
        per_batch = max(time.perf_counter() - t0, 1e-3)  # one step of nt replicas
        n_rep = int(min(cx.n_rep, max(nt, nt * int(0.8 / (10 * per_batch)))))

        def one_step(s2):
            t0 = time.perf_counter()
            mc.run_range(0, n_rep, 0, s2, 10, nt)
            return time.perf_counter() - t0, n_rep * 10
    s2 = 0
    for _ in range(args.warmup):
        one_step(s2)
        s2 += 10
    times, done = [], 0
    for _ in range(args.steps):
        dt, n = one_step(s2)
        times.append(dt)
        done += n
        s2 += 10
    tot = sum(times)
    value = done / tot
    kind = "reference" if use_ref else "port"
    sample = ("%d of 6820 replicas x 10 MC steps (configured Gaussian moves) per bench step "
              "through the reference's MonteCarlo_d step functions compiled for the CPU "
              "(oracle/_ref/refpin), one process per core; the exchange (< 0.2 %% of a step) "
              "not timed" % n_rep
              if use_ref else "%d of 6820 replicas x 10 MC steps per bench step (oracle FP32 "
              "OpenMP port)" % n_rep)
    if product_library_mapped():
        raise RuntimeError("the reference arm loaded the product's library")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded, config-1 shapes)", "impl": "reference",
           "config": bench_config(world),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": kind,
                            "sample": sample, "replicas_sampled": n_rep},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def delayed_acceptance(w, dev, tile, scale_mult, intervals, burn=2000, iters=1665):
    """Config-3 workload: the config-1 system, 2,000 plain burn-in steps whose proposals train
    the surrogate (13.64 M samples), one epoch of Adam (batch 8,192, lr 1e-3), then `intervals`
    exchange intervals of delayed-acceptance steps and, from the same state, of plain steps,
    alternately, each bracketed by CUDA events on its engine's stream (L2 flushed between).
    Per-temperature KS test on the final states of the two runs."""
    import ctypes as C
    import torch
    from scipy import stats
    from geaxdock_gpu_b200 import engine
    cx, ff = w.complexes[0], w.ff
    p = type(w.params).from_buffer_copy(w.params)
    p.record = 0
    for i in range(6):
        p.move_scale[i] = w.params.move_scale[i] * scale_mult
    spe = p.steps_per_exchange
    with engine.Engine(ff, [cx], p, device=dev) as b, engine.Engine(ff, [cx], p, device=dev) as a:
        b.set_tile(*tile)
        a.set_tile(*tile)
        b.mc_init()
        sur = engine.Surrogate(b)
        t0 = time.perf_counter()
        sur.collect(0, burn, exchange=True)
        b.sync()
        collect_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        losses = sur.train(iters)
        train_s = time.perf_counter() - t0
        info = sur.info()
        a.mc_init()
        start = b.state()
        a.set_state(start)
        a.sync()
        sa = torch.cuda.ExternalStream(a.cuda_stream(), device=dev)
        sb = torch.cuda.ExternalStream(b.cuda_stream(), device=dev)
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:%d" % dev)
        s = burn
        a.run_fused(s, spe, exchange=True)  # graph capture + warm-up
        sur.run(s, spe, exchange=True)
        a.sync()
        b.sync()
        s += spe
        ev = []
        for _ in range(intervals):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(sa)
            a.run_fused(s, spe, exchange=True)
            e[1].record(sa)
            with torch.cuda.stream(sa):
                flush.add_(1.0)
            a.sync()
            e[2].record(sb)
            sur.run(s, spe, exchange=True)
            e[3].record(sb)
            with torch.cuda.stream(sb):
                flush.add_(1.0)
            b.sync()
            ev.append(e)
            s += spe
        torch.cuda.synchronize(dev)
        plain_ms = sum(x[0].elapsed_time(x[1]) for x in ev)
        da_ms = sum(x[2].elapsed_time(x[3]) for x in ev)
        st = sur.stats()[0]
        split_used = sur.split()
        fa, fb = a.state(), b.state()
        del flush
    # null reference for the KS test: plain steps from the same start with another seed, the
    # same warm-up interval plus `intervals` intervals as the two arms
    p2 = type(p).from_buffer_copy(p)
    p2.seed = p.seed + 1
    with engine.Engine(ff, [cx], p2, device=dev) as c2:
        c2.set_tile(*tile)
        c2.mc_init()
        c2.set_state(start)
        c2.run_fused(burn, spe * (intervals + 1), exchange=True)
        c2.sync()
        fc = c2.state()
    ea, eb = fa["energy_old"]["e"][:, 9], fb["energy_old"]["e"][:, 9]
    ta, tb = fa["replica"]["idx_tmp"], fb["replica"]["idx_tmp"]
    ks = [float(stats.ks_2samp(ea[ta == t], eb[tb == t]).pvalue) for t in range(cx.n_tmp)]
    ec, tc = fc["energy_old"]["e"][:, 9], fc["replica"]["idx_tmp"]
    ks_null = [float(stats.ks_2samp(ea[ta == t], ec[tc == t]).pvalue) for t in range(cx.n_tmp)]
    rs = cx.n_rep * spe * intervals
    passed = max(1, st["passed"])
    return {"metric": "MC replica-steps/s (surrogate delayed acceptance)",
            "value": rs / (da_ms * 1e-3), "unit": UNIT,
            "plain_same_state": rs / (plain_ms * 1e-3),
            "speedup_vs_plain": plain_ms / da_ms,
            "move_scale": [p.move_scale[i] for i in range(6)],
            "stage1_pass": st["passed"] / max(1, st["proposed"]),
            "stage2_accept": st["accepted"] / passed,
            "accept": st["accepted"] / max(1, st["proposed"]),
            "surrogate_rmse": st["rmse"], "target_mu_sigma": [info["mu"], info["sigma"]],
            "surrogate_active": st["active"],
            "ks_min_p": min(ks), "ks_p_per_temperature": ks,
            "ks_null_min_p": min(ks_null), "ks_null_p_per_temperature": ks_null,
            "ks_note": "final states, 341 independent chains per temperature; ks_null: plain vs "
                       "plain with another seed from the same start (what equal distributions "
                       "give for the smallest of 20 p-values)",
            "collect_steps": burn, "collect_s": collect_s, "samples": info["n_samples"],
            "train_iterations": iters, "train_batch": 8192, "train_s": train_s,
            "train_loss_first_last": [float(losses[0]), float(losses[-1])],
            "exact_stage_split": split_used,
            "intervals": intervals, "ms_per_interval": da_ms / intervals,
            "gpu_launches_per_interval": 3 + 5 * spe + 1,
            "timing": "CUDA events on each engine's stream, L2 flushed between intervals"}


def integrated_autocorr_time(x, c=5.0):
    """Integrated autocorrelation time of each row of x [chains, steps] (Sokal's automatic
    window: the smallest M with M >= c tau(M), tau(M) = 1 + 2 sum_{k=1..M} rho(k)); a chain
    that never moves has tau = steps. FFT autocovariance, float64."""
    x = np.asarray(x, np.float64)
    n = x.shape[1]
    y = x - x.mean(axis=1, keepdims=True)
    nf = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(y, nf, axis=1)
    acov = np.fft.irfft(f * np.conj(f), nf, axis=1)[:, :n]
    var = acov[:, 0]
    tau = np.full(x.shape[0], float(n))
    ok = var > 0
    rho = acov[ok] / var[ok, None]
    t = 2.0 * np.cumsum(rho, axis=1) - 1.0  # tau(M) for M = 0..n-1
    m = np.arange(n)[None, :]
    win = np.argmax(m >= c * t, axis=1)
    found = (m >= c * t).any(axis=1)
    tau_ok = np.where(found, t[np.arange(t.shape[0]), win], float(n))
    tau[ok] = np.clip(tau_ok, 1.0, float(n))
    return tau


def _energy_series(e0, e_prop, took):
    """Each chain's current energy after every step: the proposal's where it was taken."""
    cur = np.array(e0, np.float32)
    out = np.empty(e_prop.shape, np.float32)
    for t in range(e_prop.shape[1]):
        cur = np.where(took[:, t], e_prop[:, t], cur)
        out[:, t] = cur
    return out


def sampling_efficiency(w, dev, tile, scales=(1.0, 5.0, 20.0, 40.0, 60.0, 100.0), burn=1000, n=2000,
                        iters=1665):
    """Effective samples per second of plain Monte Carlo and of delayed acceptance on the
    config-1 system, each at its best move scale. Per scale: `burn` steps with exchange from
    the initial poses (for delayed acceptance these are the surrogate's collect steps, the same
    trajectory), one epoch of training, then `n` steps without exchange (every replica a
    chain at a fixed temperature) with each chain's energy traced; the integrated
    autocorrelation time tau of each chain's energy gives n / tau effective samples, summed
    over the chains and divided by the device time of the n steps (CUDA events)."""
    import torch
    from geaxdock_gpu_b200 import engine
    cx, ff = w.complexes[0], w.ff
    rows = []
    for m in scales:
        p = type(w.params).from_buffer_copy(w.params)
        p.record = 0
        for i in range(6):
            p.move_scale[i] = w.params.move_scale[i] * m
        row = {"move_mult": m}
        with engine.Engine(ff, [cx], p, device=dev) as a:
            a.set_tile(*tile)
            a.mc_init()
            a.run_fused(0, burn, exchange=True)
            s0 = burn + 10
            a.trace_enable(s0 + n)  # absolute steps 0 .. s0 + n - 1
            a.run_fused(burn, 10, exchange=False)  # builds the 10-step graph
            a.sync()
            e0 = a.state()["energy_old"]["e"][:, 9].copy()
            st = torch.cuda.ExternalStream(a.cuda_stream(), device=dev)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(st)
            for s in range(s0, s0 + n, 10):
                a.run_fused(s, 10, exchange=False)
            ev[1].record(st)
            a.sync()
            ms = ev[0].elapsed_time(ev[1])
            te, ta = a.trace()
            te, ta = te[:, s0:], ta[:, s0:]
            ser = _energy_series(e0, te, ta == 1)
            tau = integrated_autocorr_time(ser)
            row["plain"] = {"accept": float((ta == 1).mean()), "ms": ms,
                            "tau_median": float(np.median(tau)),
                            "ess_per_s": float((n / tau).sum() / (ms * 1e-3))}
        with engine.Engine(ff, [cx], p, device=dev) as b:
            b.set_tile(*tile)
            b.mc_init()
            sur = engine.Surrogate(b, sample_cap=burn * cx.n_rep, fallback_accept=0.0)
            sur.collect(0, burn, exchange=True)
            sur.train(iters)
            s0 = burn + 20
            sur.trace_enable(s0, n)
            # two untraced calls build the step graph and settle the exact stage's split
            sur.run(burn, 10, exchange=False)
            sur.run(burn + 10, 10, exchange=False)
            b.sync()
            e0 = b.state()["energy_old"]["e"][:, 9].copy()
            st0 = sur.stats()[0]
            st = torch.cuda.ExternalStream(b.cuda_stream(), device=dev)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(st)
            for s in range(s0, s0 + n, 10):
                sur.run(s, 10, exchange=False)
            ev[1].record(st)
            b.sync()
            ms = ev[0].elapsed_time(ev[1])
            st1 = sur.stats()[0]
            _, e_tr, f_tr = sur.trace()
            ser = _energy_series(e0, e_tr, f_tr == 2)
            tau = integrated_autocorr_time(ser)
            passed = st1["passed"] - st0["passed"]
            row["delayed_acceptance"] = {
                "accept": float((f_tr == 2).mean()), "ms": ms,
                "stage1_pass": passed / max(1, st1["proposed"] - st0["proposed"]),
                "stage2_accept": (st1["accepted"] - st0["accepted"]) / max(1, passed),
                "tau_median": float(np.median(tau)),
                "ess_per_s": float((n / tau).sum() / (ms * 1e-3))}
        rows.append(row)
    bp = max(rows, key=lambda r: r["plain"]["ess_per_s"])
    bd = max(rows, key=lambda r: r["delayed_acceptance"]["ess_per_s"])
    return {"unit": "effective samples/s (sum over chains of n / tau_int of the energy)",
            "steps_traced": n, "burn": burn, "scales": rows,
            "plain_best": {"move_mult": bp["move_mult"], "ess_per_s": bp["plain"]["ess_per_s"]},
            "da_best": {"move_mult": bd["move_mult"],
                        "ess_per_s": bd["delayed_acceptance"]["ess_per_s"]},
            "da_over_plain": bd["delayed_acceptance"]["ess_per_s"] / bp["plain"]["ess_per_s"],
            "timing": "CUDA events on each engine's stream around the n traced steps"}


def batched_screen(dev, w, intervals=3):
    """Config 2: 2,048 ligands (10-64 atoms, 8 conformers) round-robin over 8 pockets (1,200-6,000
    points, 4 conformers), 16 temperatures = 1,048,576 replicas in one context; every interval is
    one graph-captured persistent launch over all complexes (10 steps) + exchange. Tile autotuned
    on this batch; device time from CUDA events; FLOP at 36 per ligand-protein pair."""
    import torch
    from geaxdock_gpu_b200 import autotune, engine
    pairs = sum(c.n_rep * c.lna * c.pnp for c in w.complexes)
    with engine.Engine(w.ff, w.complexes, w.params, device=dev) as eng:
        eng.mc_init()
        eng.sync()
        tuned = autotune.tune(eng, device=dev)
        st = torch.cuda.ExternalStream(eng.cuda_stream(), device=dev)
        spe = w.params.steps_per_exchange
        per_dump = w.params.steps_per_dump // spe
        eng.run_fused(0, spe, exchange=True)
        eng.sync()
        ms = []
        for i in range(1, intervals + 1):
            if i % per_dump == 0:
                eng.reset_records()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            eng.run_fused(i * spe, spe, exchange=True)
            e1.record(st)
            eng.sync()
            ms.append(e0.elapsed_time(e1))
        tile = eng.tile()
    avg = sum(ms) / len(ms)
    return {"workload": "config2: 2048 ligands (L 10-64, 8 conformers) x 8 pockets (P 1200-6000, "
                        "4 conformers), 16 T, 1,048,576 replicas, one persistent launch per interval",
            "value": w.n_rep * spe / (avg * 1e-3), "unit": UNIT, "ms_per_interval": avg,
            "intervals": intervals, "tflops_at_36_flop_per_pair": pairs * 36 * spe / (avg * 1e-3) / 1e12,
            "tile": {"replicas_per_cta": tile[0], "chunk_points": tile[1],
                     "unroll": tile[2], "split": tile[3], "threads": tile[4],
                     "replicas_per_lane": tile[5], "cached": tuned["cached"]}}, tile


def screen_da(dev, w, tile, move_mult=1.0, burn=100, steps=50, iters=1665, n_pockets=8):
    """Config 4: delayed acceptance on the config-2 screen with one network per pocket. The
    ligands are grouped by pocket (ligand i docks to pocket i mod 8); each pocket's ligands run
    in a context of their own (131,072 replicas, every complex keeping its batch index as RNG
    stream) with its own surrogate, trained on the proposals of that pocket's `burn` plain
    burn-in steps, and the per-ligand fallback to plain steps. The plain batched run (all
    ligands in one context) starts from the same state. Both are device-timed (CUDA events on
    each context's stream) over `steps` steps; per ligand, the best (lowest-energy) pose of its
    replicas at the end is compared between the two runs, by energy and by RMSD."""
    import contextlib
    import torch
    from geaxdock_gpu_b200 import engine
    p = type(w.params).from_buffer_copy(w.params)
    p.record = 0
    for i in range(6):
        p.move_scale[i] *= move_mult
    spe = p.steps_per_exchange
    n_cx = len(w.complexes)
    groups = [[i for i in range(n_cx) if i % n_pockets == k] for k in range(n_pockets)]
    ev = lambda: torch.cuda.Event(enable_timing=True)
    with contextlib.ExitStack() as stack:
        pk = []
        for idx in groups:
            e = stack.enter_context(engine.Engine(w.ff, [w.complexes[i] for i in idx], p,
                                                  device=dev))
            for j, i in enumerate(idx):
                e.set_rng_stream(j, i)
            e.set_tile(*tile)
            e.mc_init()
            sur = engine.Surrogate(e, fallback_accept=0.5, fallback_window=2000,
                                   sample_cap=burn * e.n_rep)
            pk.append((e, sur, idx))
        t0 = time.perf_counter()
        for e, sur, _ in pk:
            sur.collect(0, burn, exchange=True)
        for e, _, _ in pk:
            e.sync()
        collect_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        losses = [sur.train(iters) for _, sur, _ in pk]
        train_s = time.perf_counter() - t0
        a = stack.enter_context(engine.Engine(w.ff, w.complexes, p, device=dev))
        a.set_tile(*tile)
        a.mc_init()
        full = a.state()
        for e, _, idx in pk:
            st = e.state()
            for j, i in enumerate(idx):
                n = w.complexes[i].n_rep
                full[a.offsets[i]:a.offsets[i] + n] = st[e.offsets[j]:e.offsets[j] + n]
        a.set_state(full)
        a.sync()
        sa = torch.cuda.ExternalStream(a.cuda_stream(), device=dev)
        spk = [torch.cuda.ExternalStream(e.cuda_stream(), device=dev) for e, _, _ in pk]
        da_ms = plain_ms = 0.0
        for s in range(burn, burn + steps, spe):
            evs = []
            for (e, sur, _), stream in zip(pk, spk):
                e0, e1 = ev(), ev()
                e0.record(stream)
                sur.run(s, spe, exchange=True)
                e1.record(stream)
                evs.append((e0, e1))
            for e, _, _ in pk:
                e.sync()
            da_ms += sum(x.elapsed_time(y) for x, y in evs)
            e2, e3 = ev(), ev()
            e2.record(sa)
            a.run_fused(s, spe, exchange=True)
            e3.record(sa)
            a.sync()
            plain_ms += e2.elapsed_time(e3)
        fa = a.state()
        best = {"da_e": np.zeros(n_cx), "da_r": np.zeros(n_cx), "pl_e": np.zeros(n_cx),
                "pl_r": np.zeros(n_cx)}
        per_pocket = []
        for (e, sur, idx), ls in zip(pk, losses):
            st, stats = e.state(), sur.stats()
            for j, i in enumerate(idx):
                n = w.complexes[i].n_rep
                mine = st[e.offsets[j]:e.offsets[j] + n]["energy_old"]
                k = int(np.argmin(mine["e"][:, 9]))
                best["da_e"][i], best["da_r"][i] = mine["e"][k, 9], mine["rmsd"][k]
                ref = fa[a.offsets[i]:a.offsets[i] + n]["energy_old"]
                k = int(np.argmin(ref["e"][:, 9]))
                best["pl_e"][i], best["pl_r"][i] = ref["e"][k, 9], ref["rmsd"][k]
            prop = sum(x["proposed"] for x in stats)
            passed = sum(x["passed"] for x in stats)
            per_pocket.append({"ligands": len(idx), "replicas": e.n_rep,
                               "pocket_points": w.complexes[idx[0]].pnp,
                               "train_loss_first_last": [float(ls[0]), float(ls[-1])],
                               "proposed": prop, "passed": passed,
                               "accepted": sum(x["accepted"] for x in stats),
                               "stage1_pass": passed / max(1, prop),
                               "stage2_accept": sum(x["accepted"] for x in stats) / max(1, passed),
                               "rmse": float(np.sqrt(np.mean([x["rmse"] ** 2 for x in stats]))),
                               "ligands_fallen_back": sum(1 for x in stats if not x["active"])})
    prop = sum(x["proposed"] for x in per_pocket)
    passed = sum(x["passed"] for x in per_pocket)
    acc = sum(x["accepted"] for x in per_pocket)
    rs = w.n_rep * steps
    de, dr = best["da_e"] - best["pl_e"], best["da_r"] - best["pl_r"]
    return {"workload": "config4: config-2 screen (2,048 ligands x 8 pockets, 1,048,576 replicas) "
                        "with delayed acceptance, one surrogate per pocket",
            "move_scale": [p.move_scale[i] for i in range(6)],
            "value": rs / (da_ms * 1e-3), "unit": UNIT,
            "plain_same_state": rs / (plain_ms * 1e-3), "speedup_vs_plain": plain_ms / da_ms,
            "stage1_pass": passed / max(1, prop), "stage2_accept": acc / max(1, passed),
            "ligands_fallen_back_to_plain": sum(x["ligands_fallen_back"] for x in per_pocket),
            "ligands": n_cx, "networks": len(pk), "per_pocket": per_pocket,
            "collect_steps": burn, "collect_s": collect_s, "train_iterations": iters,
            "train_s": train_s, "steps": steps,
            "best_pose": {
                "energy_mean_da_plain": [float(best["da_e"].mean()), float(best["pl_e"].mean())],
                "energy_median_abs_diff": float(np.median(np.abs(de))),
                "energy_corr": float(np.corrcoef(best["da_e"], best["pl_e"])[0, 1]),
                "rmsd_mean_da_plain": [float(best["da_r"].mean()), float(best["pl_r"].mean())],
                "rmsd_median_abs_diff": float(np.median(np.abs(dr))),
                "rmsd_corr": float(np.corrcoef(best["da_r"], best["pl_r"])[0, 1]),
                "note": "per ligand, the lowest-energy replica at the end of each run, both runs "
                        "from the same burned-in state"},
            "timing": "CUDA events on each context's stream; delayed acceptance summed over the "
                      "pockets' contexts, run one after another"}


def post_mc_measure(eng, cx, args):
    """post_mc clustering (per-replica k = 50, pooled k = 500) of the timed run's records on
    the GPU, host wall clock including the upload; beside it the CPU restatement of the
    reference's k-means (oracle/kmeans.py) on the first stage of a few replicas."""
    from geaxdock_gpu_b200 import postmc
    steps, nxt = eng.records()
    recs = [steps[i, :nxt[i]] for i in range(cx.n_rep)]
    n_rec = int(nxt.sum())
    postmc.post_mc(recs[:8], seed=1)  # warm-up (module load, allocations)
    t0 = time.perf_counter()
    med, size = postmc.post_mc_steps(steps, nxt, seed=1)
    gpu_s = time.perf_counter() - t0
    out = {"records": n_rec, "replicas": cx.n_rep, "representatives": int(med.shape[0]),
           "gpu_s": gpu_s, "records_per_s": n_rec / gpu_s,
           "scope": "postmc.post_mc_steps on the records as downloaded: upload, batched k-means "
                    "(50 per replica), pooled k-means "
                    "(500), host wall clock"}
    if not args.no_cpu:
        from oracle import kmeans as ok
        n_s = 4
        t0 = time.perf_counter()
        for i in range(n_s):
            ok.cluster_by_kmeans(recs[i]["energy"]["e"][:, :9], 50, 1, i)
        cpu_s = time.perf_counter() - t0
        out["cpu_sample"] = {"s": cpu_s, "sample": "first-stage k-means of %d replicas with the "
                             "oracle's numpy restatement of seq_kmeans, one core" % n_s,
                             "first_stage_estimate_s": cpu_s * cx.n_rep / n_s}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from geaxdock_gpu_b200 import abi, engine

    dev = local_rank
    torch.cuda.set_device(dev)
    # one batch of `world` config-1 complexes (complex i drawn with seed 42 + i, RNG stream i),
    # split across the ranks by shard_batch's assignment; at N = 1 it is config 1 itself
    from geaxdock_gpu_b200 import shard, system
    mine = shard.assign_complexes([shard.complex_cost(6820, 40, 3000)] * world, world)[rank]
    w = system.config1_batch(load_raw(), mine)
    cx, ff, params = w.complexes[0], w.ff, w.params
    n_total = world * cx.n_rep  # replicas of the whole batch (every complex has 6,820)
    spe = params.steps_per_exchange
    intervals_per_dump = params.steps_per_dump // spe
    dist = None
    if world > 1:
        import torch.distributed as dist

    # ---------------- device-timed throughput ----------------
    eng = engine.Engine(ff, w.complexes, params, device=dev)
    for j, i in enumerate(mine):
        eng.set_rng_stream(j, i)
    eng.mc_init()
    eng.sync()
    stream = torch.cuda.ExternalStream(eng.cuda_stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:%d" % dev)
    it = 0

    def one_step(ev=None):
        nonlocal it
        if it and it % intervals_per_dump == 0:
            eng.reset_records()
        s1 = (it // intervals_per_dump) * params.steps_per_dump
        s2 = (it % intervals_per_dump) * spe
        if ev is not None:
            ev[0].record(stream)
        # one graph launch: the Monte Carlo kernel with the exchange fused into its end
        # (mode_t from the interval's step within the dump window, as mc_run + exchange)
        eng.run_fused(s1 + s2, spe, exchange=True)
        if ev is not None:
            ev[1].record(stream)
            ev[2].record(stream)
        it += 1

    for _ in range(args.warmup):
        one_step()
    eng.sync()
    # the tile is chosen after the warm-up intervals, from a chain state like the timed one's
    # (the autotuner leaves the chains as they were), then used for one more warm-up interval
    if args.tile:
        eng.set_tile(*(int(v) for v in args.tile.split(",")))
        tile_source = "given"
    else:
        from geaxdock_gpu_b200 import autotune
        tile_source = "autotuned (cached)" if autotune.tune(eng, device=dev)["cached"] \
            else "autotuned"
    tile_used = eng.tile()
    one_step()
    eng.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev)
    clocks.start()
    evs = []
    for _ in range(args.steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        one_step(e)
        with torch.cuda.stream(stream):
            flush.add_(1.0)  # 256 MB write between steps: L2 (126 MB) flushed
        evs.append(e)
    eng.sync()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    step_ms = [a.elapsed_time(c) for a, b, c in evs]
    mc_ms = [a.elapsed_time(b) for a, b, c in evs]
    tot_ms = sum(step_ms)
    if dist:
        from geaxdock_gpu_b200.shard import max_over_ranks
        tot_ms = max_over_ranks(tot_ms, dist)
    rs_per_step = eng.n_rep * spe
    value = n_total * spe * args.steps / (tot_ms * 1e-3)
    flops_rs = algorithmic_flops_per_replica_step(eng, w) if rank == 0 else 0.0
    post = None
    if world == 1 and not args.no_postmc:
        post = post_mc_measure(eng, cx, args)
    eng.close()
    del flush

    # ---------------- end to end through the C ABI (host buffers) ----------------
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        h2d = 0
        for c in w.complexes:
            for name in ("lig_x", "lig_y", "lig_z", "lig_center", "lig_t", "lig_c", "lig_n",
                         "prt_x", "prt_y", "prt_z", "prt_t", "prt_c", "prt_ele", "prt_seq3r",
                         "prt_hflag", "prt_hpp", "psp", "kde_x", "kde_y", "kde_z", "kde_t",
                         "mcs_x", "mcs_y", "mcs_z", "mcs_tcc", "temp"):
                h2d += getattr(c, name).nbytes
        h2d += C.sizeof(abi.EnePara)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e = engine.Engine(ff, w.complexes, params, device=dev)
        for j, i in enumerate(mine):
            e.set_rng_stream(j, i)
        e.set_tile(*tile_used)
        e.mc_init()
        it2 = 0
        d2h = 0
        # each dump window's filled records, downloaded before the counters reset into one host
        # array reused from window to window, as the reference's launcher reuses its host
        # LigRecord array (the records held per window are kept). At 100 intervals and the
        # default 2,000-step dump window there is one window, downloaded at the end.
        rec_host = np.empty(e.n_rep * e.cap, abi.RECORD_DTYPE)
        held = []

        def download():
            steps, nxt = e.records(out=rec_host)
            held.append(int(nxt.sum()))
            return steps.nbytes + nxt.nbytes

        for _ in range(args.steps):
            if it2 and it2 % intervals_per_dump == 0:
                d2h += download()
                e.reset_records()
            s2 = (it2 % intervals_per_dump) * spe
            e.run_fused((it2 // intervals_per_dump) * params.steps_per_dump + s2, spe,
                        exchange=True)
            et = e.etotal()  # the step's result read back to the host
            d2h += et.nbytes
            it2 += 1
        d2h += download()
        e.close()
        dt = time.perf_counter() - t0
        if dist:
            from geaxdock_gpu_b200.shard import max_over_ranks
            dt = max_over_ranks(dt, dist)
        e2e = {"value": n_total * spe * args.steps / dt, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "records_downloaded": sum(held),
               "scope": "gd_create + gd_mc_init + K x (gd_mc_run_fused over one interval, "
                        "the exchange inside the Monte Carlo kernel, + gd_get_etotal) + the "
                        "filled record rows of every dump window "
                        "(gd_get_record_counts + gd_get_records_raw into one host array reused "
                        "per window, as the reference's launcher downloads LigRecord per dump into "
                        "its host array) + gd_destroy, host wall clock, every rank its shard of "
                        "the batch, slowest rank"}

    if rank != 0:
        return
    mc_avg_ms = sum(mc_ms) / len(mc_ms)
    flops_launch = flops_rs * rs_per_step
    achieved = flops_launch / (mc_avg_ms * 1e-3) / 1e12
    peak = None
    try:
        import ctypes as C
        v = C.c_double()
        if engine.lib().gd_probe_fp32_peak(dev, 5, C.byref(v)) == 0:
            peak = v.value
    except Exception:
        peak = None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "gd_mc_kernel_config1_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("bytes_per_launch")
        except Exception:
            traffic = None
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None, "traffic": traffic,
                "kernel": "gd_mc_kernel", "launch_ms": mc_avg_ms,
                "flop_per_replica_step": flops_rs,
                "peak_source": "measured FP32 FMA probe (gd_probe_fp32_peak), same run"}

    da = None
    if world == 1 and not args.no_da:
        da = {"configured_moves": delayed_acceptance(w, dev, tile_used, 1.0, args.steps),
              "moves_x20": delayed_acceptance(w, dev, tile_used, 20.0, args.steps),
              "moves_x60": delayed_acceptance(w, dev, tile_used, 60.0, args.steps),
              "sampling_efficiency": sampling_efficiency(w, dev, tile_used)}

    screen = screen4 = None
    if world == 1 and not args.no_screen:
        from geaxdock_gpu_b200 import system
        t0 = time.perf_counter()
        w2 = system.config(2, load_raw())
        gen_s = time.perf_counter() - t0
        screen, tile2 = batched_screen(dev, w2)
        screen["generate_s"] = gen_s
        if not args.no_da:
            screen4 = {"configured_moves": screen_da(dev, w2, tile2, 1.0),
                       "moves_x20": screen_da(dev, w2, tile2, 20.0)}
        del w2

    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample(w)

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded, config-1 shapes)",
           "config": bench_config(world),
           "tile": {"replicas_per_cta": tile_used[0], "chunk_points": tile_used[1],
                    "unroll": tile_used[2], "split": tile_used[3], "threads": tile_used[4],
                    "replicas_per_lane": tile_used[5], "source": tile_source},
           "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
           "gpu_launches": args.steps + args.steps // max(1, intervals_per_dump),
           "delayed_acceptance": da, "batched_screen": screen, "screen_delayed_acceptance": screen4,
           "post_mc": post}
    print(json.dumps(out), flush=True)


def profile_aux(args):
    """The small kernels around the Monte Carlo kernel, on a 128-replica subset of the config-1
    system: a record stream over four 10-step intervals (copy plan + gather per interval), the
    exchange after each, and the placement of 4,096 poses (gd_place_ligand)."""
    from geaxdock_gpu_b200 import engine
    w = workload(42)
    cx = w.complexes[0].subset(n_lig=8, n_prt=2, n_tmp=8)
    params = w.params
    with engine.Engine(w.ff, [cx], params) as e:
        e.set_tile(6, 1024, 2)
        e.mc_init()
        e.stream_records(64)
        for it in range(4):
            e.mc_run(0, it * params.steps_per_exchange)
            e.exchange(int(not (it % 2)))
        steps, nxt = e.stream_flush()
        mm = np.random.default_rng(1).normal(0, 1, (4096, 6)).astype(np.float32)
        xyz = e.place_ligand(0, 0, mm)
        e.stream_stop()
    print(json.dumps({"profile_aux": {"replicas": cx.n_rep, "records": int(nxt.sum()),
                                      "poses": int(xyz.shape[0])}}), flush=True)


def da_ks_seeds(seeds, move_mult):
    """The delayed-acceptance comparison of the config-3 workload repeated with several Philox
    seeds: every per-temperature KS p-value of DA against plain (final states of the 341
    independent chains per temperature), pooled, and the same for plain against plain with
    another seed. Both arms of a comparison start from one state, and DA draws the plain
    chain's moves and accept uniforms, so the arms are positively coupled and p-values lean
    high; a difference between their distributions would instead make small p-values too
    frequent, which the one-sided uniformity test (small_p_excess_ks_p) measures."""
    from scipy import stats
    pooled, null, rows = [], [], []
    for sd in seeds:
        w = workload(42)
        w.params.seed = sd
        r = delayed_acceptance(w, 0, (6, 1024, 2), move_mult, 100)
        pooled += r["ks_p_per_temperature"]
        null += r["ks_null_p_per_temperature"]
        rows.append({"seed": sd, "ks_min_p": r["ks_min_p"], "ks_null_min_p": r["ks_null_min_p"],
                     "speedup_vs_plain": r["speedup_vs_plain"],
                     "stage1_pass": r["stage1_pass"]})
    def summary(v):
        v = np.asarray(v)
        # "greater": the p-values' CDF lies above the uniform one, i.e. small p-values are
        # too frequent, which a difference between the chains' distributions would cause
        return {"p_values": len(v), "mean": float(v.mean()),
                "frac_below_0.01": float((v < 0.01).mean()),
                "frac_below_0.05": float((v < 0.05).mean()),
                "uniformity_ks_p": float(stats.kstest(v, "uniform").pvalue),
                "small_p_excess_ks_p": float(stats.kstest(v, "uniform",
                                                          alternative="greater").pvalue),
                "values": [round(float(x), 4) for x in v]}
    return {"da_ks": {"move_mult": move_mult, "runs": rows, "da_vs_plain": summary(pooled),
                      "plain_vs_plain": summary(null)}}


def profile_da(args):
    from geaxdock_gpu_b200 import engine
    w = workload(42)
    cx, ff, params = w.complexes[0], w.ff, w.params
    params.record = 0
    for i in range(6):
        params.move_scale[i] *= args.move_mult
    with engine.Engine(ff, [cx], params) as b:
        if args.tile:
            b.set_tile(*(int(v) for v in args.tile.split(",")))
        b.mc_init()
        sur = engine.Surrogate(b, sample_cap=1 << 20, fallback_accept=0.0)
        sur.collect(0, 20, exchange=True)
        sur.train(20)
        sur.run(20, 20, exchange=True)
        b.run_fused(40, 10, exchange=True)
        b.sync()
        print(json.dumps({"profile_da": sur.stats()[0]}), flush=True)


def profile_mc(args):
    """A short plain run on a subset of the config-1 system (--profile-subset ligand
    conformers, protein conformers, temperatures; default 8, 2, 8 = 128 replicas; no records):
    four 10-step launches, small enough for multi-pass profiler captures."""
    from geaxdock_gpu_b200 import engine
    w = workload(42)
    nl, npc, nt = (int(v) for v in args.profile_subset.split(","))
    cx = w.complexes[0].subset(n_lig=nl, n_prt=npc, n_tmp=nt)
    params = w.params
    params.record = 0
    tile = tuple(int(v) for v in args.tile.split(",")) if args.tile else (6, 1024, 2)
    with engine.Engine(w.ff, [cx], params) as e:
        e.set_tile(*tile)
        e.mc_init()
        for it in range(4):
            e.mc_run(0, it * params.steps_per_exchange)
        e.sync()
    print(json.dumps({"profile_mc": {"replicas": cx.n_rep, "launches": 4, "tile": tile}}),
          flush=True)


def profile_screen(args):
    """A slice of the config-2 screen small enough for multi-pass profiler captures: the first
    --screen-ligands ligands (uneven 10-64 atoms, 8 conformers) on their pockets (uneven
    1,200-6,000 points, 4 conformers), 16 temperatures, no records, the 256-lane fill tile with
    512-point chunks; four 10-step launches of gd_mc_run."""
    from geaxdock_gpu_b200 import engine, system
    w = system.config(2, load_raw(), n_ligands=args.screen_ligands)
    p = w.params
    p.record = 0
    tile = tuple(int(v) for v in args.tile.split(",")) if args.tile else (0, 512, 1, 1, 256)
    with engine.Engine(w.ff, w.complexes, p) as e:
        e.set_tile(*tile)
        e.mc_init()
        for it in range(4):
            e.mc_run(0, it * p.steps_per_exchange)
        e.sync()
        pairs = sum(c.n_rep * c.lna * c.pnp for c in w.complexes)
    print(json.dumps({"profile_screen": {"ligands": len(w.complexes), "replicas": w.n_rep,
                                         "pairs_per_step": pairs, "launches": 4,
                                         "tile": tile}}), flush=True)


def sweep(args):
    """Device time of one 10-step gd_mc_run on the config-1 system (no records): for each tile
    of --sweep-tiles over all replicas, and, at the first of them, over the first m protein-
    conformer blocks of 620 replicas (m = 1..11), with L2 flushed before every timed launch;
    and the fused graph as 1..4 concurrent chains. Medians of 5 launches, every measurement
    from the same chain state (the one after 5 warm-up intervals; the cost of a step depends on
    where the ligands are)."""
    import torch
    from geaxdock_gpu_b200 import engine
    w = workload(42)
    cx, ff, p = w.complexes[0], w.ff, w.params
    p.record = 0
    tiles = [tuple(int(v) for v in t.split(",")) for t in args.sweep_tiles.split(";")]
    out = {"tiles": {}, "blocks": {}, "chains": {}}
    with engine.Engine(ff, [cx], p) as e:
        e.mc_init()
        e.sync()
        st = torch.cuda.ExternalStream(e.cuda_stream())
        flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
        s = [0]

        def timed(fn, reps=5):
            fn()
            fn()
            ms = []
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(st):
                    flush.add_(1.0)
                a.record(st)
                fn()
                b.record(st)
                e.sync()
                ms.append(a.elapsed_time(b))
            return round(float(np.median(ms)), 3)

        def run(r1=None):
            def f():
                e.mc_run(0, s[0], 0, r1)
                s[0] += 10
            return f

        for _ in range(5):
            run()()
        e.sync()
        saved, s0 = e.state(), s[0]

        def restore():
            e.set_state(saved)
            s[0] = s0

        for t in tiles:
            e.set_tile(*t)
            restore()
            out["tiles"][",".join(map(str, t))] = timed(run())
        e.set_tile(*tiles[0])
        block = cx.n_tmp * cx.n_lig
        for m in range(1, cx.n_prt + 1):
            restore()
            out["blocks"][m] = timed(run(m * block - 1))
        for ch in (1, 2, 3, 4):
            e.set_concurrency(ch, 3)
            restore()

            def g():
                e.run_fused(s[0], 10, exchange=True)
                s[0] += 10
            out["chains"][ch] = timed(g)
    print(json.dumps({"sweep": out}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-da", action="store_true", help="skip the delayed-acceptance runs")
    ap.add_argument("--no-screen", action="store_true", help="skip the config-2 batched screen")
    ap.add_argument("--no-postmc", action="store_true",
                    help="skip the post_mc clustering of the timed run's records")
    ap.add_argument("--tile", default="", help="replicas_per_cta,chunk_points[,unroll] (default: tuned)")
    ap.add_argument("--profile-da", action="store_true",
                    help="only a short delayed-acceptance sequence on the config-1 system (20 "
                         "collect steps, 20 Adam steps, 20 DA steps, 10 plain steps), for "
                         "profiler launch lists; prints its statistics")
    ap.add_argument("--profile-aux", action="store_true",
                    help="only the record-stream, exchange and placement kernels on a small "
                         "case, for profiler captures")
    ap.add_argument("--da-ks", default="",
                    help="only the delayed-acceptance KS comparison at --move-mult, once per "
                         "Philox seed of this comma-separated list, p-values pooled")
    ap.add_argument("--move-mult", type=float, default=1.0,
                    help="--profile-da / --screen-da: move scales multiplied by this factor")
    ap.add_argument("--profile-mc", action="store_true",
                    help="only a short plain run on a subset of the config-1 system (four "
                         "10-step launches), for multi-pass profiler captures")
    ap.add_argument("--profile-subset", default="8,2,8",
                    help="--profile-mc: ligand conformers, protein conformers and temperatures "
                         "of the config-1 subset (default 128 replicas)")
    ap.add_argument("--profile-screen", action="store_true",
                    help="only a short plain run on a --screen-ligands slice of the config-2 "
                         "screen (four 10-step launches), for multi-pass profiler captures")
    ap.add_argument("--screen-ligands", type=int, default=64)
    ap.add_argument("--sweep", action="store_true",
                    help="only the launch-time sweep over --sweep-tiles, replica blocks and "
                         "concurrent chains on the config-1 system; prints its own JSON line")
    ap.add_argument("--sweep-tiles", default="6,1024,2,1,0,1;6,1024,1,1,0,1;6,1024,2,1,0,2;"
                                               "6,512,1,1,0,2;6,1024,1,1,0,2;6,2048,1,1,0,2",
                    help="';'-separated tiles for --sweep")
    ap.add_argument("--screen-da", action="store_true",
                    help="only the config-4 run (delayed acceptance on the config-2 screen); "
                         "prints its own JSON line")
    args = ap.parse_args()
    if args.screen_da:
        from geaxdock_gpu_b200 import system
        w2 = system.config(2, load_raw())
        _, tile2 = batched_screen(0, w2, intervals=1)
        print(json.dumps(screen_da(0, w2, tile2, args.move_mult)), flush=True)
        return
    if args.profile_aux:
        profile_aux(args)
        return
    if args.da_ks:
        print(json.dumps(da_ks_seeds([int(v) for v in args.da_ks.split(",")], args.move_mult)),
              flush=True)
        return
    if args.profile_da:
        profile_da(args)
        return
    if args.profile_mc:
        profile_mc(args)
        return
    if args.sweep:
        sweep(args)
        return
    if args.profile_screen:
        profile_screen(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
