"""The two arms of bench.py describe the same workload, and the reference arm runs without the
product's library: its force field is folded by the oracle's restatement of OptimizeEnepara,
which gives the library's fold bit for bit."""
import json
import os
import subprocess
import sys

import numpy as np

from geaxdock_gpu_b200 import abi, system
from oracle import pyoracle as po
from tests.golden.fixtures import load_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_fold_gives_the_library_fold_on_the_bench_system():
    z, _, _ = load_ref("1a07C1")
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    a = system.forcefield(raw, 42)
    b = system.forcefield(raw, 42, fold=po.fold_enepara)
    assert bytes(a) == bytes(b)


def test_reference_arm_prints_our_config_without_the_library():
    sys.path.insert(0, ROOT)
    import bench
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["config"] == bench.bench_config(1)
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")


def test_integrated_autocorrelation_time_of_ar1_chains():
    """AR(1) chains x_t = phi x_{t-1} + e_t have tau_int = (1 + phi) / (1 - phi); a chain that
    never moves counts as one sample."""
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(0)
    n, chains = 20000, 64
    for phi in (0.0, 0.5, 0.9):
        x = np.zeros((chains, n))
        e = rng.normal(size=(chains, n))
        for t in range(1, n):
            x[:, t] = phi * x[:, t - 1] + e[:, t]
        tau = bench.integrated_autocorr_time(x)
        want = (1 + phi) / (1 - phi)
        assert abs(np.median(tau) / want - 1) < 0.1, (phi, np.median(tau), want)
    still = np.ones((2, 100))
    assert np.all(bench.integrated_autocorr_time(still) == 100)


def test_energy_series_keeps_the_last_taken_proposal():
    sys.path.insert(0, ROOT)
    import bench
    e0 = np.array([1.0, 2.0], np.float32)
    prop = np.array([[5, 6, 7], [8, 9, 10]], np.float32)
    took = np.array([[0, 1, 0], [1, 0, 1]], bool)
    want = np.array([[1, 6, 6], [8, 8, 10]], np.float32)
    assert np.array_equal(bench._energy_series(e0, prop, took), want)
