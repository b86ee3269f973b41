"""The reference's own Monte Carlo step code timed on the host (the benchmark's reference arm):
the harness reads the product's arrays, runs every replica of its range and its acceptance
matches what the same moves give in the oracle's restatement to within sampling noise."""
import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, system
from oracle import refbench
from tests.golden.fixtures import load_ref

pytestmark = pytest.mark.skipif(not refbench.available(),
                                reason="oracle/_ref/refpin not built (needs the reference tree)")


def test_reference_steps_run_on_the_synthetic_system(tmp_path):
    z, _, _ = load_ref("1a07C1")
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    w = system.config(0, raw)
    cx, ff, p = w.complexes[0], w.ff, w.params
    r = refbench.run(cx, ff, p, n_rep=16, steps=5, procs=4, workdir=str(tmp_path))
    assert r["replica_steps"] == 80 and r["processes"] == 4
    assert r["seconds"] > 0
    # small uniform moves (the configured 0.1 A / 0.05 rad as the reference's scales): most
    # proposals are accepted, as in the product
    assert 0.5 < r["accepted"] / r["replica_steps"] <= 1.0


def test_reference_steps_take_the_configured_gaussian_moves(tmp_path):
    """The container's move kind reaches Move_d: Gaussian moves of the configured scales give
    a different acceptance count from uniform moves of the same scales on the same replicas."""
    z, _, _ = load_ref("1a07C1")
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    w = system.config(0, raw)
    cx, ff, p = w.complexes[0], w.ff, w.params
    assert p.move_kind == abi.MOVE_GAUSSIAN
    for i in range(6):
        p.move_scale[i] *= 20.0
    g = refbench.run(cx, ff, p, n_rep=32, steps=5, procs=4, workdir=str(tmp_path))
    p.move_kind = abi.MOVE_UNIFORM
    u = refbench.run(cx, ff, p, n_rep=32, steps=5, procs=4, workdir=str(tmp_path))
    assert g["replica_steps"] == u["replica_steps"] == 160
    assert g["accepted"] != u["accepted"]
