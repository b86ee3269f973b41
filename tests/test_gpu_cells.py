"""The contacts, psp, hpc and the soft core of ele come from a per-conformer cell list
(short_range in csrc/gd_kernels.cu): energies at the edges of that grid against the FP64
oracle, which sums every pair."""
import copy

import numpy as np
import pytest

from geaxdock_gpu_b200 import abi, engine, system
from oracle import pyoracle as po
from tests.golden.fixtures import load_ref
from tests.tolerance import rel_errors

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def raw():
    z, _, _ = load_ref("1a07C1")
    return abi.enepara_raw_from_array(z["enepara_raw"])


def test_wide_protein_and_far_ligands_match_oracle(raw):
    """Half of the protein moved 700 A along each axis: the box then needs more than 2^22
    cells of 4 A, so the grid widens its cells. Poses at the pocket, at the moved half, on the
    way between them and far outside the grid."""
    w = system.config(0, raw)
    ff = w.ff
    cx = copy.deepcopy(w.complexes[0])
    half = cx.pnp // 2
    for a in (cx.prt_x, cx.prt_y, cx.prt_z):
        a[:, half:] += 700.0
    rm = po.ref_map(ff, cx)
    rng = np.random.default_rng(11)
    shifts = [(0.0, 0.0, 0.0), (700.0, 700.0, 700.0), (350.0, 350.0, 350.0),
              (-3000.0, 0.0, 0.0), (0.0, 2500.0, -2500.0)]
    mm = []
    for sh in shifts:
        for _ in range(4):
            m = np.zeros(6)
            m[:3] = np.asarray(sh) + rng.normal(0.0, 2.0, 3)
            m[3:] = rng.uniform(-3.1, 3.1, 3)
            mm.append(m)
    mm = np.asarray(mm, np.float32)
    with engine.Engine(ff, [cx], w.params) as eng:
        got = eng.eval_energy(0, 0, 0, mm)
    worst = np.zeros(10)
    contacts = 0
    for i in range(len(mm)):
        o = po.pose_energy(ff, cx, 0, 0, mm[i], rm, 64)
        worst = np.maximum(worst, rel_errors(got["e"][i], o, ff))
        assert abs(got["cms"][i] - o["cms"]) <= 2e-6, (i, got["cms"][i], o["cms"])
        contacts += int(o["hits_psp"] > 0 or o["hits_hpc"] > 0)
    assert worst.max() <= TOL, worst
    # the poses at both halves touch the protein, the far ones do not
    assert contacts >= 4
