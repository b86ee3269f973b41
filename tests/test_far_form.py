"""The pmf far radius and the far-point bins behind the pair loop's far form, checked on the CPU.

The host sets the far radius r* of a type pair from (r/2 - 6)(r - pmf0) = 26 / log2(e)
(`pmf_far_radius` in geaxdock_gpu_b200/csrc/gd_capi.cu, restated here). Beyond it the kernel's
base-2 pmf exponent tt = fma(d2, fma(b2, r^-1, cA), c2), rounded in FP32, must stay below -25.5,
so that ee = 2^tt < 2^-25 and fma(p4, ee, p4) rounds back to p4: the far form's result equals the
full form's. This checks that bound for every pmf0 of the reference's force field (the pmf term
of src/kernel_cuda_l2_calcenergy.cu), at distances from r* to 150 A.
"""
import math

import numpy as np

from geaxdock_gpu_b200 import abi
from tests.golden.fixtures import load_ref

LOG2E = 1.4426950408889634


def far_radius(pmf0: float) -> float:
    k = 26.0 / LOG2E
    a = 6.0 + 0.5 * pmf0
    r = a + math.sqrt(max(0.0, a * a - 2.0 * (6.0 * pmf0 - k)))
    return max(r, 12.0, pmf0)


def _fma32(a, b, c):
    """fma rounded once to FP32 (the product of two FP32 values is exact in FP64)."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def test_far_radius_bounds_the_fp32_pmf_exponent():
    z, _, _ = load_ref("1a07C1")
    raw = abi.enepara_raw_from_array(z["enepara_raw"])
    pmf = np.ctypeslib.as_array(raw.pmf)
    pmf0s = np.unique(pmf[:, :, 0])
    assert pmf0s.size > 10
    ca = np.float32(-0.5 * np.float32(LOG2E))
    for p0 in pmf0s.astype(np.float64):
        rs = far_radius(p0) + 0.01
        b2 = np.float32(LOG2E * (6.0 + 0.5 * p0))
        c2 = np.float32(-6.0 * LOG2E * p0)
        r = np.linspace(rs, 150.0, 4000)
        d2 = (r * r).astype(np.float32)
        ri = (1.0 / np.sqrt(d2.astype(np.float64))).astype(np.float32)
        tt = _fma32(d2, _fma32(np.full_like(d2, b2), ri, np.full_like(d2, ca)), np.full_like(d2, c2))
        assert tt.max() < -25.5, (p0, tt.max())
        # exact exponent at r*: -26 in base 2
        x = (rs - 0.01) / 2.0 - 6.0
        assert abs(LOG2E * x * ((rs - 0.01) - p0) - 26.0) < 1e-9
        # p4 >= 1 and num of any sign are left unchanged by + (.) ee for ee < 2^-25
        ee = np.float32(2.0 ** -25.0) * np.float32(0.999999)
        v = np.float32(2.0) ** np.linspace(-20, 40, 2001).astype(np.float32)
        v = np.concatenate([v, np.nextafter(v, np.float32(0)), -v]).astype(np.float32)
        assert np.array_equal(_fma32(v, np.full_like(v, ee), v), v)


def test_far_bins_put_only_far_points_past_the_switch_slot():
    """The table and the switch slot, restated: the host counts each segment's points (ordered
    by distance from the pocket centre) inside radius (b + 1) w for 64 bins, all of them at the
    last (`layout_complex`); a warp takes b = min(63, floor((max atom distance + far_r) / w)) in
    FP32 and switches at the count rounded up to even (`gd_mc_kernel`). Every point from there on
    must lie beyond far_r of every atom of the warp, on random pockets and atoms, atoms inside
    and outside the point cloud."""
    rng = np.random.default_rng(5)
    nb = 64
    checked = 0
    for trial in range(200):
        n = int(rng.integers(1, 400))
        centre = rng.normal(0, 20, 3).astype(np.float32)
        pts = (centre + rng.normal(0, rng.uniform(3, 30), (n, 3))).astype(np.float32)
        rad = np.linalg.norm(pts.astype(np.float64) - centre.astype(np.float64), axis=1)
        order = np.argsort(rad, kind="stable")
        pts, rad = pts[order], rad[order]
        far_r = np.float32(far_radius(float(rng.uniform(2.5, 7.5))) + 0.01)
        w = (rad.max() + 1e-3) / (nb - 1)
        cnt = np.array([np.count_nonzero(rad < (b + 1) * w) for b in range(nb)])
        cnt[-1] = n
        inv_w = np.float32(1.0 / w)
        atoms = (centre + rng.normal(0, rng.uniform(1, 25), (32, 3))).astype(np.float32)
        d = atoms - centre
        a = np.sqrt((d * d).sum(axis=1, dtype=np.float32), dtype=np.float32)
        rho = (a + far_r).astype(np.float32)
        b = int(np.minimum(np.floor(rho * inv_w), np.float32(nb - 1)).max())
        split = (int(cnt[b]) + 1) & ~1
        if split >= n:
            continue
        dist = np.linalg.norm(pts[split:, None, :].astype(np.float64) - atoms[None, :, :], axis=2)
        assert dist.min() >= far_r - 1e-4, (trial, dist.min(), far_r)
        checked += 1
    assert checked > 50, checked
