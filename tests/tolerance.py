"""Error metric for energy parity, written once for every parity test.

Energies are compared on the stored (normalised, unweighted) terms e_i = a_i * raw_i + b_i and
on the weighted total e_9 = sum_i w_i e_i. A term that is a sum of many signed pair
contributions is compared against its conditioning scale rather than its value:

    scale_i = |a_i| * max(|raw_i|, mag_i) + |b_i| * 2^-23      (i = 0..6)
    scale_7 = |a_7| * max(|raw_7|, 1) + ...,   scale_8 = |a_8| * max(|raw_8|, 1) + ...
    scale_9 = sum_i |w_i| * scale_i

with mag_i = sum of |contribution| / lna from the FP64 oracle. rel_i = |x_i - ref_i| / scale_i.
A value with no cancellation has mag_i == |raw_i|, so rel_i is then the plain relative error.
"""
import numpy as np

EPS32 = 2.0 ** -23


def scales(oracle: dict, ff) -> np.ndarray:
    a = np.array(ff.a_para[:9], np.float64)
    b = np.array(ff.b_para[:9], np.float64)
    w = np.array(ff.w[:9], np.float64)
    raw = np.asarray(oracle["raw"], np.float64)
    mag = np.asarray(oracle["mag"], np.float64)
    s = np.zeros(10)
    base = np.maximum(np.abs(raw[:7]), mag)
    s[:7] = np.abs(a[:7]) * base + np.abs(b[:7]) * EPS32
    s[7] = np.abs(a[7]) * max(abs(raw[7]), 1.0) + abs(b[7]) * EPS32
    s[8] = np.abs(a[8]) * max(abs(raw[8]), 1.0) + abs(b[8]) * EPS32
    s[9] = np.sum(np.abs(w) * s[:9])
    return s


def rel_errors(values, oracle: dict, ff) -> np.ndarray:
    """values: 10 stored energies (e[0..9]) to check against the FP64 oracle."""
    v = np.asarray(values, np.float64)[:10]
    ref = np.asarray(oracle["e"], np.float64)[:10]
    return np.abs(v - ref) / scales(oracle, ff)
