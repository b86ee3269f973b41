"""Error metric for energy parity, written once for every parity test.

Energies are compared on the stored (normalised, unweighted) terms e_i = a_i * raw_i + b_i and
on the weighted total e_9 = sum_i w_i e_i, relative to the FP64 oracle:

    rel_i = |x_i - ref_i| / scale_i,
    scale_i = max(|ref_i|, |a_i| * max(|raw_i|, mag_i))          (i = 0..6)
    scale_i = max(|ref_i|, |a_i| * max(|raw_i|, 1))              (i = 7 lhm, 8 dst)
    scale_9 = max(|ref_9|, sum_i |w_i| * scale_i)

mag_i is the sum of |pair contribution| / lna from the oracle. Without cancellation
(mag_i == |raw_i|) this is the plain relative error |x - ref| / |ref| (or relative to the
term's own magnitude when the offset b_i dominates); when a signed sum cancels, the error is
measured against the sum of magnitudes, the scale that FP32 accumulation can be held to.

plain_rel_errors() is the plain relative error |x - ref| / |ref| of every term and the total,
reported beside it. The reference's own FP32 CalcEnergy_d (src/kernel_cuda_l2_calcenergy.cu,
run on the CPU by the pin harness) meets the sum-of-magnitudes metric within 1e-5 on every
term of its two real complexes, but not the plain one: its electrostatic term is off by up to
3.4e-3 of its own (cancelled) value on 1a07C1 and its vdw term by 1.6e-4 on 1robA1, while its
weighted total stays within 2.1e-6 plain (tests/test_oracle_pin.py).
"""
import numpy as np


def scales(oracle: dict, ff) -> np.ndarray:
    a = np.array(ff.a_para[:9], np.float64)
    w = np.array(ff.w[:9], np.float64)
    raw = np.asarray(oracle["raw"], np.float64)
    mag = np.asarray(oracle["mag"], np.float64)
    e = np.abs(np.asarray(oracle["e"], np.float64))
    s = np.zeros(10)
    s[:7] = np.maximum(e[:7], np.abs(a[:7]) * np.maximum(np.abs(raw[:7]), mag))
    s[7] = max(e[7], abs(a[7]) * max(abs(raw[7]), 1.0))
    s[8] = max(e[8], abs(a[8]) * max(abs(raw[8]), 1.0))
    s[9] = max(e[9], float(np.sum(np.abs(w) * s[:9])))
    return np.maximum(s, 1e-30)


def rel_errors(values, oracle: dict, ff) -> np.ndarray:
    """values: 10 stored energies (e[0..9]) to check against the FP64 oracle."""
    v = np.asarray(values, np.float64)[:10]
    ref = np.asarray(oracle["e"], np.float64)[:10]
    return np.abs(v - ref) / scales(oracle, ff)


def plain_rel_errors(values, oracle: dict) -> np.ndarray:
    """|x_i - ref_i| / |ref_i| for the 9 stored terms and the total (ref_i == 0: absolute)."""
    v = np.asarray(values, np.float64)[:10]
    ref = np.asarray(oracle["e"], np.float64)[:10]
    d = np.abs(v - ref)
    return np.where(ref != 0.0, d / np.maximum(np.abs(ref), 1e-300), d)


TERMS = ("vdw", "ele", "pmf", "psp", "hdb", "hpc", "kde", "lhm", "dst", "total")


def report(label: str, sumabs: np.ndarray, plain: np.ndarray) -> str:
    """One line per metric, worst error per term, for the test log."""
    f = lambda a: " ".join("%s %.2e" % (t, x) for t, x in zip(TERMS, a))
    line = "%s\n  sum-of-magnitudes: %s\n  plain relative:    %s" % (label, f(sumabs), f(plain))
    print(line)
    return line
