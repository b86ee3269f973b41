"""ctypes front end of the oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU-baseline leg of
bench.py, as the checker and the reported CPU baseline. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from geaxdock_gpu_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


class OEnergy(C.Structure):
    _fields_ = [("e", C.c_double * 10), ("raw", C.c_double * 9), ("mag", C.c_double * 7),
                ("cms", C.c_double), ("rmsd", C.c_double),
                ("tp", C.c_int64), ("fn", C.c_int64), ("fp", C.c_int64), ("tn", C.c_int64),
                ("hits_hpc", C.c_int64), ("hits_hdb", C.c_int64), ("hits_psp", C.c_int64),
                ("hits_kde", C.c_int64), ("hits_mcs", C.c_int64)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, fp, ip, dp = C.c_void_p, abi.FP, abi.IP, C.POINTER(C.c_double)
        u32p = C.POINTER(C.c_uint32)
        L.gdo_energy_eval.argtypes = [C.POINTER(abi.EnePara), C.POINTER(abi.ComplexDesc), C.c_int,
                                      C.c_int, fp, fp, fp, fp, C.c_void_p, C.c_int,
                                      C.POINTER(OEnergy)]
        L.gdo_place_f32.argtypes = [C.POINTER(abi.ComplexDesc), C.c_int, fp, fp, fp, fp, fp]
        L.gdo_place_f64.argtypes = [C.POINTER(abi.ComplexDesc), C.c_int, fp, dp, dp, dp, dp]
        L.gdo_ref_map.argtypes = [C.POINTER(abi.EnePara), C.POINTER(abi.ComplexDesc), C.c_void_p]
        L.gdo_fold_enepara.argtypes = [C.POINTER(abi.EneParaRaw), C.POINTER(abi.EnePara)]
        L.gdo_set_temperature.argtypes = [C.c_int, C.c_float, C.c_float, C.POINTER(abi.Temp)]
        L.gdo_contact_threshold.argtypes = [C.c_float]
        L.gdo_contact_threshold.restype = C.c_float
        L.gdo_philox.argtypes = [C.c_uint32] * 6 + [u32p]
        L.gdo_expf.argtypes = [C.c_float]
        L.gdo_expf.restype = C.c_float
        L.gdo_logf.argtypes = [C.c_float]
        L.gdo_logf.restype = C.c_float
        L.gdo_sincosf.argtypes = [C.c_float, fp, fp]
        L.gdo_draw_steps.argtypes = [C.c_uint64, C.c_uint32, C.c_int, fp, C.c_int, u32p, u32p, fp, fp]
        L.gdo_metropolis_batch.argtypes = [C.c_int, fp, fp, fp, fp, ip]
        L.gdo_draw_exchange.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.gdo_draw_exchange.restype = C.c_float
        L.gdo_mc_create.argtypes = [C.POINTER(abi.EnePara), C.POINTER(abi.ComplexDesc),
                                    C.POINTER(abi.McParams), C.c_int, C.c_int]
        L.gdo_mc_create.restype = vp
        L.gdo_mc_destroy.argtypes = [vp]
        L.gdo_mc_num_replicas.argtypes = [vp]
        L.gdo_mc_init.argtypes = [vp]
        L.gdo_mc_run.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.gdo_mc_run_range.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.gdo_mc_exchange.argtypes = [vp, C.c_int]
        L.gdo_mc_reset_records.argtypes = [vp]
        L.gdo_mc_get.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.gdo_mc_set.argtypes = [vp, vp, vp, vp, vp]
        L.gdo_mc_get_records.argtypes = [vp, vp, vp]
        L.gdo_mc_refmap.argtypes = [vp]
        L.gdo_mc_refmap.restype = C.POINTER(C.c_uint8)
        L.gdo_mc_exchange_calls.argtypes = [vp]
        L.gdo_mc_set_exchange_calls.argtypes = [vp, C.c_int]
        L.gdo_exchange_apply.argtypes = [C.POINTER(abi.ComplexDesc), C.c_uint64, C.c_int, C.c_int,
                                         C.c_int, vp, fp, ip]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def energy_eval(ff, cx: abi.ComplexArrays, prt_conf, lig_conf, x, y, z, center, refmap=None,
                precision=64) -> dict:
    x, y, z = (np.ascontiguousarray(v, np.float32) for v in (x, y, z))
    center = np.ascontiguousarray(center, np.float32)
    rm = None if refmap is None else np.ascontiguousarray(refmap, np.uint8)
    d = cx.desc()
    o = OEnergy()
    lib().gdo_energy_eval(C.byref(ff), C.byref(d), prt_conf, lig_conf, abi.fptr(x), abi.fptr(y),
                          abi.fptr(z), abi.fptr(center), _ptr(rm), precision, C.byref(o))
    return dict(e=np.array(o.e[:]), raw=np.array(o.raw[:]), mag=np.array(o.mag[:]), cms=o.cms,
                rmsd=o.rmsd, tp=o.tp, fn=o.fn, fp=o.fp, tn=o.tn, hits_hpc=o.hits_hpc,
                hits_hdb=o.hits_hdb, hits_psp=o.hits_psp, hits_kde=o.hits_kde,
                hits_mcs=o.hits_mcs)


def place_f32(cx: abi.ComplexArrays, lig_conf, mm):
    mm = np.ascontiguousarray(mm, np.float32)
    L = cx.lna
    out = np.zeros((3, L), np.float32)
    c = np.zeros(3, np.float32)
    d = cx.desc()
    lib().gdo_place_f32(C.byref(d), lig_conf, abi.fptr(mm), abi.fptr(out[0]), abi.fptr(out[1]),
                        abi.fptr(out[2]), abi.fptr(c))
    return out, c


def place_f64(cx: abi.ComplexArrays, lig_conf, mm):
    mm = np.ascontiguousarray(mm, np.float32)
    L = cx.lna
    out = np.zeros((3, L), np.float64)
    c = np.zeros(3, np.float64)
    d = cx.desc()
    dp = C.POINTER(C.c_double)
    lib().gdo_place_f64(C.byref(d), lig_conf, abi.fptr(mm), out[0].ctypes.data_as(dp),
                        out[1].ctypes.data_as(dp), out[2].ctypes.data_as(dp), c.ctypes.data_as(dp))
    return out, c


def ref_map(ff, cx: abi.ComplexArrays) -> np.ndarray:
    rm = np.zeros((cx.lna, cx.pnp), np.uint8)
    d = cx.desc()
    lib().gdo_ref_map(C.byref(ff), C.byref(d), _ptr(rm))
    return rm


def pose_energy(ff, cx, prt_conf, lig_conf, mm, refmap=None, precision=64):
    xyz, c = place_f32(cx, lig_conf, mm)
    return energy_eval(ff, cx, prt_conf, lig_conf, xyz[0], xyz[1], xyz[2], c, refmap, precision)


def fold_enepara(raw: abi.EneParaRaw) -> abi.EnePara:
    out = abi.EnePara()
    lib().gdo_fold_enepara(C.byref(raw), C.byref(out))
    return out


def set_temperature(n, floor_t, ceil_t) -> np.ndarray:
    t = (abi.Temp * n)()
    lib().gdo_set_temperature(n, floor_t, ceil_t, t)
    return np.frombuffer(bytes(t), dtype=abi.TEMP_DTYPE).copy()


def contact_threshold(pmf0: float) -> float:
    return lib().gdo_contact_threshold(pmf0)


def philox(c0, c1, c2, c3, k0, k1):
    out = (C.c_uint32 * 4)()
    lib().gdo_philox(c0, c1, c2, c3, k0, k1, out)
    return list(out)


def expf(x):
    return lib().gdo_expf(x)


def logf(x):
    return lib().gdo_logf(x)


def sincosf(x):
    s, c = C.c_float(), C.c_float()
    lib().gdo_sincosf(x, C.byref(s), C.byref(c))
    return s.value, c.value


def draw_steps(seed, move_kind, scale, replica, step, stream=0):
    replica = np.ascontiguousarray(replica, np.uint32)
    step = np.ascontiguousarray(step, np.uint32)
    n = replica.size
    scale = np.ascontiguousarray(scale, np.float32)
    delta = np.zeros((n, 6), np.float32)
    u = np.zeros(n, np.float32)
    u32p = C.POINTER(C.c_uint32)
    lib().gdo_draw_steps(seed, stream, move_kind, abi.fptr(scale), n, replica.ctypes.data_as(u32p),
                         step.ctypes.data_as(u32p), abi.fptr(delta), abi.fptr(u))
    return delta, u


def metropolis(e_new, e_old, mb, u):
    e_new, e_old, mb, u = (np.ascontiguousarray(a, np.float32) for a in (e_new, e_old, mb, u))
    out = np.zeros(e_new.size, np.int32)
    lib().gdo_metropolis_batch(e_new.size, abi.fptr(e_new), abi.fptr(e_old), abi.fptr(mb),
                               abi.fptr(u), abi.iptr(out))
    return out


def draw_exchange(seed, group, call, pair, stream=0):
    return lib().gdo_draw_exchange(seed, stream, group, call, pair)


def exchange_apply(cx: abi.ComplexArrays, seed, call, mode_t, replica, etotal, acs=None, stream=0):
    """Restated ExchangeReplicas_d on caller arrays; replica (REPLICA_DTYPE) updated in place."""
    d = cx.desc()
    etotal = np.ascontiguousarray(etotal, np.float32)
    lib().gdo_exchange_apply(C.byref(d), seed, stream, call, mode_t, _ptr(replica), abi.fptr(etotal),
                             None if acs is None else abi.iptr(acs))


class MC:
    """One complex's chain set: MonteCarlo_Init_d / MonteCarlo_d / ExchangeReplicas_d restated."""

    def __init__(self, ff, cx: abi.ComplexArrays, params: abi.McParams, stream=0, precision=32):
        self.cx = cx
        self._desc = cx.desc()
        self._ff = ff
        self._params = params
        self.h = lib().gdo_mc_create(C.byref(ff), C.byref(self._desc), C.byref(params),
                                     stream, precision)
        self.n_rep = lib().gdo_mc_num_replicas(self.h)
        self.cap = params.steps_per_dump + 1

    def __del__(self):
        if getattr(self, "h", None):
            lib().gdo_mc_destroy(self.h)
            self.h = None

    def init(self):
        lib().gdo_mc_init(self.h)

    def run(self, s1, s2, n_steps, nthreads=0):
        lib().gdo_mc_run(self.h, s1, s2, n_steps, nthreads)

    def run_range(self, r0, r1, s1, s2, n_steps, nthreads=0):
        lib().gdo_mc_run_range(self.h, r0, r1, s1, s2, n_steps, nthreads)

    def exchange(self, mode_t):
        lib().gdo_mc_exchange(self.h, mode_t)

    def reset_records(self):
        lib().gdo_mc_reset_records(self.h)

    @property
    def exchange_calls(self):
        return lib().gdo_mc_exchange_calls(self.h)

    @exchange_calls.setter
    def exchange_calls(self, n):
        lib().gdo_mc_set_exchange_calls(self.h, n)

    def get(self) -> dict:
        n = self.n_rep
        rep = np.zeros(n, abi.REPLICA_DTYPE)
        mm = np.zeros((n, 6), np.float32)
        e = np.zeros(n, abi.ENERGY_DTYPE)
        et = np.zeros(n, np.float32)
        na = np.zeros(n, np.int32)
        acs = np.zeros(n, np.int32)
        lib().gdo_mc_get(self.h, _ptr(rep), _ptr(mm), _ptr(e), _ptr(et), _ptr(na), _ptr(acs))
        return dict(replica=rep, mm_old=mm, e_old=e, etotal=et, n_accept=na, acs=acs)

    def set(self, replica=None, mm_old=None, e_old=None, etotal=None):
        lib().gdo_mc_set(self.h, _ptr(replica), _ptr(mm_old), _ptr(e_old), _ptr(etotal))

    def records(self):
        steps = np.zeros((self.n_rep, self.cap), abi.RECORD_DTYPE)
        nptr = np.zeros(self.n_rep, np.int32)
        lib().gdo_mc_get_records(self.h, _ptr(steps), _ptr(nptr))
        return steps, nptr

    def refmap(self) -> np.ndarray:
        p = lib().gdo_mc_refmap(self.h)
        n = self.cx.lna * self.cx.pnp
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self.cx.lna, self.cx.pnp).copy()


def max_threads() -> int:
    return lib().gdo_max_threads()
