"""Host-side mirror of the reference's docking run over the C ABI.

The reference drives its kernels from `Run` (src/run.cu:33-288) with the loop in
src/kernel_cuda_lancher_siglegpu.cu:17-63: ResetCounter_d + MonteCarlo_Init_d, then per dump
MonteCarlo_d every steps_per_exchange steps, ExchangeReplicas_d with alternating mode_t, a
LigRecord download and an append of accepted steps to map<int, vector<LigRecordSingleStep>>.
`Engine` exposes the same operations (`mc_init`, `mc_run`, `exchange`, `reset_records`,
`records`) plus the graph-captured fused loop (`run_fused`) and `run`, the whole reference
loop. Every call goes to libgeauxdock_b200.so; there is no CPU path: if the library or a
B200 is missing the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Sequence

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgeauxdock_b200.so")

_lib = None


class GDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("geauxdock error %d: %s" % (code, msg))
        self.code = code


def lib() -> C.CDLL:
    """Loads the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libgeauxdock_b200.so is missing; run `python -m geaxdock_gpu_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, ip, fp = C.c_void_p, C.POINTER(C.c_int), abi.FP
    sig = {
        "gd_fold_enepara": [C.POINTER(abi.EneParaRaw), C.POINTER(abi.EnePara)],
        "gd_set_temperature": [C.c_int, C.c_float, C.c_float, C.POINTER(abi.Temp)],
        "gd_set_replica": [C.c_int, C.c_int, C.c_int, C.POINTER(abi.Replica)],
        "gd_create": [C.POINTER(abi.EnePara), C.POINTER(abi.ComplexDesc), C.c_int,
                      C.POINTER(abi.McParams), C.c_int, C.POINTER(vp)],
        "gd_destroy": [vp],
        "gd_release_memory": [C.c_int],
        "gd_num_replicas": [vp, ip],
        "gd_replica_offset": [vp, C.c_int, ip],
        "gd_set_tile": [vp, C.c_int, C.POINTER(abi.Tile)],
        "gd_get_tile": [vp, C.c_int, C.POINTER(abi.Tile)],
        "gd_mc_init": [vp],
        "gd_reset_records": [vp, C.c_int, C.c_int],
        "gd_mc_run": [vp, C.c_int, C.c_int, C.c_int, C.c_int],
        "gd_exchange": [vp, C.c_int, C.c_int],
        "gd_mc_run_fused": [vp, C.c_int, C.c_int, C.c_int],
        "gd_sync": [vp],
        "gd_get_records": [vp, vp, C.c_int, C.c_int],
        "gd_get_records_raw": [vp, vp, vp, C.c_int, C.c_int, C.c_int],
        "gd_get_record_counts": [vp, vp, C.c_int, C.c_int],
        "gd_records_stream": [vp, vp, C.c_int],
        "gd_records_stream_flush": [vp, vp],
        "gd_get_records_async": [vp, vp, vp, C.c_int],
        "gd_records_wait": [vp, ip],
        "gd_get_etotal": [vp, fp, C.c_int, C.c_int],
        "gd_get_replicas": [vp, vp, C.c_int, C.c_int],
        "gd_get_state": [vp, vp, C.c_int, C.c_int],
        "gd_set_state": [vp, vp, C.c_int, C.c_int],
        "gd_get_device_error": [vp, ip],
        "gd_eval_energy": [vp, C.c_int, C.c_int, C.c_int, fp, C.c_int, vp],
        "gd_eval_energy_xyz": [vp, C.c_int, C.c_int, C.c_int, fp, fp, C.c_int, vp],
        "gd_place_ligand": [vp, C.c_int, C.c_int, fp, C.c_int, fp],
        "gd_trace_enable": [vp, C.c_int],
        "gd_trace_get": [vp, fp, ip, ip],
        "gd_get_stream": [vp, C.POINTER(vp)],
        "gd_set_rng_stream": [vp, C.c_int, C.c_int],
        "gd_set_concurrency": [vp, C.c_int, C.c_int],
        "gd_get_replicas_per_cta": [vp, C.c_int, ip],
        "gd_set_wait_timeout": [vp, C.c_longlong],
        "gd_sur_create": [vp, C.POINTER(abi.SurParams)],
        "gd_sur_collect": [vp, C.c_int, C.c_int, C.c_int],
        "gd_sur_train": [vp, C.c_int, fp],
        "gd_da_run": [vp, C.c_int, C.c_int, C.c_int],
        "gd_sur_get_stats": [vp, C.POINTER(abi.SurStats)],
        "gd_sur_set_active": [vp, C.c_int, C.c_int],
        "gd_sur_predict": [vp, C.c_int, C.c_int, C.c_int, fp, C.c_int, fp],
        "gd_sur_info": [vp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                        C.POINTER(C.c_longlong)],
        "gd_da_trace_enable": [vp, C.c_int, C.c_int],
        "gd_sur_split": [vp, ip],
        "gd_da_trace_get": [vp, fp, fp, ip],
        "gd_mlp_create": [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(vp)],
        "gd_mlp_destroy": [vp],
        "gd_mlp_num_params": [vp, C.POINTER(C.c_longlong)],
        "gd_mlp_get_params": [vp, fp, C.c_longlong],
        "gd_mlp_set_params": [vp, fp, C.c_longlong],
        "gd_mlp_forward": [vp, fp, ip, C.c_int, fp],
        "gd_mlp_backward": [vp, fp, ip, fp, C.c_int, fp, fp],
        "gd_mlp_adam": [vp, C.c_float],
        "gd_kmeans": [C.c_int, fp, C.c_int, C.c_int, ip, C.c_int, ip, C.c_uint64, C.c_float,
                      C.c_int, ip, ip, ip, ip],
        "gd_kmeans_permutation": [C.c_uint64, C.c_int, C.c_int, ip],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.gd_sur_default_params.argtypes = [C.POINTER(abi.SurParams)]
    L.gd_sur_default_params.restype = None
    L.gd_last_error_string.restype = C.c_char_p
    L.gd_version.restype = C.c_char_p
    _lib = L
    return L


def check(rc: int):
    if rc != abi.GD_OK:
        raise GDError(rc, lib().gd_last_error_string().decode())


def fold_enepara(raw: abi.EneParaRaw) -> abi.EnePara:
    """OptimizeEnepara (src/util.C:717-760) through the library."""
    out = abi.EnePara()
    check(lib().gd_fold_enepara(C.byref(raw), C.byref(out)))
    return out


def set_temperature(n: int, floor_t: float, ceil_t: float) -> np.ndarray:
    """SetTemperature (src/util.C:797-840)."""
    t = (abi.Temp * n)()
    check(lib().gd_set_temperature(n, floor_t, ceil_t, t))
    return np.frombuffer(bytes(t), dtype=abi.TEMP_DTYPE).copy()


def release_memory(device: int = 0):
    """gd_release_memory: gives the device memory that destroyed contexts left in the
    library's pool back to the driver."""
    check(lib().gd_release_memory(device))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Engine:
    """One B200 context: a batch of complexes, their replicas and records."""

    def __init__(self, ff: abi.EnePara, complexes: Sequence[abi.ComplexArrays],
                 params: abi.McParams, device: int = 0):
        self.complexes = list(complexes)
        self.params = params
        self.ff = ff
        descs = (abi.ComplexDesc * len(self.complexes))(*[c.desc() for c in self.complexes])
        h = C.c_void_p()
        check(lib().gd_create(C.byref(ff), descs, len(self.complexes), C.byref(params), device,
                              C.byref(h)))
        self.h = h
        n = C.c_int()
        check(lib().gd_num_replicas(self.h, C.byref(n)))
        self.n_rep = n.value
        self.offsets = []
        for k in range(len(self.complexes)):
            o = C.c_int()
            check(lib().gd_replica_offset(self.h, k, C.byref(o)))
            self.offsets.append(o.value)
        self.cap = params.steps_per_dump + 1
        self._stream_buf = None
        self._async = None

    def close(self):
        if getattr(self, "h", None):
            lib().gd_destroy(self.h)  # waits for a background download first
            self.h = None
        self._stream_buf = None
        self._async = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- reference-shaped operations ----
    def mc_init(self):
        check(lib().gd_mc_init(self.h))

    def reset_records(self, r0=0, r1=None):
        check(lib().gd_reset_records(self.h, r0, self.n_rep - 1 if r1 is None else r1))

    def mc_run(self, s1: int, s2: int, r0=0, r1=None):
        check(lib().gd_mc_run(self.h, r0, self.n_rep - 1 if r1 is None else r1, s1, s2))

    def exchange(self, mode_t: int, mode_l: int = 4):
        check(lib().gd_exchange(self.h, mode_l, mode_t))

    def run_fused(self, s1: int, n_steps: int, exchange: bool = True):
        check(lib().gd_mc_run_fused(self.h, s1, n_steps, 1 if exchange else 0))

    def sync(self):
        check(lib().gd_sync(self.h))

    def set_tile(self, replicas_per_cta: int, chunk_points: int, unroll: int = 0,
                 split: int = 0, threads: int = 0, replicas_per_lane: int = 1,
                 complex_index: int = -1):
        """threads > 0: every complex gets as many replicas as fill a CTA of that size
        (replicas_per_cta > 0 caps them); replicas_per_lane 2: each thread of the plain launches
        holds the same atom of two replicas."""
        t = abi.Tile()
        t.replicas_per_cta, t.chunk_points, t.unroll = replicas_per_cta, chunk_points, unroll
        t.split, t.threads, t.replicas_per_lane = split, threads, replicas_per_lane
        check(lib().gd_set_tile(self.h, complex_index, C.byref(t)))

    def cuda_stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        check(lib().gd_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_concurrency(self, plain_chains: int, da_chains: int = 3):
        check(lib().gd_set_concurrency(self.h, plain_chains, da_chains))

    def set_rng_stream(self, complex_index: int, stream: int):
        check(lib().gd_set_rng_stream(self.h, complex_index, stream))

    def set_wait_timeout(self, ns: int):
        check(lib().gd_set_wait_timeout(self.h, ns))

    def replicas_per_cta(self, complex_index=0) -> int:
        n = C.c_int()
        check(lib().gd_get_replicas_per_cta(self.h, complex_index, C.byref(n)))
        return n.value

    def tile(self, complex_index=0):
        """The tile as set: (replicas_per_cta, chunk_points, unroll, split, threads,
        replicas_per_lane); in fill mode (threads > 0) replicas_per_cta is the cap (0: none)."""
        t = abi.Tile()
        check(lib().gd_get_tile(self.h, complex_index, C.byref(t)))
        return (t.replicas_per_cta, t.chunk_points, t.unroll, t.split, t.threads,
                t.replicas_per_lane)

    # ---- results ----
    def records(self, r0=0, r1=None, out=None):
        """(steps [n, m], next_ptr [n]): the filled records of each replica, m = the largest
        count (only those rows cross the bus). out: a flat RECORD_DTYPE array of at least
        n * m rows to reuse from one dump window to the next, as the reference reuses its host
        LigRecord array; steps is then a view of it."""
        r1 = self.n_rep - 1 if r1 is None else r1
        n = r1 - r0 + 1
        nxt = np.zeros(n, np.int32)
        check(lib().gd_get_record_counts(self.h, _p(nxt), r0, r1))
        m = int(min(self.cap, max(1, nxt.max(initial=0))))
        if out is None:
            steps = np.empty((n, m), abi.RECORD_DTYPE)
        else:
            if out.dtype != abi.RECORD_DTYPE or not out.flags.c_contiguous or out.size < n * m:
                raise ValueError("out must be a contiguous RECORD_DTYPE array of >= %d rows"
                                 % (n * m))
            steps = out.reshape(-1)[:n * m].reshape(n, m)
        check(lib().gd_get_records_raw(self.h, _p(steps), _p(nxt), r0, r1, m))
        return steps, nxt

    def records_async(self, out: np.ndarray, nxt: np.ndarray, cap=None):
        """gd_get_records_async: the current window's records copied into out (a flat
        RECORD_DTYPE array of at least n_rep * cap rows) and nxt (n_rep int32) in the
        background; records_wait() completes it. Both arrays must stay alive and untouched
        until then."""
        cap = self.cap if cap is None else cap
        if out.dtype != abi.RECORD_DTYPE or not out.flags.c_contiguous or \
                out.size < self.n_rep * cap:
            raise ValueError("out must be a contiguous RECORD_DTYPE array of >= %d rows"
                             % (self.n_rep * cap))
        if nxt.dtype != np.int32 or not nxt.flags.c_contiguous or nxt.size < self.n_rep:
            raise ValueError("nxt must be a contiguous int32 array of >= %d values" % self.n_rep)
        check(lib().gd_get_records_async(self.h, _p(out), _p(nxt), cap))
        self._async = (out, nxt)

    def records_wait(self):
        """(steps [n_rep, m], next_ptr [n_rep]) of the last records_async, once copied."""
        rows = C.c_int()
        check(lib().gd_records_wait(self.h, C.byref(rows)))
        out, nxt = self._async
        m = max(1, rows.value)
        return out.reshape(-1)[:self.n_rep * m].reshape(self.n_rep, m), nxt[:self.n_rep]

    def stream_records(self, cap: int) -> np.ndarray:
        """Starts gd_records_stream into a new host array [n_rep][cap] (RECORD_DTYPE): the
        records are copied while the run proceeds; stream_flush() completes and returns it."""
        buf = np.empty((self.n_rep, cap), abi.RECORD_DTYPE)
        check(lib().gd_records_stream(self.h, _p(buf), cap))
        self._stream_buf = buf
        return buf

    def stream_flush(self):
        """(steps [n_rep][cap], next_ptr [n_rep]) mirroring the device records now."""
        nxt = np.empty(self.n_rep, np.int32)
        check(lib().gd_records_stream_flush(self.h, _p(nxt)))
        return self._stream_buf, nxt

    def stream_stop(self):
        check(lib().gd_records_stream(self.h, None, 0))
        self._stream_buf = None

    def lig_records(self, r0=0, r1=None) -> bytes:
        """LigRecord array bytes (reference layout, src/dock.h:377-381)."""
        r1 = self.n_rep - 1 if r1 is None else r1
        buf = (abi.LigRecord * (r1 - r0 + 1))()
        check(lib().gd_get_records(self.h, buf, r0, r1))
        return bytes(buf)

    def etotal(self, r0=0, r1=None):
        r1 = self.n_rep - 1 if r1 is None else r1
        out = np.zeros(r1 - r0 + 1, np.float32)
        check(lib().gd_get_etotal(self.h, abi.fptr(out), r0, r1))
        return out

    def replicas(self, r0=0, r1=None):
        r1 = self.n_rep - 1 if r1 is None else r1
        out = np.zeros(r1 - r0 + 1, abi.REPLICA_DTYPE)
        check(lib().gd_get_replicas(self.h, _p(out), r0, r1))
        return out

    def state(self, r0=0, r1=None):
        r1 = self.n_rep - 1 if r1 is None else r1
        out = np.zeros(r1 - r0 + 1, abi.STATE_DTYPE)
        check(lib().gd_get_state(self.h, _p(out), r0, r1))
        return out

    def set_state(self, st: np.ndarray, r0=0):
        st = np.ascontiguousarray(st, abi.STATE_DTYPE)
        check(lib().gd_set_state(self.h, _p(st), r0, r0 + st.shape[0] - 1))

    def device_error(self) -> int:
        e = C.c_int()
        check(lib().gd_get_device_error(self.h, C.byref(e)))
        return e.value

    def eval_energy(self, complex_index: int, prt_conf: int, lig_conf: int,
                    movematrix: np.ndarray) -> np.ndarray:
        mm = np.ascontiguousarray(movematrix, np.float32).reshape(-1, 6)
        out = np.zeros(mm.shape[0], abi.ENERGY_DTYPE)
        check(lib().gd_eval_energy(self.h, complex_index, prt_conf, lig_conf, abi.fptr(mm),
                                   mm.shape[0], _p(out)))
        return out

    def eval_energy_xyz(self, complex_index: int, prt_conf: int, lig_conf: int,
                        xyz: np.ndarray, center: np.ndarray) -> np.ndarray:
        """Energies of given placed coordinates: xyz [n_poses, lna, 3] and the ligand centres
        [n_poses, 3], lab frame (CalcEnergy_d on Ligand.coord_new)."""
        n = int(np.asarray(center).size // 3)
        x = np.ascontiguousarray(xyz, np.float32).reshape(n, -1, 3)
        c = np.ascontiguousarray(center, np.float32).reshape(n, 3)
        out = np.zeros(n, abi.ENERGY_DTYPE)
        check(lib().gd_eval_energy_xyz(self.h, complex_index, prt_conf, lig_conf, abi.fptr(x),
                                       abi.fptr(c), n, _p(out)))
        return out

    def place_ligand(self, complex_index: int, lig_conf: int,
                     movematrix: np.ndarray) -> np.ndarray:
        """Placed ligand atoms of each pose, [n_poses, lna, 3] (PlaceLigand, src/util.C:457)."""
        mm = np.ascontiguousarray(movematrix, np.float32).reshape(-1, 6)
        out = np.zeros((mm.shape[0], self.complexes[complex_index].lna, 3), np.float32)
        check(lib().gd_place_ligand(self.h, complex_index, lig_conf, abi.fptr(mm), mm.shape[0],
                                    abi.fptr(out)))
        return out

    def trace_enable(self, max_steps: int):
        check(lib().gd_trace_enable(self.h, max_steps))
        self._trace_cap = max_steps

    def trace(self):
        e = np.zeros((self.n_rep, self._trace_cap), np.float32)
        a = np.zeros((self.n_rep, self._trace_cap), np.int32)
        n = C.c_int()
        check(lib().gd_trace_get(self.h, abi.fptr(e), a.ctypes.data_as(C.POINTER(C.c_int)),
                                 C.byref(n)))
        return e, a

    # ---- the reference's whole docking loop ----
    def run(self, min_records: int, exchange: bool = True, max_dumps: int = 1000) \
            -> Dict[int, List[np.void]]:
        """Run (src/run.cu) + kernel_cuda_lancher_siglegpu.cu: dumps of steps_per_dump steps
        until at least `min_records` accepted steps are gathered; returns the per-replica
        lists of accepted steps (map<int, vector<LigRecordSingleStep>>)."""
        spd, spe = self.params.steps_per_dump, self.params.steps_per_exchange
        out: Dict[int, List[np.void]] = {r: [] for r in range(self.n_rep)}
        self.reset_records()
        self.mc_init()
        s1, total = 0, 0
        for _ in range(max_dumps):
            if total >= min_records:
                break
            if s1 != 0:
                self.reset_records()
            for s2 in range(0, spd, spe):
                self.mc_run(s1, s2)
                if exchange:
                    self.exchange(int(not ((s2 // spe) % 2)))
            steps, nxt = self.records()
            for r in range(self.n_rep):
                out[r].extend(steps[r, :nxt[r]])
                total += int(nxt[r])
            s1 += spd
        self.steps_total = s1
        return out


def sur_default_params(**kw) -> abi.SurParams:
    p = abi.SurParams()
    lib().gd_sur_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Surrogate:
    """The learned energy surrogate of an Engine and its delayed-acceptance steps
    (gd_sur_* / gd_da_* of the C ABI)."""

    def __init__(self, eng: Engine, params: abi.SurParams = None, **kw):
        self.eng = eng
        self.params = params if params is not None else sur_default_params(**kw)
        check(lib().gd_sur_create(eng.h, C.byref(self.params)))
        self._tr_cap = 0

    def collect(self, s1: int, n_steps: int, exchange: bool = True):
        check(lib().gd_sur_collect(self.eng.h, s1, n_steps, int(bool(exchange))))

    def train(self, iterations: int) -> np.ndarray:
        losses = np.zeros(max(1, iterations), np.float32)
        check(lib().gd_sur_train(self.eng.h, iterations, abi.fptr(losses)))
        return losses[:iterations]

    def run(self, s1: int, n_steps: int, exchange: bool = True):
        check(lib().gd_da_run(self.eng.h, s1, n_steps, int(bool(exchange))))

    def stats(self) -> List[Dict]:
        n = len(self.eng.complexes)
        arr = (abi.SurStats * n)()
        check(lib().gd_sur_get_stats(self.eng.h, arr))
        return [{f: getattr(s, f) for f, _ in abi.SurStats._fields_ if f != "pad"} for s in arr]

    def set_active(self, complex_index: int, active: bool):
        check(lib().gd_sur_set_active(self.eng.h, complex_index, int(bool(active))))

    def predict(self, complex_index: int, prt_conf: int, lig_conf: int,
                movematrix: np.ndarray) -> np.ndarray:
        mm = np.ascontiguousarray(movematrix, np.float32).reshape(-1, 6)
        out = np.zeros(mm.shape[0], np.float32)
        check(lib().gd_sur_predict(self.eng.h, complex_index, prt_conf, lig_conf, abi.fptr(mm),
                                   mm.shape[0], abi.fptr(out)))
        return out

    def info(self) -> Dict:
        mu, sg, n = C.c_float(), C.c_float(), C.c_longlong()
        check(lib().gd_sur_info(self.eng.h, C.byref(mu), C.byref(sg), C.byref(n)))
        return {"mu": mu.value, "sigma": sg.value, "n_samples": n.value}

    def split(self) -> int:
        v = C.c_int()
        check(lib().gd_sur_split(self.eng.h, C.byref(v)))
        return v.value

    def trace_enable(self, step0: int, max_steps: int):
        check(lib().gd_da_trace_enable(self.eng.h, step0, max_steps))
        self._tr_cap = max_steps

    def trace(self):
        shp = (self.eng.n_rep, self._tr_cap)
        s = np.zeros(shp, np.float32)
        e = np.zeros(shp, np.float32)
        f = np.zeros(shp, np.int32)
        check(lib().gd_da_trace_get(self.eng.h, abi.fptr(s), abi.fptr(e),
                                    f.ctypes.data_as(C.POINTER(C.c_int))))
        return s, e, f


class Mlp:
    """The surrogate network alone (gd_mlp_*): FP32 rows in, FP32 outputs/gradients out."""

    def __init__(self, hidden: int = 256, n_embedding: int = 0, seed: int = 1, device: int = 0):
        h = C.c_void_p()
        check(lib().gd_mlp_create(device, hidden, n_embedding, seed, C.byref(h)))
        self.h = h
        self.hidden, self.n_embedding = hidden, n_embedding
        n = C.c_longlong()
        check(lib().gd_mlp_num_params(self.h, C.byref(n)))
        self.n_params = n.value

    def close(self):
        if getattr(self, "h", None):
            lib().gd_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        th = np.zeros(self.n_params, np.float32)
        check(lib().gd_mlp_get_params(self.h, abi.fptr(th), self.n_params))
        return th

    def set_params(self, th: np.ndarray):
        th = np.ascontiguousarray(th, np.float32)
        check(lib().gd_mlp_set_params(self.h, abi.fptr(th), th.size))

    @staticmethod
    def _rows(x, conf):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 64)
        cp = None
        if conf is not None:
            conf = np.ascontiguousarray(conf, np.int32)
            cp = conf.ctypes.data_as(C.POINTER(C.c_int))
        return x, conf, cp

    def forward(self, x: np.ndarray, conf: np.ndarray = None) -> np.ndarray:
        x, conf, cp = self._rows(x, conf)
        y = np.zeros(x.shape[0], np.float32)
        check(lib().gd_mlp_forward(self.h, abi.fptr(x), cp, x.shape[0], abi.fptr(y)))
        return y

    def backward(self, x: np.ndarray, t: np.ndarray, conf: np.ndarray = None):
        x, conf, cp = self._rows(x, conf)
        t = np.ascontiguousarray(t, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(self.n_params, np.float32)
        check(lib().gd_mlp_backward(self.h, abi.fptr(x), cp, abi.fptr(t), x.shape[0],
                                    abi.fptr(loss), abi.fptr(g)))
        return float(loss[0]), g

    def adam(self, lr: float = 1e-3):
        check(lib().gd_mlp_adam(self.h, lr))
