"""ctypes mirror of include/geauxdock_b200.h (the C ABI of the B200 docking engine).

The record and state structures have the reference's byte layouts:
Energy (src/dock.h:108-128), Replica (src/dock.h:302-309), LigRecordSingleStep
(src/dock.h:361-367), LigRecord (src/dock.h:377-381), Temp (src/dock.h:288-293),
EnePara (src/dock_soa.h:99-137), EnePara0 (src/dock.h:256-272).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

MAXLIG = 100
MAXPRO = 10000
MAXTP1 = 30
MAXTP2 = 24
MAXTP3 = 50
MAXTP4 = 20
MAXWEI = 10
MAXMCS = 256
MAXTMP = 40
MAXPOS = 1000
MAXKDE = 10000
STEPS_PER_DUMP = 2000
MCS_INVALID_COORD = 728492.0

GD_OK = 0
GD_ERR_INVALID = -1
GD_ERR_CUDA = -2
GD_ERR_NOMEM = -3
GD_ERR_CAPACITY = -4
GD_ERR_TIMEOUT = -5
GD_ERR_STATE = -6
GD_ERR_NODEVICE = -7
GD_ERR_RECORD_FULL = -8

MOVE_UNIFORM = 0
MOVE_GAUSSIAN = 1

F = C.c_float
I = C.c_int


class Energy(C.Structure):
    _fields_ = [("e", F * MAXWEI), ("cms", F), ("rmsd", F)]


class Replica(C.Structure):
    _fields_ = [("idx_rep", I), ("idx_prt", I), ("idx_tmp", I), ("idx_lig", I)]


class RecordStep(C.Structure):
    _fields_ = [("replica", Replica), ("energy", Energy), ("movematrix", F * 6), ("step", I)]


class LigRecord(C.Structure):
    _fields_ = [("step", RecordStep * (STEPS_PER_DUMP + 1)), ("next_ptr", I)]


class Temp(C.Structure):
    _fields_ = [("t", F), ("minus_beta", F), ("order", I)]


class EnePara(C.Structure):
    _fields_ = [
        ("p1a", (F * MAXTP1) * MAXTP2), ("p2a", (F * MAXTP1) * MAXTP2),
        ("lj0", F), ("lj1", F), ("el0", F), ("el1", F), ("ele", F * MAXTP3),
        ("a1", F), ("b1", F),
        ("pmf0", (F * MAXTP1) * MAXTP2), ("pmf1", (F * MAXTP1) * MAXTP2),
        ("hdb0", (F * MAXTP1) * MAXTP2), ("hdb1", (F * MAXTP1) * MAXTP2),
        ("hpp", F * MAXTP4), ("hpl0", F * MAXTP2), ("hpl1", F * MAXTP2), ("hpl2", F * MAXTP2),
        ("kde2", F), ("kde3", F),
        ("w", F * MAXWEI), ("a_para", F * MAXWEI), ("b_para", F * MAXWEI),
    ]


class EneParaRaw(C.Structure):
    _fields_ = [
        ("vdw", ((F * 2) * MAXTP2) * MAXTP1), ("ele", F * MAXTP3),
        ("pmf", ((F * 2) * MAXTP2) * MAXTP1), ("hpp", F * MAXTP4), ("hpl", (F * 2) * MAXTP2),
        ("hdb", ((F * 2) * MAXTP2) * MAXTP1), ("lj", F * 3), ("el", F * 2), ("kde", F),
        ("w", F * MAXWEI), ("a_para", F * MAXWEI), ("b_para", F * MAXWEI),
    ]


FP = C.POINTER(F)
IP = C.POINTER(I)


class ComplexDesc(C.Structure):
    _fields_ = [
        ("n_lig", I), ("n_prt", I), ("n_tmp", I), ("lna", I), ("pnp", I), ("pnk", I), ("pos", I),
        ("lig_x", FP), ("lig_y", FP), ("lig_z", FP), ("lig_center", FP),
        ("lig_t", IP), ("lig_c", FP), ("lig_n", IP),
        ("prt_x", FP), ("prt_y", FP), ("prt_z", FP), ("prt_t", IP), ("prt_c", IP),
        ("prt_ele", FP), ("prt_seq3r", IP), ("prt_hflag", IP), ("prt_hpp", FP),
        ("pocket_center", FP),
        ("psp", FP), ("psp_ld", I),
        ("kde_x", FP), ("kde_y", FP), ("kde_z", FP), ("kde_t", IP),
        ("mcs_x", FP), ("mcs_y", FP), ("mcs_z", FP), ("mcs_tcc", FP), ("mcs_ld", I),
        ("temp", C.POINTER(Temp)),
    ]


class McParams(C.Structure):
    _fields_ = [
        ("steps_per_exchange", I), ("steps_per_dump", I), ("move_scale", F * 6),
        ("move_kind", I), ("record", I), ("seed", C.c_uint64),
    ]


class Tile(C.Structure):
    _fields_ = [("replicas_per_cta", I), ("chunk_points", I), ("unroll", I), ("split", I),
                ("threads", I), ("replicas_per_lane", I)]


class ReplicaState(C.Structure):
    _fields_ = [
        ("movematrix_old", F * 6), ("energy_old", Energy), ("replica", Replica),
        ("n_accept", I), ("n_exchange", I),
    ]


class SurParams(C.Structure):
    _fields_ = [
        ("hidden", I), ("embedding", I), ("lr", F), ("batch", I), ("sample_cap", C.c_longlong),
        ("fallback_accept", F), ("fallback_window", C.c_longlong), ("seed", C.c_uint64),
        ("split", I), ("pad", I),
    ]


class SurStats(C.Structure):
    _fields_ = [
        ("proposed", C.c_longlong), ("passed", C.c_longlong), ("accepted", C.c_longlong),
        ("plain", C.c_longlong), ("plain_accepted", C.c_longlong), ("rmse", C.c_double),
        ("n_err", C.c_longlong), ("active", I), ("pad", I),
    ]


assert C.sizeof(Energy) == 48
assert C.sizeof(Replica) == 16
assert C.sizeof(RecordStep) == 92
assert C.sizeof(LigRecord) == 92 * (STEPS_PER_DUMP + 1) + 4
assert C.sizeof(Temp) == 12

ENERGY_DTYPE = np.dtype([("e", np.float32, (MAXWEI,)), ("cms", np.float32), ("rmsd", np.float32)])
REPLICA_DTYPE = np.dtype([("idx_rep", np.int32), ("idx_prt", np.int32), ("idx_tmp", np.int32),
                          ("idx_lig", np.int32)])
RECORD_DTYPE = np.dtype([("replica", REPLICA_DTYPE), ("energy", ENERGY_DTYPE),
                         ("movematrix", np.float32, (6,)), ("step", np.int32)])
TEMP_DTYPE = np.dtype([("t", np.float32), ("minus_beta", np.float32), ("order", np.int32)])
STATE_DTYPE = np.dtype([("movematrix_old", np.float32, (6,)), ("energy_old", ENERGY_DTYPE),
                        ("replica", REPLICA_DTYPE), ("n_accept", np.int32),
                        ("n_exchange", np.int32)])
assert RECORD_DTYPE.itemsize == 92 and STATE_DTYPE.itemsize == C.sizeof(ReplicaState)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def fptr(a: np.ndarray):
    return a.ctypes.data_as(FP)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(IP)


@dataclass
class ComplexArrays:
    """One docking complex as host arrays (the reference's `Run` inputs, src/run.h:8-19).

    Shapes: ligand arrays (n_lig, lna); protein arrays (n_prt, pnp); psp (24, psp_ld)
    indexed [ligand type][seq3r]; kde (pnk,); mcs (pos, mcs_ld) indexed by SDF atom
    number + 1; temp a TEMP_DTYPE array (n_tmp,).
    """

    lig_x: np.ndarray
    lig_y: np.ndarray
    lig_z: np.ndarray
    lig_center: np.ndarray
    lig_t: np.ndarray
    lig_c: np.ndarray
    lig_n: np.ndarray
    prt_x: np.ndarray
    prt_y: np.ndarray
    prt_z: np.ndarray
    prt_t: np.ndarray
    prt_c: np.ndarray
    prt_ele: np.ndarray
    prt_seq3r: np.ndarray
    prt_hflag: np.ndarray
    prt_hpp: np.ndarray
    pocket_center: np.ndarray
    psp: np.ndarray
    kde_x: np.ndarray
    kde_y: np.ndarray
    kde_z: np.ndarray
    kde_t: np.ndarray
    mcs_x: np.ndarray
    mcs_y: np.ndarray
    mcs_z: np.ndarray
    mcs_tcc: np.ndarray
    temp: np.ndarray
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        for name in ("lig_x", "lig_y", "lig_z", "lig_c", "prt_x", "prt_y", "prt_z", "prt_ele",
                     "prt_hpp", "psp", "kde_x", "kde_y", "kde_z", "mcs_x", "mcs_y", "mcs_z",
                     "mcs_tcc"):
            setattr(self, name, _f32(getattr(self, name)))
        for name in ("lig_t", "lig_n", "prt_t", "prt_c", "prt_seq3r", "prt_hflag", "kde_t"):
            setattr(self, name, _i32(getattr(self, name)))
        self.lig_center = _f32(self.lig_center).reshape(-1, 3)
        self.pocket_center = _f32(self.pocket_center).reshape(3)
        self.temp = np.ascontiguousarray(self.temp, dtype=TEMP_DTYPE)
        for name in ("lig_x", "lig_y", "lig_z", "lig_t", "lig_c", "lig_n"):
            assert getattr(self, name).ndim == 2, name
        for name in ("prt_x", "prt_y", "prt_z", "prt_t", "prt_c", "prt_ele", "prt_seq3r",
                     "prt_hflag", "prt_hpp"):
            assert getattr(self, name).ndim == 2, name
        assert self.psp.ndim == 2 and self.psp.shape[0] == MAXTP2
        assert self.mcs_x.ndim == 2

    @property
    def n_lig(self):
        return self.lig_x.shape[0]

    @property
    def lna(self):
        return self.lig_x.shape[1]

    @property
    def n_prt(self):
        return self.prt_x.shape[0]

    @property
    def pnp(self):
        return self.prt_x.shape[1]

    @property
    def pnk(self):
        return self.kde_x.shape[0]

    @property
    def pos(self):
        return self.mcs_x.shape[0]

    @property
    def n_tmp(self):
        return self.temp.shape[0]

    @property
    def n_rep(self):
        return self.n_prt * self.n_tmp * self.n_lig

    def desc(self) -> ComplexDesc:
        d = ComplexDesc()
        d.n_lig, d.n_prt, d.n_tmp = self.n_lig, self.n_prt, self.n_tmp
        d.lna, d.pnp, d.pnk, d.pos = self.lna, self.pnp, self.pnk, self.pos
        for name in ("lig_x", "lig_y", "lig_z", "lig_center", "lig_c", "prt_x", "prt_y", "prt_z",
                     "prt_ele", "prt_hpp", "pocket_center", "psp", "kde_x", "kde_y", "kde_z",
                     "mcs_x", "mcs_y", "mcs_z", "mcs_tcc"):
            setattr(d, name, fptr(getattr(self, name)))
        for name in ("lig_t", "lig_n", "prt_t", "prt_c", "prt_seq3r", "prt_hflag", "kde_t"):
            setattr(d, name, iptr(getattr(self, name)))
        d.psp_ld = self.psp.shape[1]
        d.mcs_ld = self.mcs_x.shape[1]
        d.temp = self.temp.ctypes.data_as(C.POINTER(Temp))
        return d

    def subset(self, n_lig=None, n_prt=None, n_tmp=None) -> "ComplexArrays":
        """A smaller complex: the first n_lig / n_prt conformers and n_tmp temperatures."""
        nl = self.n_lig if n_lig is None else n_lig
        npr = self.n_prt if n_prt is None else n_prt
        kw = {k: getattr(self, k) for k in self.__dataclass_fields__ if k != "_keep"}
        for k in ("lig_x", "lig_y", "lig_z", "lig_center", "lig_t", "lig_c", "lig_n"):
            kw[k] = kw[k][:nl]
        for k in ("prt_x", "prt_y", "prt_z", "prt_t", "prt_c", "prt_ele", "prt_seq3r",
                  "prt_hflag", "prt_hpp"):
            kw[k] = kw[k][:npr]
        if n_tmp is not None:
            kw["temp"] = kw["temp"][:n_tmp]
        return ComplexArrays(**kw)


def enepara_from_array(a: np.ndarray) -> EnePara:
    a = _f32(a)
    assert a.nbytes == C.sizeof(EnePara)
    ep = EnePara()
    C.memmove(C.addressof(ep), a.ctypes.data, a.nbytes)
    return ep


def enepara_raw_from_array(a: np.ndarray) -> EneParaRaw:
    a = _f32(a)
    assert a.nbytes == C.sizeof(EneParaRaw)
    ep = EneParaRaw()
    C.memmove(C.addressof(ep), a.ctypes.data, a.nbytes)
    return ep


def struct_to_array(s) -> np.ndarray:
    return np.frombuffer(bytes(s), dtype=np.float32).copy()


def mc_params(steps_per_exchange=10, steps_per_dump=STEPS_PER_DUMP, move_scale=(0.02, 0.02, 0.02,
              0.08, 0.08, 0.08), move_kind=MOVE_UNIFORM, record=1, seed=42) -> McParams:
    p = McParams()
    p.steps_per_exchange = steps_per_exchange
    p.steps_per_dump = steps_per_dump
    for i in range(6):
        p.move_scale[i] = move_scale[i]
    p.move_kind = move_kind
    p.record = record
    p.seed = seed
    return p
