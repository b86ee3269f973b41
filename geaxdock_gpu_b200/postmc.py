"""Post-Monte-Carlo clustering and the trajectory output of the reference's `dock` program.

post_mc (src/post_mc.C:40-101): every replica's records are clustered by k-means on their 9
energy terms into 50 clusters, the representatives of all replicas are pooled and clustered
into 500, and the 500 representatives, sorted by total energy, are the run's result, written
by printStates (src/util.C:1504-1545) as a space-separated table. The k-means runs on the
GPU, all replicas of the first stage in one batch (gd_kmeans, csrc/gd_kmeans.cu); the shuffle
that the reference draws without a seed is a seeded permutation here (first stage `seed`,
second stage `seed + 1`).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import abi
from .engine import check, lib

DIM = abi.MAXWEI - 1  # the clustered coordinates: energy terms 0..8


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def kmeans(objects: np.ndarray, seg_off: Sequence[int], k: Sequence[int], seed: int,
           threshold: float = 0.001, max_iter: int = 500, device: int = 0):
    """Batched k-means (gd_kmeans): returns (membership [n], medoid [clusters],
    size [clusters], passes [n_seg], cluster_base [n_seg])."""
    obj = np.ascontiguousarray(objects, dtype=np.float32).reshape(-1, DIM)
    off = _i32(seg_off)
    kk = _i32(k)
    n_seg = kk.shape[0]
    n = obj.shape[0]
    counts = np.minimum(kk, np.diff(off))
    base = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32)
    total = int(counts.sum())
    mem = np.empty(n, np.int32)
    med = np.empty(max(total, 1), np.int32)
    size = np.empty(max(total, 1), np.int32)
    passes = np.empty(n_seg, np.int32)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    check(lib().gd_kmeans(device, obj.ctypes.data_as(abi.FP), n, DIM, ip(off), n_seg, ip(kk),
                          seed, threshold, max_iter, ip(mem), ip(med), ip(size), ip(passes)))
    return mem, med[:total], size[:total], passes, base


def permutation(seed: int, segment: int, n: int) -> np.ndarray:
    out = np.empty(n, np.int32)
    check(lib().gd_kmeans_permutation(seed, segment, n,
                                      out.ctypes.data_as(C.POINTER(C.c_int))))
    return out


def _order(E: np.ndarray, seg_off, k, med, size):
    """Per segment: its clusters' representatives (empty clusters dropped), sorted by total
    energy (stable) when the segment was clustered, in record order when it was not; all
    segments in segment order. Returns (object indices into E, cluster sizes)."""
    off = np.asarray(seg_off, np.int64)
    kk = np.asarray(k, np.int64)
    n_s = np.diff(off)
    cnt = np.minimum(kk, n_s)
    seg = np.repeat(np.arange(cnt.shape[0]), cnt)
    ok = med >= 0
    m = med[ok].astype(np.int64)
    clustered = (n_s >= kk)[seg[ok]]
    energy = np.where(clustered, E[m, abi.MAXWEI - 1], np.float32(0.0))
    order = np.lexsort((np.flatnonzero(ok), energy, seg[ok]))  # segment, energy, cluster
    return m[order], np.asarray(size)[ok][order]


def post_mc_indices(E: np.ndarray, seg_off, seed: int = 0, k1: int = 50, k2: int = 500,
                    device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """post_mc on the energy rows E [n][10] of all records, segment s = the records of replica
    s: (indices into E of the representatives, sorted by total energy; cluster sizes)."""
    E = np.asarray(E, np.float32)
    off = np.asarray(seg_off, np.int32)
    k = [k1] * (off.shape[0] - 1)
    _, med, size, _, _ = kmeans(E[:, :DIM], off, k, seed, device=device)
    pool, _ = _order(E, off, k, med, size)
    off2 = np.asarray([0, pool.shape[0]], np.int32)
    Ep = E[pool]
    _, med2, size2, _, _ = kmeans(Ep[:, :DIM], off2, [k2], seed + 1, device=device)
    fin, sz = _order(Ep, off2, [k2], med2, size2)
    return pool[fin], sz


def post_mc(replica_records: Dict[int, np.ndarray] | List[np.ndarray], seed: int = 0,
            k1: int = 50, k2: int = 500, device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """The run's representative records (RECORD_DTYPE, sorted by total energy) and their
    cluster sizes, from each replica's records (multi_reps_records)."""
    recs = [replica_records[i] for i in range(len(replica_records))]
    if not recs:
        return np.zeros(0, abi.RECORD_DTYPE), np.zeros(0, np.int32)
    off = np.concatenate([[0], np.cumsum([r.shape[0] for r in recs])]).astype(np.int64)
    E = np.concatenate([r["energy"]["e"] for r in recs])
    idx, sz = post_mc_indices(E, off, seed, k1, k2, device)
    rep = np.searchsorted(off, idx, side="right") - 1
    out = np.array([recs[r][i - off[r]] for r, i in zip(rep, idx)], dtype=abi.RECORD_DTYPE)
    return out.reshape(-1), sz


def post_mc_steps(steps: np.ndarray, next_ptr: np.ndarray, seed: int = 0, k1: int = 50,
                  k2: int = 500, device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """post_mc on Engine.records() output directly (steps [n_rep][m], the first next_ptr[r]
    of row r filled), without building per-replica arrays."""
    n, m = steps.shape
    nxt = np.asarray(next_ptr, np.int64)
    fi = np.flatnonzero((np.arange(m)[None, :] < nxt[:, None]).ravel())
    flat = steps.reshape(-1)
    E = flat["energy"]["e"][fi]
    off = np.concatenate([[0], np.cumsum(nxt)])
    idx, sz = post_mc_indices(E, off, seed, k1, k2, device)
    return flat[fi[idx]], sz


def write_states(records: np.ndarray, path: str):
    """printStates (src/util.C:1504-1545): header, then per record `lig prt cms rmsd mv1..mv6
    vdw ele pmf psp hdb hpc kde lhm edst ener` in fixed notation with 4 decimals."""
    with open(path, "w") as f:
        f.write("lig prt cms rmsd mv1 mv2 mv3 mv4 mv5 mv6 "
                "vdw ele pmf psp hdb hpc kde lhm edst ener\n")
        for s in records:
            e = s["energy"]
            vals = [float(e["cms"]), float(e["rmsd"])] + [float(v) for v in s["movematrix"]] + \
                [float(v) for v in e["e"]]
            f.write("%d %d " % (int(s["replica"]["idx_lig"]), int(s["replica"]["idx_prt"])) +
                    " ".join("%.4f" % v for v in vals[:-1]) + " %.4f\n" % vals[-1])
