"""CPU oracle of the post-Monte-Carlo clustering (test infrastructure only).

Restates seq_kmeans (src/seq_kmeans.c: first k objects seed the centres; Lloyd passes with
the squared Euclidean distance summed dimension by dimension in float, ties to the lower
index; centres = float member sums in object order / member count; repeat while the changed
fraction > threshold and `loop++ < 500`) and clusterByKmeans (src/util.C:1801-1880: fewer
records than clusters -> every record its own cluster; records shuffled first; a cluster's
representative is its last member, the reference's medoid loop never updating its running
distance; representatives sorted by total energy), on the shuffle the library uses (a seeded
Feistel permutation, restated here from its definition in csrc/gd_kmeans.cu) instead of the
reference's unseeded random_shuffle. Float32 numpy arithmetic throughout, no fused
multiply-add, so results are comparable bit for bit with the GPU.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

F32 = np.float32
M32 = 0xFFFFFFFF


def lowbias32(x: int) -> int:
    x &= M32
    x ^= x >> 16
    x = (x * 0x7FEB352D) & M32
    x ^= x >> 15
    x = (x * 0x846CA68B) & M32
    x ^= x >> 16
    return x


def permutation(seed: int, seg: int, n: int) -> np.ndarray:
    """perm[i] = the object at shuffled position i of segment `seg` of n objects."""
    if n <= 1:
        return np.zeros(n, np.int64)
    b = 0
    while (1 << b) < n:
        b += 1
    if b & 1:
        b += 1
    h = b // 2
    mask = (1 << h) - 1
    keys = [lowbias32((seed & M32) ^ lowbias32(((seed >> 32) + 0x9E3779B9 * (seg * 4 + r + 1))
                                                & M32)) for r in range(4)]
    out = np.empty(n, np.int64)
    for i in range(n):
        x = i
        while True:
            l, r = x >> h, x & mask
            for k in keys:
                f = lowbias32(r ^ k) & mask
                l, r = r, l ^ f
            x = (l << h) | r
            if x < n:
                break
        out[i] = x
    return out


def seq_kmeans(objects: np.ndarray, k: int, threshold: float = 0.001, max_iter: int = 500):
    """(membership, centres, passes) for objects [n][d] in their given order."""
    obj = np.asarray(objects, F32)
    n, d = obj.shape
    cen = obj[:k].copy()
    mem = np.full(n, -1, np.int64)
    thr = F32(threshold)
    loop = 0
    while True:
        # distances [n][k]: float sum over dimensions in order, no contraction
        dist = np.zeros((n, k), F32)
        for j in range(d):
            t = (obj[:, j:j + 1] - cen[None, :, j]).astype(F32)
            dist = (dist + (t * t).astype(F32)).astype(F32)
        idx = np.argmin(dist, axis=1)  # first minimum: ties to the lower cluster index
        delta = F32(np.count_nonzero(idx != mem))
        mem = idx
        for c in range(k):
            members = np.flatnonzero(mem == c)
            if members.size:
                s = np.zeros(d, F32)
                for p in members:  # object order
                    s = (s + obj[p]).astype(F32)
                cen[c] = (s / F32(members.size)).astype(F32)
        delta = F32(delta / F32(n))
        if not (delta > thr):
            break
        old = loop
        loop += 1
        if not (old < max_iter):
            break
    return mem, cen, loop + 1


def cluster_by_kmeans(objects: np.ndarray, k: int, seed: int, seg: int,
                      threshold: float = 0.001, max_iter: int = 500):
    """(membership [n] in original order, representative object per cluster (-1 if empty),
    cluster sizes, passes) of one segment."""
    obj = np.asarray(objects, F32)
    n = obj.shape[0]
    if n < k:
        return np.arange(n), np.arange(n), np.ones(n, np.int64), 0
    perm = permutation(seed, seg, n)
    mem_sh, _, passes = seq_kmeans(obj[perm], k, threshold, max_iter)
    membership = np.empty(n, np.int64)
    membership[perm] = mem_sh
    rep = np.full(k, -1, np.int64)
    size = np.zeros(k, np.int64)
    for p in range(n):
        c = mem_sh[p]
        rep[c] = perm[p]
        size[c] += 1
    return membership, rep, size, passes


def energy_order(total_energy: np.ndarray) -> np.ndarray:
    """Stable ascending order by total energy (medoidEnergyLessThan, src/util.C:1582)."""
    return np.argsort(np.asarray(total_energy, F32), kind="stable")


def post_mc(records: List[np.ndarray], seed: int, k1: int = 50, k2: int = 500
            ) -> Tuple[np.ndarray, np.ndarray]:
    """post_mc (src/post_mc.C:40-101) on per-replica record arrays (RECORD_DTYPE): k1 clusters
    per replica (segment i shuffled with `seed`), their representatives pooled in replica
    order, k2 clusters over the pool (shuffled with seed + 1); a clustered segment's
    representatives are sorted by energy, an unclustered one (fewer records than clusters)
    keeps its records in order, as clusterByKmeans returns them. Returns (representative
    records, cluster sizes)."""
    def one(rec, k, sd, seg):
        _, rep, size, _ = cluster_by_kmeans(rec["energy"]["e"][:, :9], k, sd, seg)
        ok = rep >= 0
        out, sz = rec[rep[ok]], size[ok]
        if rec.shape[0] >= k:
            o = energy_order(out["energy"]["e"][:, 9])
            out, sz = out[o], sz[o]
        return out, sz
    pool = [one(rec, k1, seed, i)[0] for i, rec in enumerate(records)]
    pool = np.concatenate(pool) if pool else np.zeros(0, records[0].dtype)
    return one(pool, k2, seed + 1, 0)
