"""Tile autotuner with a JSON cache.

The fused kernel's tile is (replicas per CTA, protein points per shared-memory chunk, point
pairs in flight per lane, protein split, CTA lanes in fill mode, replicas per thread).
`tune(engine)` times a candidate grid with gd_autotune (Monte Carlo steps of every replica,
each candidate from the same copy of the chain state, which is put back afterwards), re-times
the fastest few with more launches, applies the fastest and stores it in a JSON cache keyed by
(ligand atoms, protein points, replicas, device name); later engines with the same key reuse
the entry without timing.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Dict, List, Optional, Sequence, Tuple

from . import abi
from .engine import Engine, check, lib

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tile_cache.json")


def candidates(lna: int, ragged: bool = False,
               pack: bool = None) -> List[Tuple[int, int, int, int, int, int]]:
    """(replicas_per_cta, chunk_points, unroll, split, threads, replicas_per_lane) candidates:
    one replica count for every complex that fills 128..256 lanes for the largest ligand, and
    for a ragged batch also CTAs of 128..256 lanes that every complex fills with as many
    replicas as fit; with `pack` (default: uniform batches, whose timing is cheap) each also
    with two replicas per thread. Candidates that a batch cannot take are skipped by the
    timing."""
    ks = sorted({max(1, t // lna) for t in (128, 160, 192, 224, 256)} | {1})
    ks = [k for k in ks if k * lna <= 256]
    packs = (1, 2) if (not ragged if pack is None else pack) else (1,)
    out = []
    for p in packs:
        for chunk in (256, 512, 1024):
            # four point pairs in flight only with one replica per lane (no packed variant)
            for unroll in ((1, 2, 4) if p == 1 else (1, 2)):
                for k in ks:
                    out.append((k, chunk, unroll, 1, 0, p))
                if ragged:
                    for threads in (128, 192, 256):
                        if threads >= lna:
                            out.append((0, chunk, unroll, 1, threads, p))
    return out


def _key(eng: Engine, device_name: str) -> str:
    cx = eng.complexes
    lna = max(c.lna for c in cx)
    pnp = max(c.pnp for c in cx)
    return "lna%d_pnp%d_rep%d_%s" % (lna, pnp, eng.n_rep, device_name.replace(" ", "_"))


def _device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda%d" % device


def time_candidates(eng: Engine, cands: Sequence[Tuple[int, ...]], repeats: int = 2):
    arr = (abi.Tile * len(cands))()
    for i, c in enumerate(cands):
        k, ch, u = c[:3]
        arr[i].replicas_per_cta, arr[i].chunk_points, arr[i].unroll = k, ch, u
        arr[i].split = c[3] if len(c) > 3 else 1
        arr[i].threads = c[4] if len(c) > 4 else 0
        arr[i].replicas_per_lane = c[5] if len(c) > 5 else 1
    best = abi.Tile()
    ms = (C.c_float * len(cands))()
    fn = lib().gd_autotune
    fn.argtypes = [C.c_void_p, C.POINTER(abi.Tile), C.c_int, C.c_int, C.POINTER(abi.Tile),
                   C.POINTER(C.c_float)]
    fn.restype = C.c_int
    check(fn(eng.h, arr, len(cands), repeats, C.byref(best), ms))
    return (best.replicas_per_cta, best.chunk_points, best.unroll, best.split, best.threads,
            best.replicas_per_lane), list(ms)


def tune(eng: Engine, cache_path: Optional[str] = DEFAULT_CACHE, device: int = 0,
         repeats: int = 2, force: bool = False, finalists: int = 4) -> Dict:
    name = _device_name(device)
    key = _key(eng, name)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if key in cache and not force and len(cache[key]["tile"]) == 6:
        eng.set_tile(*cache[key]["tile"])
        return dict(cache[key], cached=True)
    lna = max(c.lna for c in eng.complexes)
    ragged = len({c.lna for c in eng.complexes}) > 1
    cands = candidates(lna, ragged)
    best, ms = time_candidates(eng, cands, repeats)
    # second round: the fastest few again with more launches each, since neighbours in the
    # first round's ranking are often within its noise
    ranked = sorted((m, i) for i, m in enumerate(ms) if m > 0)
    final = [cands[i] for _, i in ranked[:finalists]]
    final_ms = []
    if len(final) > 1:
        best, final_ms = time_candidates(eng, final, 3 * repeats)
    entry = {"tile": list(best),
             "ms": {",".join(str(v) for v in c): round(m, 4) for c, m in zip(cands, ms)},
             "final_ms": {",".join(str(v) for v in c): round(m, 4)
                          for c, m in zip(final, final_ms)}}
    cache[key] = entry
    if cache_path:
        try:
            with open(cache_path, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return dict(entry, cached=False)
