"""Seeded synthetic pair sets with the shapes of the benchmark workloads.

No public dataset is used.  Bases and mutations come from the C generator
``libgasal_workloads.so`` (csrc/workload_gen.c): every pair draws from its own
xoshiro256** stream seeded by splitmix64 over (seed, pair index), so a pair's
sequences do not depend on the thread count or on the batch size, and a
10M-pair workload takes seconds on the host's cores.  Workload k's default
seed is ``20261203 + k``.  Batches are laid out as GASAL2's host batches are:
each sequence at an 8-byte aligned offset, N-padded.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Tuple

import numpy as np

from .capi import (Batch, Params, LOCAL, GLOBAL, SEMI_GLOBAL, KSW, TARGET, WITH_START, WITH_TB, TRUE)

SEED_BASE = 20261203
_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _gen() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libgasal_workloads.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C gasal_b200/csrc)")
        L = C.CDLL(path)
        L.gbw_lengths.argtypes = [C.c_int, C.c_uint64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_int]
        L.gbw_fill.argtypes = [C.c_int, C.c_uint64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_int]
        L.gbw_lengths.restype = L.gbw_fill.restype = C.c_int
        L.gbw_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def generate(w: int, n: int, seed: int, cuts=None, threads: int = 0, idx=None) -> List[Batch]:
    """Workload w, pairs [0, n) -- or, with idx, the pairs whose workload
    indexes idx[0..n) lists -- split into the batches [cuts[k], cuts[k+1]) of
    that list (one batch when cuts is None).  Each batch is laid out on its
    own."""
    L = _gen()
    if idx is not None:
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        n = len(idx)
    q_len = np.empty(n, np.uint32)
    t_len = np.empty(n, np.uint32)
    q_op = np.empty(n, np.uint8)
    h0 = np.empty(n, np.uint32)
    if L.gbw_lengths(w, seed, 0, _ptr(idx), n, _ptr(q_len), _ptr(t_len), _ptr(q_op), _ptr(h0), threads) != 0:
        raise MemoryError("workload generator failed")
    cuts = [0, n] if cuts is None else list(cuts)
    out = []
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        ql, tl = q_len[lo:hi], t_len[lo:hi]
        qp = (ql.astype(np.int64) + 7) & ~7
        tp = (tl.astype(np.int64) + 7) & ~7
        qo = np.zeros(hi - lo, np.int64)
        to = np.zeros(hi - lo, np.int64)
        if hi - lo > 1:
            np.cumsum(qp[:-1], out=qo[1:])
            np.cumsum(tp[:-1], out=to[1:])
        qb, tb = int(qp.sum()), int(tp.sum())
        if qb >= 2 ** 32 or tb >= 2 ** 32:
            raise ValueError("a batch exceeds 4 GiB of bases; split it")
        q = np.empty(qb, np.uint8)
        t = np.empty(tb, np.uint8)
        sub = None if idx is None else idx[lo:hi]
        if L.gbw_fill(w, seed, lo, _ptr(sub), hi - lo, _ptr(qo), _ptr(to), _ptr(q), _ptr(t), threads) != 0:
            raise MemoryError("workload generator failed")
        b = Batch(q, t, qo.astype(np.uint32), to.astype(np.uint32), np.ascontiguousarray(ql),
                  np.ascontiguousarray(tl))
        if w == 1:
            b.q_op = np.ascontiguousarray(q_op[lo:hi])
            b.t_op = np.zeros(hi - lo, np.uint8)
        if w in (3, 4):
            b.seed = np.ascontiguousarray(h0[lo:hi])
        out.append(b)
    return out


def pair_cells(w: int, n: int, seed: int, threads: int = 0) -> np.ndarray:
    """qlen * tlen of every pair of workload w (the generator's first pass
    only: no bases are written)."""
    L = _gen()
    q_len = np.empty(n, np.uint32)
    t_len = np.empty(n, np.uint32)
    if L.gbw_lengths(w, seed, 0, None, n, _ptr(q_len), _ptr(t_len), None, None, threads) != 0:
        raise MemoryError("workload generator failed")
    return q_len.astype(np.int64) * t_len


def _cuts(n: int, shares) -> list:
    return [int(x) for x in np.round(np.cumsum((0.0,) + tuple(shares)) * n).astype(np.int64)]


def workload0(n=20000, seed=SEED_BASE + 0) -> Batch:
    """Query U[100,150] with 0.1% N; target = 0-20 random flank bases each
    side + query, then 2% substitutions and 0.5% indels (1-3 bp)."""
    return generate(0, n, seed)[0]


WORKLOAD1_PARAMS = [
    Params(algo=LOCAL, start_pos=WITH_START, second_best=TRUE, reverse_complement=1),
    Params(algo=GLOBAL, start_pos=WITH_START, reverse_complement=1),
    Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, reverse_complement=1),
]


def workload1(n=1_000_000, seed=SEED_BASE + 1) -> List[Tuple[Params, Batch]]:
    """150 bp queries, 150-300 bp targets (3% subs, 1% indels), half of the
    queries REVERSE_COMPLEMENT; thirds LOCAL (second best) / GLOBAL /
    SEMI_GLOBAL (head = tail = TARGET), all WITH_START.  One (Params, Batch)
    per launch."""
    parts = generate(1, n, seed, _cuts(n, (1 / 3, 1 / 3, 1 / 3)))
    return [(p, b) for p, b in zip(WORKLOAD1_PARAMS, parts) if b.n > 0]


def workload2(n=2_000_000, seed=SEED_BASE + 2) -> Batch:
    """Query log-uniform 50-1000; target = query with per-pair 1-8% subs and
    0.5-3% indels of length 1-10 (GLOBAL, WITH_TB)."""
    return generate(2, n, seed)[0]


def workload3(n=4_000_000, seed=SEED_BASE + 3) -> Batch:
    """ksw extension: query U[250,2000], indel rate per pair from
    {0.5,2,5,10}% (1-3 bp) plus 1-5% subs, seed score h0 U[20,60]."""
    return generate(3, n, seed)[0]


WORKLOAD4_PARAMS = [
    Params(algo=LOCAL, start_pos=WITH_START),
    Params(algo=LOCAL, start_pos=WITH_TB),
    Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET),
    Params(algo=KSW, zdrop=100),
]
WORKLOAD4_SHARES = (0.30, 0.20, 0.25, 0.25)


def workload4(n=10_000_000, seed=SEED_BASE + 4) -> List[Tuple[Params, Batch]]:
    """Mixed production batch: query lengths log-normal (median 250, sigma 0.8,
    clipped to [50, 5000]); 60% short-read-like pairs (1-2% subs, 0.2% indels),
    30% long-read-like (5-12% errors, 75% of them indels of 1-5 bp), 10%
    unrelated random targets; split into four launches -- LOCAL WITH_START
    30%, LOCAL WITH_TB 20%, SEMI_GLOBAL (TARGET, TARGET) WITH_START 25%, ksw
    (h0 U[20,60], z-drop 100) 25%."""
    parts = generate(4, n, seed, _cuts(n, WORKLOAD4_SHARES))
    return [(p, b) for p, b in zip(WORKLOAD4_PARAMS, parts) if b.n > 0]


def generator_threads() -> int:
    return int(_gen().gbw_threads())


def concat_parts(parts, shuffle_seed=None):
    """One batch holding every pair of [(Params, Batch)] parts, for the mixed
    dispatch (gb_align_dev_mixed): returns (kinds, batch, kind, index_in_part),
    kind[j] being the part pair j comes from.  Sequence bytes are laid out part after part; the pair
    entries (offsets, lengths, ops, seeds, kind) are in part order, or in a
    seeded random order when shuffle_seed is given -- GASAL2's offsets may
    point anywhere in the batch, so the pairs of different kinds interleave
    without moving bytes.  Seeds are 0 for parts without them."""
    kinds = [p for p, _ in parts]
    qb = np.cumsum([0] + [int(b.q.shape[0]) for _, b in parts])
    tb = np.cumsum([0] + [int(b.t.shape[0]) for _, b in parts])
    part_of = np.concatenate([np.full(b.n, k, dtype=np.uint8) for k, (_, b) in enumerate(parts)])
    index_in = np.concatenate([np.arange(b.n, dtype=np.int64) for _, b in parts])
    q_off = np.concatenate([b.q_off.astype(np.uint64) + qb[k] for k, (_, b) in enumerate(parts)])
    t_off = np.concatenate([b.t_off.astype(np.uint64) + tb[k] for k, (_, b) in enumerate(parts)])
    if q_off.size and (q_off.max() >= 2**32 or t_off.max() >= 2**32):
        raise ValueError("the combined batch exceeds 32-bit byte offsets")
    q_len = np.concatenate([b.q_len for _, b in parts])
    t_len = np.concatenate([b.t_len for _, b in parts])
    has_ops = any(b.q_op is not None for _, b in parts)
    q_op = np.concatenate([b.q_op if b.q_op is not None else np.zeros(b.n, np.uint8) for _, b in parts]) \
        if has_ops else None
    t_op = np.concatenate([b.t_op if b.t_op is not None else np.zeros(b.n, np.uint8) for _, b in parts]) \
        if has_ops else None
    seed = np.concatenate([b.seed if b.seed is not None else np.zeros(b.n, np.uint32) for _, b in parts])
    order = np.arange(part_of.shape[0])
    if shuffle_seed is not None:
        order = np.random.default_rng(shuffle_seed).permutation(part_of.shape[0])
    pick = lambda a: None if a is None else np.ascontiguousarray(a[order])
    batch = Batch(q=np.concatenate([b.q for _, b in parts]), t=np.concatenate([b.t for _, b in parts]),
                  q_off=pick(q_off).astype(np.uint32), t_off=pick(t_off).astype(np.uint32),
                  q_len=pick(q_len), t_len=pick(t_len), q_op=pick(q_op), t_op=pick(t_op), seed=pick(seed))
    return kinds, batch, pick(part_of), pick(index_in)
