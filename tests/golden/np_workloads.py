"""The numpy generator the committed golden fixtures' inputs were made with.

TEST INFRASTRUCTURE: make_golden.py (beside this file) imports it so that the
fixture recipe keeps reproducing the fixtures' inputs.  The package's own
workloads (gasal_b200/workloads.py) come from a C generator with per-pair
xoshiro256** streams; this module is numpy PCG64 with mutations vectorised over
the batch, seeded with ``20261203 + k`` for workload k.
"""
from __future__ import annotations

import numpy as np

from gasal_b200.capi import (Batch, Params, LOCAL, GLOBAL, SEMI_GLOBAL, KSW, TARGET, WITH_START,
                   WITHOUT_START, WITH_TB, TRUE, FALSE, REVERSE_COMPLEMENT, N_CODE)

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
SEED_BASE = 20261203


def _random_bases(rng, n):
    return ACGT[rng.integers(0, 4, size=n, dtype=np.uint8)]


def _stage_flat(flat: np.ndarray, lens: np.ndarray):
    """Lay out sequences (concatenated in ``flat``) at 8-byte aligned offsets,
    N-padded, as GASAL2's host batch does."""
    lens = lens.astype(np.int64)
    padded = (lens + 7) // 8 * 8
    offs = np.zeros(len(lens), dtype=np.int64)
    offs[1:] = np.cumsum(padded)[:-1]
    total = int(padded.sum())
    if total >= 2 ** 32:
        raise ValueError("batch exceeds 4 GiB of bases; split it")
    buf = np.full(total, N_CODE, dtype=np.uint8)
    starts = np.zeros(len(lens), dtype=np.int64)
    starts[1:] = np.cumsum(lens)[:-1]
    pos = np.repeat(offs - starts, lens) + np.arange(int(lens.sum()), dtype=np.int64)
    buf[pos] = flat
    return buf, offs.astype(np.uint32), lens.astype(np.uint32)


def mutate(rng, flat: np.ndarray, lens: np.ndarray, sub_rate, ins_rate, del_rate, max_indel):
    """Apply substitutions, insertions and deletions (lengths U{1..max_indel})
    independently per position.  Rates may be scalars or per-pair arrays."""
    n = len(lens)
    lens = lens.astype(np.int64)
    N = len(flat)
    scalar = all(np.ndim(r) == 0 for r in (sub_rate, ins_rate, del_rate))
    pid = None if scalar else np.repeat(np.arange(n, dtype=np.int32), lens)
    u = rng.random(N, dtype=np.float32)
    if scalar:
        ps, pi, pd = np.float32(sub_rate), np.float32(ins_rate), np.float32(del_rate)
    else:
        ps = np.asarray(sub_rate, dtype=np.float32)[pid]
        pi = np.asarray(ins_rate, dtype=np.float32)[pid]
        pd = np.asarray(del_rate, dtype=np.float32)[pid]
    is_sub = u < ps
    ins_at = np.nonzero((u >= ps) & (u < ps + pi))[0]
    del_at = np.nonzero((u >= ps + pi) & (u < ps + pi + pd))[0]
    del u
    out = flat.copy()
    sub_idx = np.nonzero(is_sub)[0]
    codes = np.searchsorted(ACGT, out[sub_idx])
    codes = np.where(codes < 4, codes, 0)
    out[sub_idx] = ACGT[(codes + rng.integers(1, 4, size=len(sub_idx))) % 4]
    # pair boundaries: a deletion never crosses into the next pair
    ends = np.cumsum(lens)
    keep = np.ones(N, dtype=bool)
    dl = rng.integers(1, max_indel + 1, size=len(del_at))
    del_end = np.minimum(del_at + dl, ends[np.searchsorted(ends, del_at, side="right")])
    for k in range(max_indel):
        idx = del_at + k
        keep[idx[idx < del_end]] = False
    # insertion: after this position, il random bases
    rep = keep.astype(np.int64)
    il = rng.integers(1, max_indel + 1, size=len(ins_at))
    rep[ins_at] += il
    newflat = np.repeat(out, rep)
    first = np.cumsum(rep) - rep
    ins_mask = np.ones(len(newflat), dtype=bool)
    ins_mask[first[keep]] = False
    newflat[ins_mask] = _random_bases(rng, int(ins_mask.sum()))
    starts = ends - lens
    newlens = np.add.reduceat(rep, starts) if N else np.zeros(n, np.int64)
    newlens = np.where(lens > 0, newlens, 0)
    return newflat, newlens.astype(np.int64)


def _per_pair_slices(flat, lens):
    starts = np.zeros(len(lens), dtype=np.int64)
    starts[1:] = np.cumsum(lens)[:-1]
    return starts


def _clip(rng, flat, lens, lo, hi):
    """Truncate sequences longer than hi and extend ones shorter than lo with
    random bases, keeping everything vectorised."""
    lens = lens.astype(np.int64)
    target = np.clip(lens, lo, hi)
    starts = _per_pair_slices(flat, lens)
    keep_n = np.minimum(lens, target)
    pid = np.repeat(np.arange(len(lens)), keep_n)
    within = np.arange(int(keep_n.sum())) - np.repeat(np.cumsum(keep_n) - keep_n, keep_n)
    kept = flat[np.repeat(starts, keep_n) + within]
    extra = target - keep_n
    if extra.sum() == 0:
        return kept, target
    rep = keep_n + extra
    out = np.empty(int(rep.sum()), dtype=np.uint8)
    ostart = np.cumsum(rep) - rep
    okeep = np.repeat(ostart, keep_n) + within
    out[okeep] = kept
    mask = np.ones(len(out), dtype=bool)
    mask[okeep] = False
    out[mask] = _random_bases(rng, int(mask.sum()))
    del pid
    return out, target


def _flank(rng, flat, lens, left, right):
    """Surround each sequence with left[i] / right[i] random bases."""
    lens = lens.astype(np.int64)
    tot = left + lens + right
    out = _random_bases(rng, int(tot.sum()))
    ostart = np.cumsum(tot) - tot
    starts = _per_pair_slices(flat, lens)
    within = np.arange(int(lens.sum())) - np.repeat(starts, lens)
    out[np.repeat(ostart + left, lens) + within] = flat
    return out, tot


def _to_batch(qflat, qlens, tflat, tlens, q_op=None, seed=None) -> Batch:
    q, qo, ql = _stage_flat(qflat, qlens)
    t, to, tl = _stage_flat(tflat, tlens)
    return Batch(q, t, qo, to, ql, tl,
                 q_op=None if q_op is None else np.ascontiguousarray(q_op, dtype=np.uint8),
                 t_op=None if q_op is None else np.zeros(len(ql), dtype=np.uint8),
                 seed=None if seed is None else np.ascontiguousarray(seed, dtype=np.uint32))


def short_read_pairs(n, seed=SEED_BASE, qlo=100, qhi=150, flank_max=20, sub=0.02, indel=0.005,
                     max_indel=3, n_rate=0.001, tlo=None, thi=None):
    """Workload 0 shape: query U[qlo,qhi] with n_rate N; target = query with
    0..flank_max random flanking bases each side, then substitutions and indels."""
    rng = np.random.default_rng(seed)
    qlens = rng.integers(qlo, qhi + 1, size=n)
    qflat = _random_bases(rng, int(qlens.sum()))
    if n_rate > 0:
        m = rng.random(len(qflat)) < n_rate
        qflat[m] = N_CODE
    left = rng.integers(0, flank_max + 1, size=n)
    right = rng.integers(0, flank_max + 1, size=n)
    tflat, tlens = _flank(rng, qflat, qlens, left, right)
    tflat, tlens = mutate(rng, tflat, tlens, sub, indel / 2, indel / 2, max_indel)
    if tlo is not None:
        tflat, tlens = _clip(rng, tflat, tlens, tlo, thi)
    return qflat, qlens, tflat, tlens, rng


def workload0(n=20000, seed=SEED_BASE + 0) -> Batch:
    qf, ql, tf, tl, _ = short_read_pairs(n, seed)
    return _to_batch(qf, ql, tf, tl)


WORKLOAD1_PARAMS = [
    Params(algo=LOCAL, start_pos=WITH_START, second_best=TRUE, reverse_complement=1),
    Params(algo=GLOBAL, start_pos=WITH_START, reverse_complement=1),
    Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, reverse_complement=1),
]


def workload1(n=1_000_000, seed=SEED_BASE + 1):
    """Workload 1: 150 bp queries, 150-300 bp targets (3% subs, 1% indels),
    50% of queries flagged REVERSE_COMPLEMENT; split in thirds LOCAL (second
    best) / GLOBAL / SEMI_GLOBAL (head=tail=TARGET), all WITH_START.
    Returns [(Params, Batch)] for the three launches."""
    rng0 = np.random.default_rng(seed)
    qf, ql, tf, tl, rng = short_read_pairs(n, seed, qlo=150, qhi=150, flank_max=75, sub=0.03,
                                           indel=0.01, n_rate=0.0, tlo=150, thi=300)
    q_op = np.where(rng0.random(n) < 0.5, REVERSE_COMPLEMENT, 0).astype(np.uint8)
    b = _to_batch(qf, ql, tf, tl, q_op=q_op)
    thirds = np.array_split(np.arange(n), 3)
    return [(p, _slice_batch(b, idx)) for p, idx in zip(WORKLOAD1_PARAMS, thirds)]


def _slice_batch(b: Batch, idx: np.ndarray) -> Batch:
    """Contiguous index range -> batch with rebased offsets (no copy of pairs
    outside the range)."""
    lo, hi = int(idx[0]), int(idx[-1]) + 1
    def part(buf, off, ln):
        o0 = int(off[lo])
        end = int(off[hi - 1]) + int((int(ln[hi - 1]) + 7) // 8 * 8)
        return np.ascontiguousarray(buf[o0:end]), (off[lo:hi] - np.uint32(o0)).astype(np.uint32)
    q, qo = part(b.q, b.q_off, b.q_len)
    t, to = part(b.t, b.t_off, b.t_len)
    sl = slice(lo, hi)
    return Batch(q, t, qo, to, np.ascontiguousarray(b.q_len[sl]), np.ascontiguousarray(b.t_len[sl]),
                 q_op=None if b.q_op is None else np.ascontiguousarray(b.q_op[sl]),
                 t_op=None if b.t_op is None else np.ascontiguousarray(b.t_op[sl]),
                 seed=None if b.seed is None else np.ascontiguousarray(b.seed[sl]))


def workload2(n=2_000_000, seed=SEED_BASE + 2) -> Batch:
    """Workload 2: query length log-uniform 50-1000; target = query with per-pair
    1-8% substitutions and 0.5-3% indels of length 1-10 (GLOBAL, WITH_TB)."""
    rng = np.random.default_rng(seed)
    ql = np.exp(rng.uniform(np.log(50), np.log(1000), size=n)).astype(np.int64)
    qf = _random_bases(rng, int(ql.sum()))
    sub = rng.uniform(0.01, 0.08, size=n)
    ind = rng.uniform(0.005, 0.03, size=n)
    tf, tl = mutate(rng, qf, ql, sub, ind / 2, ind / 2, 10)
    tf, tl = _clip(rng, tf, tl, 1, 1 << 30)
    return _to_batch(qf, ql, tf, tl)


def workload3(n=4_000_000, seed=SEED_BASE + 3) -> Batch:
    """Workload 3: ksw extension, query U[250,2000], indel rate per pair from
    {0.5,2,5,10}% plus 1-5% substitutions, seed score h0 U[20,60]."""
    rng = np.random.default_rng(seed)
    ql = rng.integers(250, 2001, size=n)
    qf = _random_bases(rng, int(ql.sum()))
    ind = rng.choice(np.array([0.005, 0.02, 0.05, 0.10]), size=n)
    sub = rng.uniform(0.01, 0.05, size=n)
    tf, tl = mutate(rng, qf, ql, sub, ind / 2, ind / 2, 3)
    tf, tl = _clip(rng, tf, tl, 1, 1 << 30)
    h0 = rng.integers(20, 61, size=n)
    return _to_batch(qf, ql, tf, tl, seed=h0)


WORKLOAD4_PARAMS = [
    Params(algo=LOCAL, start_pos=WITH_START),
    Params(algo=LOCAL, start_pos=WITH_TB),
    Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET),
    Params(algo=KSW, zdrop=100),
]
WORKLOAD4_SHARES = (0.30, 0.20, 0.25, 0.25)


def workload4(n=10_000_000, seed=SEED_BASE + 4):
    """Workload 4: query lengths log-normal (median 250, sigma 0.8, clipped to
    [50, 5000]); 60% short-read-like pairs (1-2% substitutions, 0.2% indels),
    30% long-read-like (5-12% errors, 75% of them indels of length 1-5), 10%
    unrelated random targets of similar length; split into four launches --
    LOCAL WITH_START 30%, LOCAL WITH_TB 20%, SEMI_GLOBAL (TARGET, TARGET)
    WITH_START 25%, ksw (h0 U[20,60], z-drop 100) 25% -- one per stream.
    Returns [(Params, Batch)]."""
    rng = np.random.default_rng(seed)
    ql = np.clip(np.round(250 * np.exp(rng.normal(0, 0.8, size=n))), 50, 5000).astype(np.int64)
    kind = rng.choice(3, size=n, p=[0.6, 0.3, 0.1])
    qf = _random_bases(rng, int(ql.sum()))
    err = np.where(kind == 0, rng.uniform(0.01, 0.02, n), rng.uniform(0.05, 0.12, n))
    sub = np.where(kind == 0, err, 0.25 * err)
    ind = np.where(kind == 0, 0.002, 0.75 * err)
    tf, tl = mutate(rng, qf, ql, sub, ind / 2, ind / 2, 5)
    tl = tl.astype(np.int64)
    # unrelated pairs: replace the target by random bases of the same length
    unrel = np.repeat(kind == 2, tl)
    tf[unrel] = _random_bases(rng, int(unrel.sum()))
    tf, tl = _clip(rng, tf, tl, 1, 1 << 30)
    h0 = rng.integers(20, 61, size=n)
    b = _to_batch(qf, ql, tf, tl, seed=h0)
    cuts = np.round(np.cumsum((0,) + WORKLOAD4_SHARES) * n).astype(np.int64)
    out = []
    for p, lo, hi in zip(WORKLOAD4_PARAMS, cuts[:-1], cuts[1:]):
        if hi > lo:
            out.append((p, _slice_batch(b, np.arange(lo, hi))))
    return out
