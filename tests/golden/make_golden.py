"""Builds the golden fixtures: reference GASAL2 outputs on seeded inputs.

    python tests/golden/make_golden.py --out DIR [--only NAME]

Runs the UNMODIFIED reference library compiled for sm_100a
(oracle/_ref/libgasal_ref_mql2048.so, built by `make -C oracle ref`) through
its own C++ API, on every case in CASES, and writes DIR/<case>.npz holding the
inputs and, per launch configuration, every result array the reference
defines.  Needs a GPU.  The committed fixtures in tests/golden/*.npz were made
by this script; tests compare the scalar oracle and the CUDA path to them.

Inputs that would make the reference read outside its own buffers (see the
filters below) are left out of the cases, because the reference's result is
undefined there.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import np_workloads as W  # noqa: E402  (the generator these fixtures were made with)
from gasal_b200.capi import (Batch, Params, LOCAL, GLOBAL, SEMI_GLOBAL, BANDED, KSW,  # noqa: E402
                             WITHOUT_START, WITH_START, WITH_TB, NONE, QUERY, TARGET, BOTH)

ACGT = b"ACGT"


def rand_seq(rng, n, alphabet=ACGT):
    return bytes(np.frombuffer(alphabet, dtype=np.uint8)[rng.integers(0, len(alphabet), size=n)])


def mutate_bytes(rng, s: bytes, sub=0.05, indel=0.03) -> bytes:
    out = bytearray()
    for ch in s:
        u = rng.random()
        if u < sub:
            out.append(ACGT[(ACGT.index(ch) + int(rng.integers(1, 4))) % 4] if ch in ACGT else ch)
        elif u < sub + indel / 2:
            out.append(ch)
            out += rand_seq(rng, int(rng.integers(1, 4)))
        elif u < sub + indel:
            pass
        else:
            out.append(ch)
    return bytes(out)


EDGE_LENS = [1, 2, 3, 5, 7, 8, 9, 15, 16, 17, 24, 31, 33, 40]


def case_edge(seed=11):
    """Every (query, target) length pair around multiples of 8; half related
    (target mutated from query), half random."""
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for lq in EDGE_LENS:
        for lt in EDGE_LENS:
            q = rand_seq(rng, lq)
            if rng.random() < 0.5:
                t = mutate_bytes(rng, q)[:lt]
                t = t + rand_seq(rng, lt - len(t))
            else:
                t = rand_seq(rng, lt)
            qs.append(q)
            ts.append(t)
    seeds = rng.integers(0, 61, size=len(qs))
    return Batch.from_seqs(qs, ts, seed=seeds)


def case_special(seed=12):
    """N-rich, all-N, lower case, homopolymers, long gaps."""
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for i in range(160):
        lq = int(rng.integers(1, 70))
        kind = i % 8
        if kind == 0:
            q = b"N" * lq
            t = rand_seq(rng, int(rng.integers(1, 70)))
        elif kind == 1:
            q = rand_seq(rng, lq, b"ACGTN")
            t = mutate_bytes(rng, q)
        elif kind == 2:
            q = rand_seq(rng, lq, b"acgt")
            t = mutate_bytes(rng, q.upper()).lower()
        elif kind == 3:
            q = b"A" * lq
            t = b"A" * int(rng.integers(1, 70))
        elif kind == 4:
            q = rand_seq(rng, lq)
            cut = int(rng.integers(0, lq + 1))
            t = q[:cut] + rand_seq(rng, int(rng.integers(5, 30))) + q[cut:]
        elif kind == 5:
            q = rand_seq(rng, lq)
            a, c = sorted(rng.integers(0, lq + 1, size=2))
            t = q[:a] + q[c:]
            if not t:
                t = b"G"
        elif kind == 6:
            q = rand_seq(rng, lq, b"ACGTRYKM")
            t = mutate_bytes(rng, q.replace(b"R", b"A"))
        else:
            q = rand_seq(rng, lq)
            t = rand_seq(rng, int(rng.integers(1, 70)))
        qs.append(q)
        ts.append(t)
    seeds = rng.integers(0, 61, size=len(qs))
    return Batch.from_seqs(qs, ts, seed=seeds)


def case_rc(seed=13):
    """Reverse / complement ops on query and target, lengths 1..48."""
    rng = np.random.default_rng(seed)
    # A one-word sequence that is reversed makes the reference read the packed
    # word just before it (pack_rc_seqs.h:286,303); the leading pair without
    # ops keeps that read inside the buffer for every later pair.
    qs, ts, qo, to = [rand_seq(rng, 16)], [rand_seq(rng, 16)], [0], [0]
    for lq in range(1, 49):
        for op in range(4):
            q = rand_seq(rng, lq)
            t = mutate_bytes(rng, q) or b"C"
            qs.append(q)
            ts.append(t)
            qo.append(op)
            to.append((op + lq) % 4)
    return Batch.from_seqs(qs, ts, q_op=qo, t_op=to)


def case_short(seed=14, n=1500):
    """Workload-0 shape (100-150 bp, flanks, 2% subs, 0.5% indels, 0.1% N)."""
    return W.workload0(n, seed=seed)


def case_w1(seed=15, n=1500):
    """Workload-1 shape: 150 bp queries, 150-300 bp targets, RC on half."""
    qf, ql, tf, tl, rng = W.short_read_pairs(n, seed, qlo=150, qhi=150, flank_max=75, sub=0.03,
                                             indel=0.01, n_rate=0.0, tlo=150, thi=300)
    q_op = np.where(np.random.default_rng(seed + 1).random(n) < 0.5, 3, 0)
    return W._to_batch(qf, ql, tf, tl, q_op=q_op)


def case_long(seed=16, n=120):
    """Workload-2 shape: log-uniform 50-1000 bp, per-pair mutation rates."""
    return W.workload2(n, seed=seed)


def case_ksw(seed=17, n=120):
    """Workload-3 shape: ksw extension inputs (250-2000 bp, h0 20-60)."""
    return W.workload3(n, seed=seed)


def case_empty(seed=18):
    """Empty queries and/or targets among ordinary pairs.  ksw returns the
    seed score for them; LOCAL returns zeros."""
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for i in range(48):
        lq, lt = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        kind = i % 4
        q = rand_seq(rng, lq) if kind in (0, 2) else b""
        t = (mutate_bytes(rng, q) or b"A") if kind == 0 else (rand_seq(rng, lt) if kind == 1 else b"")
        qs.append(q)
        ts.append(t)
    seeds = rng.integers(0, 61, size=len(qs))
    return Batch.from_seqs(qs, ts, seed=seeds)


def semi_start_ok(b: Batch, tail: int) -> np.ndarray:
    """Pairs on which the reference's semi-global start pass stays inside its
    reversed-target array.  With a QUERY/BOTH tail the end row can be set to the
    query length (semiglobal_kernel_template.h:206-207); the start pass then
    begins at word target_regs-((read_len>>3)+1), negative when the query is
    longer than the padded target (:273,301,321)."""
    if tail not in (QUERY, BOTH):
        return np.ones(b.n, dtype=bool)
    tregs = (b.t_len.astype(np.int64) + 7) // 8
    return (b.q_len.astype(np.int64) >> 3) + 1 <= tregs


def configs_for(case: str):
    cfg = []
    if case in ("edge", "special", "short"):
        for s in (WITHOUT_START, WITH_START, WITH_TB):
            for sb in (0, 1):
                cfg.append(Params(algo=LOCAL, start_pos=s, second_best=sb))
        for s in (WITHOUT_START, WITH_TB):
            cfg.append(Params(algo=GLOBAL, start_pos=s))
        for h in (NONE, QUERY, TARGET, BOTH):
            for t in (NONE, QUERY, TARGET, BOTH):
                cfg.append(Params(algo=SEMI_GLOBAL, start_pos=WITHOUT_START, head=h, tail=t, second_best=1))
                cfg.append(Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=h, tail=t, second_best=0))
        for k in (8, 16, 40):
            cfg.append(Params(algo=BANDED, k_band=k))
        cfg.append(Params(algo=KSW))
        if case == "edge":
            cfg.append(Params(algo=LOCAL, start_pos=WITH_START, second_best=1, match=2, mismatch=3, gap_open=4, gap_extend=2))
            cfg.append(Params(algo=GLOBAL, start_pos=WITH_TB, match=2, mismatch=3, gap_open=4, gap_extend=2))
            cfg.append(Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, match=2, mismatch=3, gap_open=4, gap_extend=2))
            cfg.append(Params(algo=KSW, match=2, mismatch=3, gap_open=4, gap_extend=2))
    elif case == "rc":
        for a, s, sb in ((LOCAL, WITH_START, 1), (GLOBAL, WITH_TB, 0), (LOCAL, WITH_TB, 0), (KSW, WITHOUT_START, 0)):
            cfg.append(Params(algo=a, start_pos=s, second_best=sb, reverse_complement=1))
        cfg.append(Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, reverse_complement=1))
    elif case == "w1":
        cfg += [Params(algo=LOCAL, start_pos=WITH_START, second_best=1, reverse_complement=1),
                Params(algo=GLOBAL, start_pos=WITH_START, reverse_complement=1),
                Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, reverse_complement=1),
                Params(algo=LOCAL, start_pos=WITH_TB, reverse_complement=1)]
    elif case == "long":
        cfg += [Params(algo=GLOBAL, start_pos=WITH_TB), Params(algo=LOCAL, start_pos=WITH_START, second_best=1),
                Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=BOTH, tail=BOTH)]
    elif case == "ksw":
        cfg += [Params(algo=KSW), Params(algo=LOCAL, start_pos=WITHOUT_START)]
    elif case == "empty":
        cfg += [Params(algo=KSW), Params(algo=KSW, match=2, mismatch=3, gap_open=4, gap_extend=2),
                Params(algo=LOCAL, start_pos=WITHOUT_START)]
    return cfg


CASES = {
    "edge": case_edge,
    "special": case_special,
    "rc": case_rc,
    "short": case_short,
    "w1": case_w1,
    "long": case_long,
    "ksw": case_ksw,
    "empty": case_empty,
}


def build_inputs(name: str) -> Batch:
    return CASES[name]()


def subset_for(b: Batch, p: Params) -> np.ndarray:
    """Indices of the pairs a configuration is run on."""
    ok = np.ones(b.n, dtype=bool)
    if p.algo == SEMI_GLOBAL and p.start_pos == WITH_START:
        ok &= semi_start_ok(b, p.tail)
    if p.start_pos == WITH_TB and p.algo in (LOCAL, GLOBAL):
        ok &= cigar_fits(b, p)
    return np.nonzero(ok)[0]


def cigar_fits(b: Batch, p: Params) -> np.ndarray:
    """The reference writes each CIGAR into the pair's own padded query slot
    (get_tb.h:13,94); a longer CIGAR runs into the next pair's slot while that
    pair's thread writes there too, so its bytes are a data race.  The number
    of operations does not depend on the bytes, so the host build of the
    reference kernels decides which pairs stay inside their slot."""
    from oracle.bindings import ref_host_align
    o = ref_host_align(p, b)
    slot = (b.q_len.astype(np.int64) + 7) // 8 * 8
    return o.n_cigar.astype(np.int64) <= slot


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    from oracle.bindings import ref_gpu_align
    os.makedirs(args.out, exist_ok=True)
    for name in CASES:
        if args.only and name != args.only:
            continue
        b = build_inputs(name)
        store = {("in__" + k): v for k, v in b.arrays().items()}
        for p in configs_for(name):
            idx = subset_for(b, p)
            sb = b if len(idx) == b.n else b.subset(idx)
            out, _ = ref_gpu_align(p, sb, want_packed=(name == "rc"))
            key = p.key()
            store[f"idx__{key}"] = idx.astype(np.int32)
            for f, v in out.as_dict(p, sb).items():
                store[f"out__{key}__{f}"] = v
            if name == "rc":
                store[f"out__{key}__packed_q"] = out.packed_q
                store[f"out__{key}__packed_t"] = out.packed_t
            print(f"{name:8s} {key:60s} n={sb.n}", flush=True)
        np.savez_compressed(os.path.join(args.out, f"{name}.npz"), **store)


if __name__ == "__main__":
    main()
