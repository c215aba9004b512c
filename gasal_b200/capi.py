"""ctypes mirror of include/gasal_b200_capi.h and a numpy batch container.

The structs here are field-for-field copies of ``gb_params_t``, ``gb_batch_t``
and ``gb_out_t``.  ``Batch`` holds one batch in GASAL2's staging layout: ASCII
bases, every sequence at its byte offset, N-padded to a multiple of 8
(reference src/host_batch.cpp:100-146, src/gasal_align.cu:152-175).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# enum values of include/gasal.h (reference src/gasal.h:37-72)
WITHOUT_START, WITH_START, WITH_TB = 0, 1, 2
FALSE, TRUE = 0, 1
NONE, QUERY, TARGET, BOTH = 0, 1, 2, 3
UNKNOWN, GLOBAL, SEMI_GLOBAL, LOCAL, MICROLOCAL, BANDED, KSW = 0, 1, 2, 3, 4, 5, 6
FORWARD_NATURAL, REVERSE_NATURAL, FORWARD_COMPLEMENT, REVERSE_COMPLEMENT = 0, 1, 2, 3

ALGO_NAMES = {GLOBAL: "global", SEMI_GLOBAL: "semi_global", LOCAL: "local", BANDED: "banded", KSW: "ksw"}
N_CODE = 0x4E

GB_OK = 0
GB_STATUS = {0: "ok", -1: "bad argument", -2: "CUDA error", -3: "not ready", -4: "no work",
             -5: "allocation failed", -6: "limit exceeded"}


class GbParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "algo", "start_pos", "second_best", "head", "tail", "k_band", "reverse_complement", "zdrop",
        "match", "mismatch", "gap_open", "gap_extend")]


class GbBatch(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("q_bytes", C.c_uint32), ("t_bytes", C.c_uint32),
        ("q", C.c_void_p), ("t", C.c_void_p),
        ("q_off", C.c_void_p), ("t_off", C.c_void_p), ("q_len", C.c_void_p), ("t_len", C.c_void_p),
        ("q_op", C.c_void_p), ("t_op", C.c_void_p), ("seed", C.c_void_p)]


class GbOut(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2",
        "cigar", "n_cigar", "packed_q", "packed_t")]


@dataclass
class Params:
    """Per-launch options (the fields of GASAL2's ``Parameters`` the path reads)."""
    algo: int = LOCAL
    start_pos: int = WITHOUT_START
    second_best: int = FALSE
    head: int = TARGET
    tail: int = TARGET
    k_band: int = 0
    reverse_complement: int = 0
    zdrop: int = 0
    match: int = 1
    mismatch: int = 4
    gap_open: int = 6
    gap_extend: int = 1

    def to_c(self) -> GbParams:
        return GbParams(*[int(getattr(self, f)) for f, _ in GbParams._fields_])

    def key(self) -> str:
        return (f"{ALGO_NAMES.get(self.algo, self.algo)}_s{self.start_pos}_b{self.second_best}"
                f"_h{self.head}t{self.tail}_k{self.k_band}_rc{self.reverse_complement}_z{self.zdrop}"
                f"_m{self.match}x{self.mismatch}o{self.gap_open}e{self.gap_extend}")


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


@dataclass
class Batch:
    q: np.ndarray          # uint8 [q_bytes]
    t: np.ndarray          # uint8 [t_bytes]
    q_off: np.ndarray      # uint32 [n]
    t_off: np.ndarray
    q_len: np.ndarray
    t_len: np.ndarray
    q_op: Optional[np.ndarray] = None   # uint8 [n]
    t_op: Optional[np.ndarray] = None
    seed: Optional[np.ndarray] = None   # uint32 [n]
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n(self) -> int:
        return int(self.q_len.shape[0])

    @staticmethod
    def from_seqs(queries, targets, q_op=None, t_op=None, seed=None) -> "Batch":
        """Stage a list of byte strings exactly as gasal_host_batch_fill does."""
        def stage(seqs):
            lens = np.array([len(s) for s in seqs], dtype=np.uint32)
            padded = (lens + 7) & ~np.uint32(7)
            offs = np.zeros(len(seqs), dtype=np.uint32)
            if len(seqs) > 1:
                offs[1:] = np.cumsum(padded[:-1], dtype=np.uint64).astype(np.uint32)
            buf = np.full(int(padded.sum()), N_CODE, dtype=np.uint8)
            for s, o in zip(seqs, offs):
                if len(s):
                    buf[int(o):int(o) + len(s)] = np.frombuffer(bytes(s), dtype=np.uint8)
            return buf, offs, lens
        q, qo, ql = stage(queries)
        t, to, tl = stage(targets)
        b = Batch(q, t, qo, to, ql, tl)
        if q_op is not None:
            b.q_op = np.ascontiguousarray(q_op, dtype=np.uint8)
        if t_op is not None:
            b.t_op = np.ascontiguousarray(t_op, dtype=np.uint8)
        if seed is not None:
            b.seed = np.ascontiguousarray(seed, dtype=np.uint32)
        return b

    def seq(self, i: int, which: str = "q") -> bytes:
        buf, off, ln = (self.q, self.q_off, self.q_len) if which == "q" else (self.t, self.t_off, self.t_len)
        return bytes(buf[int(off[i]):int(off[i]) + int(ln[i])])

    def subset(self, idx) -> "Batch":
        idx = np.asarray(idx)
        qs = [self.seq(int(i), "q") for i in idx]
        ts = [self.seq(int(i), "t") for i in idx]
        return Batch.from_seqs(qs, ts,
                               None if self.q_op is None else self.q_op[idx],
                               None if self.t_op is None else self.t_op[idx],
                               None if self.seed is None else self.seed[idx])

    def to_c(self) -> GbBatch:
        return GbBatch(self.n, int(self.q.shape[0]), int(self.t.shape[0]),
                       _ptr(self.q), _ptr(self.t), _ptr(self.q_off), _ptr(self.t_off),
                       _ptr(self.q_len), _ptr(self.t_len), _ptr(self.q_op), _ptr(self.t_op),
                       _ptr(self.seed))

    def cells(self) -> int:
        return int(np.dot(self.q_len.astype(np.int64), self.t_len.astype(np.int64)))

    def padded_cells(self) -> int:
        q8 = (self.q_len.astype(np.int64) + 7) // 8 * 8
        t8 = (self.t_len.astype(np.int64) + 7) // 8 * 8
        return int(np.dot(q8, t8))

    def arrays(self) -> dict:
        d = dict(q=self.q, t=self.t, q_off=self.q_off, t_off=self.t_off, q_len=self.q_len, t_len=self.t_len)
        for k in ("q_op", "t_op", "seed"):
            v = getattr(self, k)
            if v is not None:
                d[k] = v
        return d

    @staticmethod
    def from_arrays(d) -> "Batch":
        return Batch(*(np.ascontiguousarray(d[k]) for k in ("q", "t", "q_off", "t_off", "q_len", "t_len")),
                     q_op=d["q_op"] if "q_op" in d else None,
                     t_op=d["t_op"] if "t_op" in d else None,
                     seed=d["seed"] if "seed" in d else None)


OUT_FIELDS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")


def has_cigar(p: Params) -> bool:
    """Whether a launch with these options writes CIGARs: LOCAL and GLOBAL
    WITH_TB, and (an extension) target-tail SEMI_GLOBAL WITH_TB."""
    return p.start_pos == WITH_TB and (p.algo in (LOCAL, GLOBAL) or (p.algo == SEMI_GLOBAL and p.tail == TARGET))


class Outputs:
    """Host arrays for every result a launch can produce."""

    def __init__(self, batch: Batch, want_packed: bool = False):
        n = batch.n
        for f in OUT_FIELDS:
            setattr(self, f, np.zeros(n, dtype=np.int32))
        self.cigar = np.zeros(int(batch.q.shape[0]), dtype=np.uint8)
        self.n_cigar = np.zeros(n, dtype=np.uint32)
        self.packed_q = np.zeros(int(batch.q.shape[0]) // 8, dtype=np.uint32) if want_packed else None
        self.packed_t = np.zeros(int(batch.t.shape[0]) // 8, dtype=np.uint32) if want_packed else None

    def to_c(self) -> GbOut:
        return GbOut(*[_ptr(getattr(self, f)) for f, _ in GbOut._fields_])

    def fields_for(self, p: Params) -> list:
        """Result arrays the reference defines for these options (src/res.cpp:8-70,
        kernels write only what their template instance computes)."""
        f = ["score"]
        if p.algo == GLOBAL:
            pass
        elif p.algo == KSW:
            f += ["q_end", "t_end"]
        elif p.algo == BANDED:
            f += ["q_end", "t_end"]
            if p.start_pos == WITH_START:  # an extension: the reference's banded kernel has no start
                f += ["q_start", "t_start"]
        else:
            f += ["q_end", "t_end"]
            if p.start_pos in (WITH_START, WITH_TB) and not (p.algo == SEMI_GLOBAL and p.start_pos == WITH_TB
                                                             and p.tail != TARGET):
                f += ["q_start", "t_start"]  # target-tail SEMI_GLOBAL WITH_TB: an extension
            if p.second_best and p.algo in (LOCAL, SEMI_GLOBAL):
                f += ["score2", "q_end2", "t_end2"]
        return f

    def as_dict(self, p: Params, batch: Optional[Batch] = None) -> dict:
        d = {k: getattr(self, k).copy() for k in self.fields_for(p)}
        if has_cigar(p):
            d["n_cigar"] = self.n_cigar.copy()
            d["cigar"] = self.cigar.copy()
        return d


def cigar_ops(out_cigar: np.ndarray, n_cigar: np.ndarray, q_off: np.ndarray, i: int):
    """Decode pair i's run-length CIGAR bytes ((count << 2) | op, written last
    operation first) into [(op, count)] in forward order."""
    o = int(q_off[i])
    raw = out_cigar[o:o + int(n_cigar[i])]
    return [(int(b) & 3, int(b) >> 2) for b in raw[::-1]]
