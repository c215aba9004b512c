"""ctypes loaders for the checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline / reference legs -- never by the product package.

  oracle_align      scalar C restatement (liboracle_gasal.so), OpenMP over pairs
  ref_host_align    reference kernel headers compiled for the host
                    (_ref/libgasal_ref_host.so)
  ref_gpu_align     reference GASAL2 built for sm_100a, driven through its own
                    C++ API (_ref/libgasal_ref_mqlN.so; needs a GPU)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from gasal_b200.capi import Batch, Outputs, Params

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def _load(name):
    if name not in _libs:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle` / `make -C oracle ref`)")
        _libs[name] = C.CDLL(path)
    return _libs[name]


def _call(fn, p: Params, b: Batch, want_packed=False, extra=()):
    out = Outputs(b, want_packed)
    cp, cb, co = p.to_c(), b.to_c(), out.to_c()
    rc = fn(C.byref(cp), C.byref(cb), C.byref(co), *extra)
    if rc != 0:
        raise RuntimeError(f"{fn.__name__} returned {rc}")
    return out


ORC_ALL = 0x0F  # every reference quirk on (gasal_oracle.h)


def oracle_align(p: Params, b: Batch, threads: int = 0, want_packed=False, compat: int = ORC_ALL,
                 mql: int = 2048) -> Outputs:
    lib = _load("liboracle_gasal.so")
    fn = lib.oracle_align_ex
    fn.restype = C.c_int
    return _call(fn, p, b, want_packed, (C.c_int(threads), C.c_int(compat), C.c_int(mql)))


def oracle_cigar_text(cigar: np.ndarray, q_off: np.ndarray, n_cigar: np.ndarray, stride: int):
    """Forward CIGAR strings (the reference test program's decode); returns
    (list of str, int32 lengths with -1 where stride was too small)."""
    lib = _load("liboracle_gasal.so")
    n = len(n_cigar)
    cig = np.ascontiguousarray(cigar, dtype=np.uint8)
    qo = np.ascontiguousarray(q_off, dtype=np.uint32)
    nc = np.ascontiguousarray(n_cigar, dtype=np.uint32)
    text = np.zeros(n * stride, dtype=np.uint8)
    lens = np.zeros(n, dtype=np.int32)
    fn = lib.oracle_cigar_text
    fn.restype = None
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    fn(cig.ctypes.data, qo.ctypes.data, nc.ctypes.data, n, text.ctypes.data, stride, lens.ctypes.data)
    strs = [bytes(text[i * stride:i * stride + max(int(lens[i]), 0)]).decode() for i in range(n)]
    return strs, lens


def ref_host_align(p: Params, b: Batch, threads: int = 0, want_packed=False) -> Outputs:
    lib = _load(os.path.join("_ref", "libgasal_ref_host.so"))
    fn = lib.ref_host_align
    fn.restype = C.c_int
    return _call(fn, p, b, want_packed, (C.c_int(threads),))


def ref_gpu_align(p: Params, b: Batch, want_packed=False, mql: int = 2048, repeats: int = 1):
    """Returns (Outputs, ms_per_call) where ms is host wall time from
    gasal_aln_async to gasal_is_aln_async_done()==0, averaged over repeats."""
    lib = _load(os.path.join("_ref", f"libgasal_ref_mql{mql}.so"))
    fn = lib.ref_gpu_align
    fn.restype = C.c_int
    ms = C.c_double(0.0)
    out = _call(fn, p, b, want_packed, (C.c_int(repeats), C.byref(ms)))
    return out, ms.value


def max_padded_len(b: Batch) -> int:
    return int(max(((b.q_len.astype(np.int64) + 7) // 8 * 8).max(), ((b.t_len.astype(np.int64) + 7) // 8 * 8).max()))
