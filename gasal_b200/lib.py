"""Python binding of libgasal_b200.so (the C ABI of include/gasal_b200_capi.h).

This module is the host-side mirror of GASAL2's interface for Python callers:
``Streams`` wraps the storage API (gasal_init_streams, gasal_host_batch_fill,
gasal_op_fill, gasal_aln_async, gasal_is_aln_async_done -- reference
src/ctors.h, src/host_batch.h, src/interfaces.h, src/gasal_align.h) and
``align`` is the one-shot batch call.  The library is compiled CUDA for
sm_100a; there is no CPU path, and every call raises if the shared library is
missing or returns an error.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .capi import (Batch, GbBatch, GbOut, GbParams, Outputs, Params, GB_STATUS, KSW, WITH_TB, QUERY,
                   TARGET, _ptr)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgasal_b200.so")
_lib = None


class GasalError(RuntimeError):
    pass


def build(quiet: bool = True) -> str:
    """Compile the CUDA library in place (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), "-j8"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return LIB_PATH


class GbDevBatch(C.Structure):
    _fields_ = [("n", C.c_int32), ("q_bytes", C.c_uint32), ("t_bytes", C.c_uint32)] + \
               [(k, C.c_void_p) for k in ("q", "t", "pq", "pt", "q_off", "t_off", "q_len", "t_len", "q_op",
                                           "t_op", "seed", "h_q_len", "h_t_len")]


class GbDevOut(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2",
                                           "t_end2", "cigar", "n_cigar")]


class GbTuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("wc_min_qregs", C.c_int32), ("min_order_pairs", C.c_int32),
                ("ksw_warp", C.c_int32), ("split_start", C.c_int32), ("persistent", C.c_int32),
                ("wc_group", C.c_int32)]


class GbBandStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("pairs", "accepted", "retried", "handed_back", "cells")]


class GbStorageView(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in (
        "host_query_batch_offsets", "host_target_batch_offsets", "host_query_batch_lens",
        "host_target_batch_lens", "host_query_op", "host_target_op", "host_seed_scores", "aln_score",
        "query_batch_end", "target_batch_end", "query_batch_start", "target_batch_start", "cigar",
        "n_cigar_ops", "aln_score2", "query_batch_end2", "target_batch_end2", "stream")] + \
        [("host_max_n_alns", C.c_uint32), ("host_max_query_batch_bytes", C.c_uint32),
         ("host_max_target_batch_bytes", C.c_uint32)]


# name -> (restype, argtypes)
SIGNATURES = {
    "gasal_c_params_new": (C.c_void_p, []),
    "gasal_c_params_set": (C.c_int, [C.c_void_p, C.POINTER(GbParams)]),
    "gasal_c_params_free": (None, [C.c_void_p]),
    "gasal_c_copy_subst_scores": (C.c_int, [C.c_int32] * 4),
    "gasal_c_init_gpu_storage_v": (C.c_void_p, [C.c_int]),
    "gasal_c_init_streams": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "gasal_c_destroy_streams": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gasal_c_destroy_gpu_storage_v": (C.c_int, [C.c_void_p]),
    "gasal_c_storage": (C.c_void_p, [C.c_void_p, C.c_int]),
    "gasal_c_storage_view": (C.c_int, [C.c_void_p, C.POINTER(GbStorageView)]),
    "gasal_c_host_batch_fill": (C.c_uint32, [C.c_void_p, C.c_uint32, C.c_char_p, C.c_uint32, C.c_int]),
    "gasal_c_host_batch_add": (C.c_uint32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int]),
    "gasal_c_host_batch_fill_mt": (C.c_uint32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_int, C.c_int]),
    "gasal_c_host_batch_reset": (C.c_int, [C.c_void_p]),
    "gasal_c_op_fill": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int]),
    "gasal_c_host_alns_resize": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "gasal_c_set_device": (C.c_int, [C.c_int]),
    "gasal_c_aln_async": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]),
    "gasal_c_is_aln_async_done": (C.c_int, [C.c_void_p]),
    "gb_align": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbBatch), C.POINTER(GbOut)]),
    "gb_align_dev": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbDevBatch), C.POINTER(GbDevOut), C.c_void_p]),
    "gb_pack_dev": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "gb_revcomp_dev": (C.c_int, [C.c_void_p] * 8 + [C.c_int32, C.c_void_p]),
    "gb_align_dev_noalloc": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbDevBatch), C.POINTER(GbDevOut),
                                       C.c_void_p]),
    "gb_align_dev_mixed": (C.c_int, [C.POINTER(GbParams), C.c_int, C.c_void_p, C.POINTER(GbDevBatch),
                                     C.POINTER(GbDevOut), C.c_void_p]),
    "gb_mixed_check": (C.c_int, [C.POINTER(GbParams), C.c_int, C.c_void_p, C.c_int32, C.c_int, C.c_void_p]),
    "gb_release_workspaces": (C.c_int, []),
    "gb_set_reference_reverse": (C.c_int, [C.c_int]),
    "gb_set_reference_max_query_len": (C.c_int, [C.c_int]),
    "gb_set_tb_budget_mb": (C.c_int, [C.c_int64]),
    "gb_version": (C.c_char_p, []),
    "gb_set_graphs": (C.c_int, [C.c_int]),
    "gb_graph_stats": (C.c_int, [C.POINTER(C.c_int64)]),
    "gb_set_tuning": (C.c_int, [C.POINTER(GbTuning)]),
    "gb_get_tuning": (C.c_int, [C.POINTER(GbTuning)]),
    "gb_band_param_count": (C.c_int, []),
    "gb_band_feature_stride": (C.c_int, []),
    "gb_band_model_new": (C.c_void_p, [C.c_uint64]),
    "gb_band_model_free": (None, [C.c_void_p]),
    "gb_band_model_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "gb_band_features": (C.c_int, [C.POINTER(GbDevBatch), C.c_void_p, C.c_void_p]),
    "gb_band_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "gb_band_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    "gb_band_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                     C.POINTER(C.c_float)]),
    "gb_set_band_model": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "gb_ksw_align_max_off": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbDevBatch), C.POINTER(GbDevOut), C.c_void_p,
                                       C.c_void_p]),
    "gb_ksw_band_align": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbDevBatch), C.POINTER(GbDevOut), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.POINTER(GbBandStats)]),
    "gb_last_error": (C.c_char_p, []),
    "gb_cigar_text": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                C.c_void_p]),
    "gb_autotune": (C.c_int, [C.POINTER(GbParams), C.POINTER(GbDevBatch), C.POINTER(GbDevOut), C.c_void_p, C.c_int,
                              C.POINTER(GbTuning), C.POINTER(C.c_double)]),
    "gb_kernel_timing": (C.c_int, [C.c_int]),
    "gb_kernel_timing_read": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "gb_probe_int_peak": (C.c_int, [C.POINTER(C.c_double)] * 3),
    "gb_probe_dpx16x2_peak": (C.c_int, [C.POINTER(C.c_double)]),
}


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GasalError(f"{LIB_PATH} is not built; run gasal_b200.lib.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        raise GasalError(f"{what} failed: {GB_STATUS.get(rc, rc)}")


def align(p: Params, b: Batch, want_packed: bool = False) -> Outputs:
    """Align one batch on the GPU (host buffers in, host buffers out)."""
    out = Outputs(b, want_packed)
    cp, cb, co = p.to_c(), b.to_c(), out.to_c()
    _check(lib().gb_align(C.byref(cp), C.byref(cb), C.byref(co)), "gb_align")
    return out


def set_reference_max_query_len(mql: int):
    _check(lib().gb_set_reference_max_query_len(int(mql)), "gb_set_reference_max_query_len")


def set_reference_reverse(on: bool):
    _check(lib().gb_set_reference_reverse(1 if on else 0), "gb_set_reference_reverse")


def set_tb_budget_mb(mb: int):
    _check(lib().gb_set_tb_budget_mb(int(mb)), "gb_set_tb_budget_mb")


def set_graphs(on: bool):
    """Run each gasal_aln_async batch as a CUDA graph (default on)."""
    _check(lib().gb_set_graphs(1 if on else 0), "gb_set_graphs")


def graph_stats() -> dict:
    c = (C.c_int64 * 4)()
    _check(lib().gb_graph_stats(c), "gb_graph_stats")
    return {"relaunched": c[0], "updated": c[1], "instantiated": c[2], "capture_refused": c[3]}


def get_tuning() -> dict:
    t = GbTuning()
    _check(lib().gb_get_tuning(C.byref(t)), "gb_get_tuning")
    return {k: getattr(t, k) for k, _ in GbTuning._fields_}


# The plain full-DP form: every pair one per thread, in input order, on a grid
# over the batch (no device work counter, no length ordering, no warp kernels,
# start passes inside the forward launch).
PLAIN_FORM = dict(min_order_pairs=1 << 30, ksw_warp=0, split_start=0, persistent=0)


def set_tuning(**kw):
    """Change any of block, wc_min_qregs, min_order_pairs, ksw_warp, split_start, persistent, wc_group."""
    cur = get_tuning()
    bad = set(kw) - set(cur)
    if bad:
        raise GasalError(f"unknown tuning keys {sorted(bad)}")
    cur.update({k: int(v) for k, v in kw.items()})
    t = GbTuning(*[cur[k] for k, _ in GbTuning._fields_])
    _check(lib().gb_set_tuning(C.byref(t)), "gb_set_tuning")


KERNEL_KINDS = ("pack", "revcomp", "dp", "traceback", "order", "span")
# kernels behind one mark of each kind; "span" marks the alignment phase's wall clock, no kernel of its own
KERNELS_PER_MARK = {"pack": 1, "revcomp": 1, "dp": 1, "traceback": 1, "order": 3, "span": 0}


def kernel_timing(on: bool):
    _check(lib().gb_kernel_timing(1 if on else 0), "gb_kernel_timing")


def kernel_timing_read() -> dict:
    ms = (C.c_double * len(KERNEL_KINDS))()
    n = (C.c_int64 * len(KERNEL_KINDS))()
    _check(lib().gb_kernel_timing_read(ms, n), "gb_kernel_timing_read")
    return {k: (ms[i], n[i]) for i, k in enumerate(KERNEL_KINDS)}


def probe_int_peak() -> dict:
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    _check(lib().gb_probe_int_peak(C.byref(a), C.byref(b), C.byref(c)), "gb_probe_int_peak")
    d = C.c_double()
    _check(lib().gb_probe_dpx16x2_peak(C.byref(d)), "gb_probe_dpx16x2_peak")
    return {"iadd_tops": a.value, "imnmx_tops": b.value, "dpx_tops": c.value, "dpx16x2_halfword_tops": d.value}


def _dev_structs(dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray):
    b = GbDevBatch()
    b.n = int(h_q_len.shape[0])
    b.q_bytes, b.t_bytes = int(dev["q_bytes"]), int(dev["t_bytes"])
    for k in ("q", "t", "pq", "pt", "q_off", "t_off", "q_len", "t_len", "q_op", "t_op", "seed"):
        setattr(b, k, dev.get(k))
    b.h_q_len, b.h_t_len = _ptr(h_q_len), _ptr(h_t_len)
    o = GbDevOut()
    for k, _ in GbDevOut._fields_:
        setattr(o, k, dev.get("out_" + k))
    return b, o


def autotune(p: Params, dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray, stream_handle: int = 0,
             reps: int = 2) -> dict:
    """gb_autotune on a device-resident batch (same ``dev`` map as
    align_dev): installs and returns the fastest launch tuning."""
    b, o = _dev_structs(dev, h_q_len, h_t_len)
    cp = p.to_c()
    t = GbTuning()
    ms = C.c_double()
    rc = lib().gb_autotune(C.byref(cp), C.byref(b), C.byref(o), C.c_void_p(stream_handle), int(reps), C.byref(t),
                           C.byref(ms))
    if rc != 0:
        raise GasalError(f"gb_autotune failed: {GB_STATUS.get(rc, rc)} ({lib().gb_last_error().decode()})")
    d = {k: getattr(t, k) for k, _ in GbTuning._fields_}
    d["ms"] = ms.value
    return d


BAND_BLOB_MAGIC = b"GBBAND01"


def band_blob(params: np.ndarray, feature_stride: int) -> bytes:
    """Serialised band-model weights: magic, parameter count and feature
    stride (uint32 little endian), the float32 parameters in the
    gb_band_model_params layout, then a CRC-32 of everything before it."""
    import struct
    import zlib
    p = np.ascontiguousarray(params, dtype="<f4")
    body = BAND_BLOB_MAGIC + struct.pack("<II", p.shape[0], int(feature_stride)) + p.tobytes()
    return body + struct.pack("<I", zlib.crc32(body) & 0xFFFFFFFF)


def band_unblob(blob: bytes, n_params: int, feature_stride: int) -> np.ndarray:
    """Parameters from band_blob(); raises GasalError when the magic, the
    sizes or the checksum do not match this library's model."""
    import struct
    import zlib
    head = len(BAND_BLOB_MAGIC) + 8
    if len(blob) < head + 4 or blob[:len(BAND_BLOB_MAGIC)] != BAND_BLOB_MAGIC:
        raise GasalError("band model blob: bad magic or truncated")
    n, stride = struct.unpack("<II", blob[len(BAND_BLOB_MAGIC):head])
    if n != n_params or stride != feature_stride:
        raise GasalError(f"band model blob: {n} parameters / stride {stride}, library has {n_params} / {feature_stride}")
    if len(blob) != head + 4 * n + 4:
        raise GasalError("band model blob: wrong length")
    (crc,) = struct.unpack("<I", blob[-4:])
    if zlib.crc32(blob[:-4]) & 0xFFFFFFFF != crc:
        raise GasalError("band model blob: checksum mismatch")
    return np.frombuffer(blob[head:head + 4 * n], dtype="<f4").astype(np.float32)


class BandModel:
    """The learned ksw band MLP (gb_band_model_*): parameters live on the
    current device; train_step runs the hand-written gradient and Adam
    kernels; save / load keep the weights in a checksummed file."""

    def __init__(self, seed: int = 1):
        self._m = lib().gb_band_model_new(int(seed))
        if not self._m:
            raise GasalError("gb_band_model_new failed")
        self.n_params = lib().gb_band_param_count()

    @property
    def handle(self):
        return self._m

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        _check(lib().gb_band_model_params(self._m, out.ctypes.data, None), "gb_band_model_params")
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.n_params,)
        _check(lib().gb_band_model_params(self._m, None, p.ctypes.data), "gb_band_model_params")

    def predict(self, feat_ptr: int, n: int, out_ptr: int, stream: int = 0):
        _check(lib().gb_band_predict(self._m, feat_ptr, int(n), out_ptr, stream), "gb_band_predict")

    def grad(self, feat_ptr: int, label_ptr: int, n: int, tau: float, grad_ptr: int, loss_ptr: int, stream: int = 0):
        _check(lib().gb_band_grad(self._m, feat_ptr, label_ptr, int(n), float(tau), grad_ptr, loss_ptr, stream),
               "gb_band_grad")

    def train_step(self, feat_ptr: int, label_ptr: int, n: int, tau: float, lr: float, stream: int = 0) -> float:
        loss = C.c_float()
        _check(lib().gb_band_train_step(self._m, feat_ptr, label_ptr, int(n), float(tau), float(lr), stream,
                                        C.byref(loss)), "gb_band_train_step")
        return loss.value

    def save(self, path: str):
        with open(path, "wb") as f:
            f.write(band_blob(self.params(), lib().gb_band_feature_stride()))

    def load(self, path: str):
        with open(path, "rb") as f:
            self.set_params(band_unblob(f.read(), self.n_params, lib().gb_band_feature_stride()))

    def install(self, band_min: int = 16, band_max: int = 1024):
        _check(lib().gb_set_band_model(self._m, int(band_min), int(band_max)), "gb_set_band_model")

    @staticmethod
    def uninstall():
        _check(lib().gb_set_band_model(None, 0, 0), "gb_set_band_model")

    def close(self):
        if self._m:
            lib().gb_band_model_free(self._m)
            self._m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def band_features(dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray, feat_ptr: int, stream: int = 0):
    """gb_band_features: packs dev['q'/'t'] into dev['pq'/'pt'] and writes
    n x gb_band_feature_stride() floats at feat_ptr."""
    b, _ = _dev_structs(dev, h_q_len, h_t_len)
    _check(lib().gb_band_features(C.byref(b), feat_ptr, stream), "gb_band_features")


def ksw_band_align(p: Params, dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray, band_ptr: Optional[int],
                   ok_ptr: Optional[int] = None, stream: int = 0) -> dict:
    """gb_ksw_band_align: banded ksw with its certificate and the exact
    fallback; returns the band statistics (syncs the stream)."""
    b, o = _dev_structs(dev, h_q_len, h_t_len)
    cp = p.to_c()
    st = GbBandStats()
    _check(lib().gb_ksw_band_align(C.byref(cp), C.byref(b), C.byref(o), band_ptr, ok_ptr, stream, C.byref(st)),
           "gb_ksw_band_align")
    return {k: getattr(st, k) for k, _ in GbBandStats._fields_}


def ksw_align_max_off(p: Params, dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray, max_off_ptr: int,
                      stream: int = 0):
    """gb_ksw_align_max_off: the unbanded ksw with each pair's max_off (the
    largest |column - row| where the running maximum rose) in max_off_ptr."""
    b, o = _dev_structs(dev, h_q_len, h_t_len)
    cp = p.to_c()
    _check(lib().gb_ksw_align_max_off(C.byref(cp), C.byref(b), C.byref(o), max_off_ptr, stream),
           "gb_ksw_align_max_off")


def cigar_text_dev(cigar_ptr: int, q_off_ptr: int, n_cigar_ptr: int, n: int, text_ptr: int, stride: int,
                   text_len_ptr: int, stream_handle: int = 0):
    """gb_cigar_text on device buffers: forward CIGAR strings in stride-byte
    slots, lengths (-1: did not fit) in text_len."""
    _check(lib().gb_cigar_text(C.c_void_p(cigar_ptr), C.c_void_p(q_off_ptr), C.c_void_p(n_cigar_ptr), int(n),
                               C.c_void_p(text_ptr), int(stride), C.c_void_p(text_len_ptr), C.c_void_p(stream_handle)),
           "gb_cigar_text")


def pack_dev(ascii_ptr: int, nbytes: int, packed_ptr: int, stream_handle: int = 0):
    """The pack kernel alone on device buffers (gb_pack_dev)."""
    _check(lib().gb_pack_dev(C.c_void_p(ascii_ptr), nbytes, C.c_void_p(packed_ptr), C.c_void_p(stream_handle)),
           "gb_pack_dev")


def revcomp_dev(dev: dict, n: int, stream_handle: int = 0):
    """The reverse/complement kernel alone on a device batch's packed words
    (gb_revcomp_dev); dev holds pq, pt, q_off, t_off, q_len, t_len, q_op, t_op."""
    args = [C.c_void_p(dev.get(k)) for k in ("pq", "pt", "q_off", "t_off", "q_len", "t_len", "q_op", "t_op")]
    _check(lib().gb_revcomp_dev(*args, n, C.c_void_p(stream_handle)), "gb_revcomp_dev")


def align_dev(p: Params, dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray, stream_handle: int = 0,
              noalloc: bool = False):
    """Kernel-level call on device-resident buffers.  ``dev`` maps the
    gb_dev_batch_t / gb_dev_out_t field names to device addresses (ints).
    noalloc=True calls gb_align_dev_noalloc, which allocates nothing."""
    b, o = _dev_structs(dev, h_q_len, h_t_len)
    cp = p.to_c()
    if noalloc:
        _check(lib().gb_align_dev_noalloc(C.byref(cp), C.byref(b), C.byref(o), C.c_void_p(stream_handle)),
               "gb_align_dev_noalloc")
    else:
        _check(lib().gb_align_dev(C.byref(cp), C.byref(b), C.byref(o), C.c_void_p(stream_handle)),
               "gb_align_dev")


MIXED_MAX_KINDS = 8


def release_workspaces():
    """gb_release_workspaces: free the per-stream buffers the device-level
    entry points keep between calls (waits for the device first)."""
    _check(lib().gb_release_workspaces(), "gb_release_workspaces")



def _kinds_c(kinds):
    if not 1 <= len(kinds) <= MIXED_MAX_KINDS:
        raise GasalError(f"mixed dispatch takes 1..{MIXED_MAX_KINDS} kinds, got {len(kinds)}")
    arr = (GbParams * len(kinds))()
    for j, k in enumerate(kinds):
        arr[j] = k.to_c()
    return arr


def mixed_check(kinds, h_kind: np.ndarray, has_seed: bool = True) -> np.ndarray:
    """gb_mixed_check: the argument check of align_dev_mixed (no GPU needed);
    returns the pairs of each kind."""
    h_kind = np.ascontiguousarray(h_kind, dtype=np.uint8)
    arr = _kinds_c(kinds)
    counts = np.zeros(len(kinds), dtype=np.uint32)
    _check(lib().gb_mixed_check(arr, len(kinds), _ptr(h_kind), int(h_kind.shape[0]), int(bool(has_seed)),
                                _ptr(counts)), "gb_mixed_check")
    return counts


def align_dev_mixed(kinds, h_kind: np.ndarray, dev: dict, h_q_len: np.ndarray, h_t_len: np.ndarray,
                    stream_handle: int = 0):
    """gb_align_dev_mixed: pair i of the device batch (same ``dev`` map as
    align_dev) aligned under kinds[h_kind[i]]; the kinds run concurrently."""
    h_kind = np.ascontiguousarray(h_kind, dtype=np.uint8)
    b, o = _dev_structs(dev, h_q_len, h_t_len)
    arr = _kinds_c(kinds)
    _check(lib().gb_align_dev_mixed(arr, len(kinds), _ptr(h_kind), C.byref(b), C.byref(o),
                                    C.c_void_p(stream_handle)), "gb_align_dev_mixed")


class Streams:
    """GASAL2's stream storage vector: gasal_init_gpu_storage_v +
    gasal_init_streams (reference src/ctors.cpp:17-128)."""

    def __init__(self, n_streams: int, max_query_len: int, max_target_len: int, max_n_alns: int, params: Params):
        L = lib()
        self.params = params
        self._p = L.gasal_c_params_new()
        cp = params.to_c()
        _check(L.gasal_c_params_set(self._p, C.byref(cp)), "gasal_c_params_set")
        _check(L.gasal_c_copy_subst_scores(params.match, params.mismatch, params.gap_open, params.gap_extend),
               "gasal_copy_subst_scores")
        self._v = L.gasal_c_init_gpu_storage_v(n_streams)
        _check(L.gasal_c_init_streams(self._v, max_query_len, max_target_len, max_n_alns, self._p),
               "gasal_init_streams")
        self.n = n_streams
        self._views = []
        for i in range(n_streams):
            v = GbStorageView()
            _check(L.gasal_c_storage_view(L.gasal_c_storage(self._v, i), C.byref(v)), "gasal_c_storage_view")
            self._views.append(v)

    def storage(self, i: int):
        return lib().gasal_c_storage(self._v, i)

    def view(self, i: int) -> GbStorageView:
        v = GbStorageView()
        _check(lib().gasal_c_storage_view(self.storage(i), C.byref(v)), "gasal_c_storage_view")
        return v

    @staticmethod
    def _arr(ptr, ctype, n):
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,))

    def fill(self, i: int, b: Batch):
        """Stage a batch exactly as GASAL2 callers do: one
        gasal_host_batch_fill per sequence, then offsets / lengths / ops /
        seed scores written into the storage's pinned host arrays."""
        L = lib()
        s = self.storage(i)
        v = self.view(i)
        n = b.n
        if n > v.host_max_n_alns:
            raise GasalError("batch larger than max_n_alns")
        qoff = self._arr(v.host_query_batch_offsets, C.c_uint32, n)
        toff = self._arr(v.host_target_batch_offsets, C.c_uint32, n)
        qi = ti = 0
        qbuf, tbuf = b.q.ctypes.data, b.t.ctypes.data
        for k in range(n):
            qoff[k] = qi
            toff[k] = ti
            qi = L.gasal_c_host_batch_fill(s, qi, C.c_char_p(qbuf + int(b.q_off[k])), int(b.q_len[k]), QUERY)
            ti = L.gasal_c_host_batch_fill(s, ti, C.c_char_p(tbuf + int(b.t_off[k])), int(b.t_len[k]), TARGET)
        self._arr(v.host_query_batch_lens, C.c_uint32, n)[:] = b.q_len
        self._arr(v.host_target_batch_lens, C.c_uint32, n)[:] = b.t_len
        zeros = np.zeros(n, dtype=np.uint8)
        _check(L.gasal_c_op_fill(s, _ptr(b.q_op if b.q_op is not None else zeros), n, QUERY), "gasal_op_fill")
        _check(L.gasal_c_op_fill(s, _ptr(b.t_op if b.t_op is not None else zeros), n, TARGET), "gasal_op_fill")
        if self.params.algo == KSW:
            self._arr(v.host_seed_scores, C.c_uint32, n)[:] = b.seed if b.seed is not None else 0
        return qi, ti

    def fill_fast(self, i: int, b: Batch):
        """Stage a batch whose layout already is GASAL2's (padded, offsets
        ascending) with one gasal_host_batch_fill per side: the whole padded
        buffer is one multiple-of-8 "sequence", so nothing is padded and the
        page's data size (what gasal_aln_async copies) covers all of it."""
        L = lib()
        s = self.storage(i)
        v = self.view(i)
        n = b.n
        nq, nt = int(b.q.shape[0]), int(b.t.shape[0])
        if nq % 8 or nt % 8:
            raise GasalError("fill_fast needs 8-byte padded buffers")
        qi = L.gasal_c_host_batch_fill(s, 0, C.c_char_p(b.q.ctypes.data), nq, QUERY)
        ti = L.gasal_c_host_batch_fill(s, 0, C.c_char_p(b.t.ctypes.data), nt, TARGET)
        if qi != nq or ti != nt:
            raise GasalError("host page smaller than the batch; create the storage with larger maxima or use fill()")
        self._arr(v.host_query_batch_offsets, C.c_uint32, n)[:] = b.q_off
        self._arr(v.host_target_batch_offsets, C.c_uint32, n)[:] = b.t_off
        self._arr(v.host_query_batch_lens, C.c_uint32, n)[:] = b.q_len
        self._arr(v.host_target_batch_lens, C.c_uint32, n)[:] = b.t_len
        zeros = np.zeros(n, dtype=np.uint8)
        _check(L.gasal_c_op_fill(s, _ptr(b.q_op if b.q_op is not None else zeros), n, QUERY), "gasal_op_fill")
        _check(L.gasal_c_op_fill(s, _ptr(b.t_op if b.t_op is not None else zeros), n, TARGET), "gasal_op_fill")
        if self.params.algo == KSW:
            self._arr(v.host_seed_scores, C.c_uint32, n)[:] = b.seed if b.seed is not None else 0
        return qi, ti

    def fill_bulk(self, i: int, b: Batch, threads: int = 0):
        """fill_fast with the sequence copies split over host threads
        (gasal_c_host_batch_fill_mt; 0 = every hardware thread)."""
        L = lib()
        s = self.storage(i)
        v = self.view(i)
        n = b.n
        nq, nt = int(b.q.shape[0]), int(b.t.shape[0])
        if nq % 8 or nt % 8:
            raise GasalError("fill_bulk needs 8-byte padded buffers")
        _check(L.gasal_c_host_batch_reset(s), "gasal_host_batch_reset")
        qi = L.gasal_c_host_batch_fill_mt(s, 0, b.q.ctypes.data, nq, QUERY, threads)
        ti = L.gasal_c_host_batch_fill_mt(s, 0, b.t.ctypes.data, nt, TARGET, threads)
        if qi != nq or ti != nt:
            raise GasalError("host page smaller than the batch; create the storage with larger maxima or use fill()")
        self._arr(v.host_query_batch_offsets, C.c_uint32, n)[:] = b.q_off
        self._arr(v.host_target_batch_offsets, C.c_uint32, n)[:] = b.t_off
        self._arr(v.host_query_batch_lens, C.c_uint32, n)[:] = b.q_len
        self._arr(v.host_target_batch_lens, C.c_uint32, n)[:] = b.t_len
        zeros = np.zeros(n, dtype=np.uint8)
        _check(L.gasal_c_op_fill(s, _ptr(b.q_op if b.q_op is not None else zeros), n, QUERY), "gasal_op_fill")
        _check(L.gasal_c_op_fill(s, _ptr(b.t_op if b.t_op is not None else zeros), n, TARGET), "gasal_op_fill")
        if self.params.algo == KSW:
            self._arr(v.host_seed_scores, C.c_uint32, n)[:] = b.seed if b.seed is not None else 0
        return qi, ti

    def aln_async(self, i: int, qbytes: int, tbytes: int, n: int):
        _check(lib().gasal_c_aln_async(self.storage(i), qbytes, tbytes, n, self._p), "gasal_aln_async")

    def is_done(self, i: int) -> int:
        rc = lib().gasal_c_is_aln_async_done(self.storage(i))
        if rc not in (0, -1, -2):
            raise GasalError(f"gasal_is_aln_async_done: {GB_STATUS.get(rc, rc)}")
        return rc

    def wait(self, i: int):
        while self.is_done(i) == -1:
            pass

    def results(self, i: int, n: int, b: Optional[Batch] = None) -> dict:
        v = self.view(i)
        p = self.params
        d = {}
        def get(name, ptr, ct=C.c_int32):
            if ptr:
                d[name] = self._arr(ptr, ct, n).copy()
        get("score", v.aln_score)
        get("q_end", v.query_batch_end)
        get("t_end", v.target_batch_end)
        get("q_start", v.query_batch_start)
        get("t_start", v.target_batch_start)
        if p.second_best:
            get("score2", v.aln_score2)
            get("q_end2", v.query_batch_end2)
            get("t_end2", v.target_batch_end2)
        if p.start_pos == WITH_TB:
            get("n_cigar", v.n_cigar_ops, C.c_uint32)
            if b is not None and v.cigar:
                d["cigar"] = self._arr(v.cigar, C.c_uint8, int(b.q.shape[0])).copy()
        return d

    def close(self):
        if self._v:
            L = lib()
            L.gasal_c_destroy_streams(self._v, self._p)
            L.gasal_c_destroy_gpu_storage_v(self._v)
            L.gasal_c_params_free(self._p)
            self._v = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
