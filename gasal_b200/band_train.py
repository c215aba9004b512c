"""Training the learned ksw band (no reference counterpart).

Labels: labels_max_off() takes them from the plain (unbanded) ksw's own
max_off -- the largest |column - row| where its running maximum rose, as
ksw_extend2 tracks it -- plus a margin; labels() from the banded kernel
itself: log2 of the narrowest band in a ladder whose result the certificate
keeps (log2(2048) when none does).  The model is trained with the pinball loss at quantile tau
(tau > 0.5 prefers bands a little wider than needed: a refused band costs a
full recomputation, a wider one only a few more columns).

Everything runs on the current CUDA device through the C ABI; torch only
holds the device buffers.
"""
from __future__ import annotations

import numpy as np

from . import lib as gl
from .capi import Batch, Params

# the widest band of each warp-kernel tile cost (a banded row spans at most
# 2w + 8 columns: one 64- or 128-column tile, then whole 256-column tiles)
LADDER = (28, 60, 124, 252, 380, 508, 636, 764, 892, 1020)
NO_BAND = 11.0  # log2(2048): no ladder band was kept


def ladder_label(k: int) -> float:
    """Label of ladder rung k: the middle of the log2 interval of predictions
    that widths_from_pred maps to that rung (from 16, the narrowest band, for
    the first), so a prediction off by less than half an interval still
    lands on the rung."""
    lo = np.log2(16.0) if k == 0 else np.log2(LADDER[k - 1])
    return float(0.5 * (lo + np.log2(LADDER[k])))


class DeviceBatch:
    """A Batch copied to the device, with the gb_dev_batch_t / gb_dev_out_t
    address map the C ABI wrappers take."""

    def __init__(self, torch, b: Batch, dev, outs=("score", "q_end", "t_end")):
        def t_(a, dt=None):
            return torch.from_numpy(np.ascontiguousarray(a).view(dt or a.dtype)).to(dev)
        self.b = b
        self.keep = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
                     "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32),
                     "pq": torch.zeros(b.q.shape[0] // 8, dtype=torch.int32, device=dev),
                     "pt": torch.zeros(b.t.shape[0] // 8, dtype=torch.int32, device=dev)}
        if b.seed is not None:
            self.keep["seed"] = t_(b.seed, np.int32)
        for k in outs:
            self.keep["out_" + k] = torch.zeros(b.n, dtype=torch.int32, device=dev)
        m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0]}
        for k, src in (("q", "q"), ("t", "t"), ("pq", "pq"), ("pt", "pt"), ("q_off", "qo"), ("t_off", "to"),
                       ("q_len", "ql"), ("t_len", "tl"), ("seed", "seed")):
            if src in self.keep:
                m[k] = self.keep[src].data_ptr()
        for k in outs:
            m["out_" + k] = self.keep["out_" + k].data_ptr()
        self.map = m

    def out(self, k):
        return self.keep["out_" + k]


def features(torch, db: DeviceBatch, stream: int = 0):
    stride = gl.lib().gb_band_feature_stride()
    f = torch.zeros((db.b.n, stride), dtype=torch.float32, device=db.keep["q"].device)
    gl.band_features(db.map, db.b.q_len, db.b.t_len, f.data_ptr(), stream)
    return f


def labels(torch, p: Params, db: DeviceBatch, ladder=LADDER, stream: int = 0) -> np.ndarray:
    """The label (ladder_label) of the narrowest ladder band the certificate
    keeps, per pair; NO_BAND when none does."""
    n = db.b.n
    dev = db.keep["q"].device
    lab = np.full(n, NO_BAND, dtype=np.float32)
    done = np.zeros(n, dtype=bool)
    ok = torch.zeros(n, dtype=torch.uint8, device=dev)
    for k, w in enumerate(ladder):
        band = torch.full((n,), int(w), dtype=torch.int32, device=dev)
        gl.ksw_band_align(p, db.map, db.b.q_len, db.b.t_len, band.data_ptr(), ok.data_ptr(), stream)
        kept = ok.cpu().numpy().astype(bool)
        new = kept & ~done
        lab[new] = ladder_label(k) if tuple(ladder) == LADDER else np.log2(w)
        done |= kept
    return lab


MAX_OFF_MARGIN = 16  # diagonals added to max_off: the certificate needs room beside the path


def labels_max_off(torch, p: Params, db: DeviceBatch, margin: int = MAX_OFF_MARGIN, stream: int = 0):
    """log2(max_off + margin) per pair, max_off from the plain (unbanded) ksw
    itself: the largest |column - row| over the cells where its running
    maximum rose -- how far from the main diagonal the alignment reached.
    Returns (labels, max_off)."""
    dev = db.keep["q"].device
    mo = torch.zeros(db.b.n, dtype=torch.int32, device=dev)
    gl.ksw_align_max_off(p, db.map, db.b.q_len, db.b.t_len, mo.data_ptr(), stream)
    torch.cuda.synchronize()
    m = mo.cpu().numpy()
    return np.log2(m.astype(np.float64) + margin).astype(np.float32), m


def widths_from_pred(pred: np.ndarray, q_len: np.ndarray, t_len: np.ndarray, bmin: int = 16,
                     bmax: int = 1024) -> np.ndarray:
    """The per-pair half-widths the library derives from predictions
    (band_from_pred_kernel): ceil(2^y) clamped to [bmin, bmax], widened to
    the widest band of the same warp-kernel tile cost (2w + 8 columns in one
    64- or 128-column tile, or whole 256-column tiles), -1 (unbanded) where
    the band covers the matrix."""
    y = np.clip(np.asarray(pred, dtype=np.float32), 0, 20)
    w = np.ceil(np.exp2(y)).astype(np.int64)
    w = np.clip(w, bmin, bmax)
    span = 2 * w + 8
    w = np.where(span <= 64, 28, np.where(span <= 128, 60, 128 * ((span + 255) // 256) - 4))
    w = np.minimum(w, bmax)
    cover = np.maximum(q_len, t_len).astype(np.int64)
    return np.where(w >= cover, -1, w).astype(np.int32)


def train(torch, model: "gl.BandModel", feat, lab: np.ndarray, steps: int = 400, batch: int = 8192,
          tau: float = 0.8, lr: float = 3e-3, seed: int = 0, stream: int = 0) -> list:
    """Adam on random mini-batches; returns the loss trace."""
    dev = feat.device
    y = torch.from_numpy(np.ascontiguousarray(lab, dtype=np.float32)).to(dev)
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = feat.shape[0]
    trace = []
    for _ in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), generator=g).to(dev)
        fb = feat.index_select(0, idx).contiguous()
        yb = y.index_select(0, idx).contiguous()
        trace.append(model.train_step(fb.data_ptr(), yb.data_ptr(), fb.shape[0], tau, lr, stream))
    return trace
