"""NumPy restatements of the learned-band feature and MLP kernels
(gasal_b200/csrc/mlband.cu), used by the tests as their checker: the
11-mer diagonal histogram (integer work, compared exactly) and the MLP
forward pass and pinball-loss gradient (FP32, compared with tolerances)."""
import numpy as np

K = 11
FEATS, STRIDE, H = 67, 68, 64
CODE2 = {1: 0, 3: 1, 7: 2, 4: 3}


def _kmers(codes):
    """(start, kmer) for every window of 11 valid bases."""
    out = []
    k, valid = 0, 0
    for p, c in enumerate(codes):
        b = CODE2.get(int(c), 4)
        valid = valid + 1 if b < 4 else 0
        k = ((k << 2) | (b & 3)) & ((1 << 22) - 1)
        if valid >= K:
            out.append((p - K + 1, k))
    return out


def _slot(k):
    return ((k * 2654435761) & 0xFFFFFFFF) >> 20


def _bin(d):
    a = abs(d)
    if a < 8:
        b = a
    else:
        e = a.bit_length() - 1
        b = min(31, 8 + 4 * (e - 3) + ((a >> (e - 2)) & 3))
    return 32 + b if d < 0 else b


def features(b):
    """n x 68 float32, as band_feature_kernel writes them."""
    out = np.zeros((b.n, STRIDE), dtype=np.float32)
    for i in range(b.n):
        q = b.q[b.q_off[i]:b.q_off[i] + b.q_len[i]] & 0x0F
        t = b.t[b.t_off[i]:b.t_off[i] + b.t_len[i]] & 0x0F
        tab = {}
        for pos, k in _kmers(t):
            s = _slot(k)
            tab[s] = max(tab.get(s, 0), ((k + 1) << 32) | pos)
        hist = np.zeros(64, dtype=np.int64)
        for pos, k in _kmers(q):
            v = tab.get(_slot(k), 0)
            if (v >> 32) == k + 1:
                hist[_bin(int(v & 0xFFFFFFFF) - pos)] += 1
        nq = int(b.q_len[i]) - K + 1
        inv = np.float32(1.0) / np.float32(nq) if nq > 0 else np.float32(0.0)
        out[i, 3:67] = hist.astype(np.float32) * inv
        out[i, 0] = np.float32(b.q_len[i]) * np.float32(1 / 1024)
        out[i, 1] = np.float32(b.t_len[i]) * np.float32(1 / 1024)
        out[i, 2] = np.float32(int(b.t_len[i]) - int(b.q_len[i])) * np.float32(1 / 128)
    return out


def unpack(p):
    o = 0
    W1 = p[o:o + H * FEATS].reshape(H, FEATS); o += H * FEATS
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def bf16(x):
    """round-to-nearest-even to bfloat16, back to float32"""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p.astype(np.float64))
    x = x[:, :FEATS].astype(np.float64)
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3 + b3, (x, h1, h2)


def grad(p, x, y, tau):
    """gradient of mean pinball loss, and the loss sum"""
    W1, b1, W2, b2, W3, b3 = unpack(p.astype(np.float64))
    out, (x, h1, h2) = forward(p, x)
    r = y.astype(np.float64) - out
    loss = np.sum(np.where(r > 0, tau * r, (tau - 1) * r))
    dy = np.where(r > 0, -tau, 1 - tau) / len(y)
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = (dy[:, None] * W3[None, :]) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return g, loss
