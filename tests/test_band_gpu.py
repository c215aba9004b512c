"""Learned ksw band on the GPU: feature kernel (exact against the NumPy
checker), MLP forward (BF16 weights, FP32 accumulation: 1e-3 relative) and
pinball-loss gradient (FP32 atomics: 1e-3 relative + 1e-6 absolute) against
NumPy, a training run that lowers the loss, and the band certificate: for
every band width every result -- kept banded or recomputed -- must equal the
unbanded oracle bit for bit."""
import numpy as np
import pytest

import band_ref as R
from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, KSW
from oracle.bindings import oracle_align

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda", 0)
OUTS = ("score", "q_end", "t_end")


def _dev(b):
    def t_(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt or a.dtype)).to(DEV)
    keep = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
            "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32), "seed": t_(b.seed, np.int32),
            "pq": torch.zeros(b.q.shape[0] // 8, dtype=torch.int32, device=DEV),
            "pt": torch.zeros(b.t.shape[0] // 8, dtype=torch.int32, device=DEV)}
    for k in OUTS:
        keep[k] = torch.full((b.n,), -7, dtype=torch.int32, device=DEV)
    m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0], "seed": keep["seed"].data_ptr()}
    for k, src in (("q", "q"), ("t", "t"), ("pq", "pq"), ("pt", "pt"), ("q_off", "qo"), ("t_off", "to"),
                   ("q_len", "ql"), ("t_len", "tl")):
        m[k] = keep[src].data_ptr()
    for k in OUTS:
        m["out_" + k] = keep[k].data_ptr()
    return m, keep


def _stream():
    return torch.cuda.current_stream().cuda_stream


def test_features_exact():
    b = W.workload3(60, seed=120)
    m, keep = _dev(b)
    feat = torch.zeros((b.n, 68), dtype=torch.float32, device=DEV)
    gl.band_features(m, b.q_len, b.t_len, feat.data_ptr(), _stream())
    torch.cuda.synchronize()
    got = feat.cpu().numpy()
    exp = R.features(b)
    assert np.array_equal(got, exp), np.argwhere(got != exp)[:5]


def test_forward_and_gradient_match_numpy():
    rng = np.random.default_rng(121)
    model = gl.BandModel(seed=5)
    p = model.params()
    p = p + rng.normal(0, 0.05, p.shape).astype(np.float32)
    model.set_params(p)
    n = 333
    x = np.abs(rng.normal(0, 0.5, (n, 68))).astype(np.float32)
    x[:, 67] = 0
    y = rng.normal(6, 1.5, n).astype(np.float32)
    xd, yd = torch.from_numpy(x).to(DEV), torch.from_numpy(y).to(DEV)
    out = torch.zeros(n, dtype=torch.float32, device=DEV)
    model.predict(xd.data_ptr(), n, out.data_ptr(), _stream())
    g = torch.zeros(model.n_params, dtype=torch.float32, device=DEV)
    loss = torch.zeros(1, dtype=torch.float32, device=DEV)
    model.grad(xd.data_ptr(), yd.data_ptr(), n, 0.9, g.data_ptr(), loss.data_ptr(), _stream())
    torch.cuda.synchronize()
    exp_out, _ = R.forward(R.bf16(p), x)
    assert np.allclose(out.cpu().numpy(), exp_out, rtol=1e-3, atol=1e-3)
    exp_g, exp_loss = R.grad(p, x, y, 0.9)
    got_g = g.cpu().numpy()
    assert np.allclose(got_g, exp_g, rtol=1e-3, atol=1e-6), np.max(np.abs(got_g - exp_g))
    assert abs(loss.item() - exp_loss) < 1e-3 * abs(exp_loss) + 1e-4
    model.close()


def test_training_lowers_the_loss():
    rng = np.random.default_rng(122)
    model = gl.BandModel(seed=6)
    n = 4096
    x = np.abs(rng.normal(0, 0.5, (n, 68))).astype(np.float32)
    y = (4 + 3 * x[:, 0] + 2 * x[:, 5]).astype(np.float32)
    xd, yd = torch.from_numpy(x).to(DEV), torch.from_numpy(y).to(DEV)
    first = model.train_step(xd.data_ptr(), yd.data_ptr(), n, 0.5, 1e-2, _stream())
    for _ in range(300):
        last = model.train_step(xd.data_ptr(), yd.data_ptr(), n, 0.5, 1e-2, _stream())
    assert last < 0.25 * first, (first, last)
    model.close()


@pytest.mark.parametrize("zdrop", [0, 100])
def test_band_certificate_never_changes_a_result(zdrop):
    """Every band width from 0 to beyond the matrix: the kept banded results
    and the recomputed ones together equal the unbanded oracle."""
    b = W.workload3(1200, seed=123 + zdrop)
    p = Params(algo=KSW, zdrop=zdrop)
    exp = oracle_align(p, b).as_dict(p)
    m, keep = _dev(b)
    kept = {}
    for w in (0, 8, 24, 64, 128, 256, 512, 4096):
        for k in OUTS:
            keep[k].fill_(-7)
        band = torch.full((b.n,), w, dtype=torch.int32, device=DEV)
        ok = torch.zeros(b.n, dtype=torch.uint8, device=DEV)
        st = gl.ksw_band_align(p, m, b.q_len, b.t_len, band.data_ptr(), ok.data_ptr(), _stream())
        for k in OUTS:
            got = keep[k].cpu().numpy()
            bad = np.nonzero(got != exp[k])[0]
            assert len(bad) == 0, f"w={w} {k}: {len(bad)} differ, first {bad[:5]}"
        assert st["accepted"] + st["retried"] + st["handed_back"] == b.n
        assert int(ok.sum().item()) == st["accepted"] + st["handed_back"]
        kept[w] = st["accepted"]
    assert kept[4096] == b.n          # a band wider than every matrix keeps everything
    assert kept[0] < kept[512]        # and narrow bands are refused more often


@pytest.mark.parametrize("zdrop", [0, 100])
def test_max_off_matches_oracle(zdrop):
    """gb_ksw_align_max_off: the unbanded results and each pair's max_off
    (largest |column - row| where the running maximum rose) equal the
    oracle's, on the warp kernel and on pairs it hands to the one-thread
    kernel (seed scores of 2^15 and more)."""
    b = W.workload3(1200, seed=125 + zdrop)
    b.seed = b.seed.copy()
    b.seed[::97] = 40000  # seed + match*qlen >= 2^15: the one-thread kernel's pairs
    p = Params(algo=KSW, zdrop=zdrop)
    r = oracle_align(p, b)
    exp = r.as_dict(p)
    m, keep = _dev(b)
    mo = torch.full((b.n,), -7, dtype=torch.int32, device=DEV)
    gl.ksw_align_max_off(p, m, b.q_len, b.t_len, mo.data_ptr(), _stream())
    torch.cuda.synchronize()
    for k in OUTS:
        assert np.array_equal(keep[k].cpu().numpy(), exp[k]), k
    got = mo.cpu().numpy()
    bad = np.nonzero(got != r.score2)[0]
    assert len(bad) == 0, f"{len(bad)} max_off differ, first {bad[:5]}: {got[bad[:5]]} vs {r.score2[bad[:5]]}"
    assert got.max() > 0


def test_installed_model_path_matches_oracle():
    b = W.workload3(800, seed=124)
    p = Params(algo=KSW, zdrop=100)
    model = gl.BandModel(seed=7)
    try:
        model.install(16, 512)
        got = gl.align(p, b).as_dict(p)
    finally:
        gl.BandModel.uninstall()
        model.close()
    exp = oracle_align(p, b).as_dict(p)
    for k in OUTS:
        assert np.array_equal(got[k], exp[k]), k


def test_trained_band_beats_a_fixed_band_of_the_same_width():
    """What the trained network gains over the banded method without it: on
    held-out pairs its per-pair bands keep more banded results (fewer exact
    recomputations) and compute fewer cells than one fixed band of the same
    mean width -- and every result still equals the oracle."""
    from gasal_b200 import band_train as BT
    p = Params(algo=KSW, zdrop=100)
    tb = W.workload3(16000, seed=130)
    tdb = BT.DeviceBatch(torch, tb, DEV)
    feat = BT.features(torch, tdb)
    lab = BT.labels(torch, p, tdb)
    model = gl.BandModel(seed=13)
    BT.train(torch, model, feat, lab, steps=400, batch=4096, tau=0.8, lr=3e-3)
    eb = W.workload3(12000, seed=131)
    edb = BT.DeviceBatch(torch, eb, DEV)
    ef = BT.features(torch, edb)
    pred = torch.zeros(eb.n, dtype=torch.float32, device=DEV)
    model.predict(ef.data_ptr(), eb.n, pred.data_ptr(), _stream())
    torch.cuda.synchronize()
    model.close()
    # the same transform as band_from_pred_kernel
    learned = BT.widths_from_pred(pred.cpu().numpy(), eb.q_len, eb.t_len)
    cover = np.maximum(eb.q_len, eb.t_len).astype(np.int64)
    mean_w = int(np.mean(np.where(learned < 0, cover, learned)))
    fixed = np.full(eb.n, (mean_w + 7) & ~7, np.int32)
    exp = oracle_align(p, eb).as_dict(p)
    stats = {}
    for name, band in (("learned", learned), ("fixed", fixed)):
        bt = torch.from_numpy(band).to(DEV)
        for k in OUTS:
            edb.out(k).fill_(-7)
        stats[name] = gl.ksw_band_align(p, edb.map, eb.q_len, eb.t_len, bt.data_ptr(), None, _stream())
        for k in OUTS:
            assert np.array_equal(edb.out(k).cpu().numpy(), exp[k]), (name, k)
    kept = {k: v["accepted"] / eb.n for k, v in stats.items()}
    assert kept["learned"] > kept["fixed"] + 0.03, (kept, mean_w)
    assert stats["learned"]["cells"] < stats["fixed"]["cells"], stats


def test_band_model_save_load_gives_the_same_weights(tmp_path):
    torch = pytest.importorskip("torch")
    from gasal_b200 import lib as gl
    a = gl.BandModel(seed=5)
    b = gl.BandModel(seed=6)
    assert not np.array_equal(a.params(), b.params())
    path = str(tmp_path / "band.bin")
    a.save(path)
    b.load(path)
    assert np.array_equal(a.params(), b.params())
    a.close()
    b.close()
