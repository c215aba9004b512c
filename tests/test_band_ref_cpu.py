"""The NumPy checker of the learned-band kernels, checked itself: its
pinball-loss gradient against central finite differences (float64), its
diagonal binning against the documented bin edges, and its features on a
hand-made pair."""
import numpy as np

import band_ref as R
from gasal_b200.capi import Batch


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    n_par = R.H * R.FEATS + R.H + R.H * R.H + R.H + R.H + 1
    p = rng.normal(0, 0.3, n_par)
    x = np.abs(rng.normal(0, 1, (40, R.STRIDE)))
    y = rng.normal(5, 2, 40)
    g, _ = R.grad(p, x, y, 0.9)
    idx = rng.choice(n_par, 60, replace=False)
    for i in idx:
        e = np.zeros(n_par)
        e[i] = 1e-6
        lp = R.grad(p + e, x, y, 0.9)[1] / len(y)
        lm = R.grad(p - e, x, y, 0.9)[1] / len(y)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) < 1e-5 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_diagonal_bins():
    assert [R._bin(d) for d in range(0, 8)] == list(range(8))
    assert R._bin(8) == 8 and R._bin(15) == 11 and R._bin(16) == 12 and R._bin(31) == 15
    assert R._bin(511) == 31 and R._bin(100000) == 31
    assert R._bin(-1) == 33 and R._bin(-16) == 44


def test_features_of_a_shifted_copy():
    rng = np.random.default_rng(4)
    q = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 60)])
    t = b"GG" + q                                    # every 11-mer of q sits 2 to the right
    f = R.features(Batch.from_seqs([q], [t]))
    nq = len(q) - 10
    assert round(float(f[0, 3 + 2]) * nq) == nq      # all in the d = +2 bin
    assert abs(f[0, 0] - len(q) / 1024) < 1e-7 and abs(f[0, 2] - 2 / 128) < 1e-7


def test_band_model_blob_round_trip_and_checksum():
    """The weights file: round trip, and every corruption is refused."""
    import numpy as np
    import pytest
    from gasal_b200 import lib as gl
    n, stride = gl.lib().gb_band_param_count(), gl.lib().gb_band_feature_stride()
    p = np.random.default_rng(3).standard_normal(n).astype(np.float32)
    blob = gl.band_blob(p, stride)
    assert np.array_equal(gl.band_unblob(blob, n, stride), p)
    flipped = bytearray(blob)
    flipped[40] ^= 0x01
    with pytest.raises(gl.GasalError, match="checksum"):
        gl.band_unblob(bytes(flipped), n, stride)
    with pytest.raises(gl.GasalError, match="magic"):
        gl.band_unblob(b"XX" + blob[2:], n, stride)
    with pytest.raises(gl.GasalError):
        gl.band_unblob(blob[:-8], n, stride)
    with pytest.raises(gl.GasalError, match="parameters"):
        gl.band_unblob(gl.band_blob(p[:-1], stride), n, stride)
