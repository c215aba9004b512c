"""ksw on the warp-per-pair kernel (ksw_wc.cu) against the oracle and the
one-thread kernel: every tile count (queries up to 2046 bases), the compare
scorer (IUPAC codes, scores beyond a byte), z-drop, empty sequences, and the
pairs the warp kernel hands back (longer queries, seed scores past its key
range)."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Batch, Params, KSW
from oracle.bindings import oracle_align

pytestmark = pytest.mark.gpu


def _check(p, b, what=""):
    got = gl.align(p, b).as_dict(p)
    exp = oracle_align(p, b).as_dict(p)
    for k, v in exp.items():
        bad = np.nonzero(got[k] != v)[0]
        assert len(bad) == 0, f"{what} {p.key()} {k}: {len(bad)} differ, first {bad[:5]} got {got[k][bad[:5]]} " \
                              f"want {v[bad[:5]]}"
    return got


@pytest.fixture(autouse=True)
def _warp_on():
    saved = gl.get_tuning()
    gl.set_tuning(ksw_warp=1)
    yield
    gl.set_tuning(**saved)


@pytest.mark.parametrize("zdrop", [0, 100, 5])
def test_workload3_all_tile_counts(zdrop):
    """250-2000 bp: 2, 4 and 8 tiles in one launch."""
    b = W.workload3(3000, seed=90 + zdrop)
    _check(Params(algo=KSW, zdrop=zdrop), b)


def test_short_pairs_one_tile():
    b = W.workload0(3000, seed=91)
    b.seed = np.random.default_rng(91).integers(0, 61, b.n).astype(np.uint32)
    _check(Params(algo=KSW), b)
    _check(Params(algo=KSW, zdrop=10), b)


def test_warp_equals_one_thread_kernel():
    b = W.workload3(1500, seed=92)
    p = Params(algo=KSW, zdrop=100)
    warp = gl.align(p, b).as_dict(p)
    gl.set_tuning(ksw_warp=0)
    one = gl.align(p, b).as_dict(p)
    for k in warp:
        assert np.array_equal(warp[k], one[k]), k


def test_compare_scorer_iupac_and_wide_scores():
    rng = np.random.default_rng(93)
    qs, ts = [], []
    for i in range(600):
        n = int(rng.integers(1, 700))
        alpha = b"ACGTNRYKM" if i % 2 else b"ACGT"
        q = bytes(np.frombuffer(alpha, np.uint8)[rng.integers(0, len(alpha), n)])
        t = bytearray(q)
        for _ in range(n // 20 + 1):
            t[int(rng.integers(0, len(t)))] = alpha[int(rng.integers(0, len(alpha)))]
        qs.append(q)
        ts.append(bytes(t) + bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(rng.integers(0, 30)))]))
    b = Batch.from_seqs(qs, ts, seed=rng.integers(0, 61, len(qs)))
    _check(Params(algo=KSW), b, "iupac")
    _check(Params(algo=KSW, match=200, mismatch=300, gap_open=250, gap_extend=30, zdrop=500), b, "wide")


def test_handed_back_pairs():
    """Queries past 2046 bases and seed scores past the key range go to the
    one-thread kernel in the same call; the rest stay on the warp kernel."""
    rng = np.random.default_rng(94)
    qs, ts, seeds = [], [], []
    for i in range(300):
        n = int(rng.integers(2040, 2300)) if i % 3 == 0 else int(rng.integers(100, 900))
        q = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)])
        t = bytearray(q)
        for _ in range(n // 25):
            t[int(rng.integers(0, len(t)))] = b"ACGT"[int(rng.integers(0, 4))]
        qs.append(q)
        ts.append(bytes(t))
        seeds.append(600000 if i % 7 == 0 else int(rng.integers(20, 61)))
    b = Batch.from_seqs(qs, ts, seed=np.array(seeds, dtype=np.uint32))
    _check(Params(algo=KSW), b)
    _check(Params(algo=KSW, zdrop=100), b)


def test_empty_sequences():
    qs = [b"", b"ACGTACGT", b"", b"ACGTTGCA" * 40, b"A"]
    ts = [b"ACGT", b"", b"", b"ACGTTGCA" * 38, b"A"]
    b = Batch.from_seqs(qs * 700, ts * 700, seed=np.arange(3500, dtype=np.uint32) % 61)
    got = _check(Params(algo=KSW), b)
    assert got["score"][0] == 0 and got["score"][2] == 2  # the seed score comes back unchanged


def test_scores_near_the_16_bit_row_limit():
    """H and E are stored as 16-bit halves: pairs whose seed + match * qlen
    reaches 2^15 are handed to the one-thread kernel, the rest stay; both
    sides of the limit must match the oracle."""
    rng = np.random.default_rng(95)
    qs, ts, seeds = [], [], []
    for i in range(400):
        n = int(rng.integers(1500, 1700))
        q = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)])
        t = bytearray(q)
        for _ in range(n // 50):
            t[int(rng.integers(0, len(t)))] = b"ACGT"[int(rng.integers(0, 4))]
        qs.append(q)
        ts.append(bytes(t))
        seeds.append(int(rng.integers(0, 2000)))
    b = Batch.from_seqs(qs, ts, seed=np.array(seeds, dtype=np.uint32))
    _check(Params(algo=KSW, match=20, mismatch=30, gap_open=40, gap_extend=5), b)


def test_long_class_columns_past_4095():
    """Queries of 4,100-8,190 bases run in the 8192-column length class; the
    row maximum's key must carry columns past 4095 (near-identical pairs
    put the maximum in the last columns)."""
    rng = np.random.default_rng(96)
    qs, ts, seeds = [], [], []
    for i in range(90):
        n = int(rng.integers(4100, 8191)) if i % 3 else int(rng.integers(4100, 4400))
        q = bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)])
        t = bytearray(q)
        for _ in range(n // 200):
            t[int(rng.integers(0, len(t)))] = b"ACGT"[int(rng.integers(0, 4))]
        qs.append(q)
        ts.append(bytes(t) + bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(rng.integers(0, 40)))]))
        seeds.append(int(rng.integers(20, 61)))
    b = Batch.from_seqs(qs, ts, seed=np.array(seeds, dtype=np.uint32))
    got = _check(Params(algo=KSW, zdrop=100), b)
    assert int((got["q_end"] > 4096).sum()) > 45  # the maxima sit past column 4096
    _check(Params(algo=KSW), b)
