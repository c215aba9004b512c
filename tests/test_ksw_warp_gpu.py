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


def _short_mixed(n, seed):
    """Queries of 1-300 bases (most of them on lane groups, 31 words or fewer,
    the rest on the 32-lane kernel), related and unrelated targets of 0-400
    bases, N runs and IUPAC codes in some pairs, seeds 0-60 and a few of
    40000 (handed back to the one-thread kernel)."""
    rng = np.random.default_rng(seed)
    qs, ts, h0 = [], [], []
    for k in range(n):
        ql = int(rng.integers(1, 300)) if k % 11 else 0
        q = bytearray(rng.choice(list(b"ACGT"), size=ql).tolist())
        if k % 3 == 0:
            t = bytearray(rng.choice(list(b"ACGT"), size=int(rng.integers(0, 400))).tolist())
        else:
            t = bytearray(q)
            for _ in range(int(rng.integers(0, 8))):
                if not t:
                    break
                a = int(rng.integers(0, len(t)))
                if rng.random() < 0.5:
                    del t[a:a + int(rng.integers(1, 5))]
                else:
                    t[a:a] = bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(1, 5))).tolist())
            t += bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(0, 60))).tolist())
        if k % 7 == 1 and len(q) > 10:
            q[3:6] = b"NNN"
        if k % 13 == 2 and len(t) > 10:
            t[4] = ord("R")
        qs.append(bytes(q))
        ts.append(bytes(t))
        h0.append(40000 if k % 97 == 5 else int(rng.integers(0, 61)))
    return Batch.from_seqs(qs, ts, seed=np.array(h0, dtype=np.uint32))


@pytest.mark.parametrize("n", [1500, 6000])
@pytest.mark.parametrize("zdrop", [0, 100, 8])
def test_lane_groups_short_pairs(n, zdrop):
    """Short pairs four to a warp (lane groups of 8): below the ordering
    threshold (every pair visited, longer ones skipped) and above it (the
    length order's suffix); empty sequences, N runs, IUPAC codes, seeds that
    hand pairs back, all against the oracle."""
    b = _short_mixed(n, 700 + zdrop + n)
    _check(Params(algo=KSW, zdrop=zdrop), b, f"n={n}")


def test_lane_groups_off_gives_the_same():
    """GASAL_B200_KSW_GROUPS=0 (every pair on 32-lane warps) and the default
    give identical outputs (checked in a child process: the setting is read
    once)."""
    import json, os, subprocess, sys
    child = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from gasal_b200 import lib as gl, workloads as W
from gasal_b200.capi import Params, KSW
p, b = W.workload4(20000, seed=731)[3]
o = gl.align(Params(algo=KSW, zdrop=100), b).as_dict(Params(algo=KSW, zdrop=100))
print(json.dumps({k: v.tolist() for k, v in o.items()}))
"""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for on in ("1", "0"):
        env = dict(os.environ, GASAL_B200_KSW_GROUPS=on)
        r = subprocess.run([sys.executable, "-c", child, root], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    assert outs[0] == outs[1]


def test_zdrop_hand_case_on_the_warp_kernel():
    """The hand-derived z-drop case (tests/test_extensions_cpu.py): 16
    matches, one mismatch, 7 matches, h0 20.  z-drop 1 stops at the mismatch
    row's tile: (36, 16, 16); z-drop 0 or 5 runs to (39, 24, 24).  Replicated
    so the batch runs on the warp-per-pair kernel and its lane groups."""
    q = b"ACGT" * 4 + b"A" + b"GATTACA"
    t = b"ACGT" * 4 + b"C" + b"GATTACA"
    n = 4096
    b = Batch.from_seqs([q] * n, [t] * n, seed=np.full(n, 20, dtype=np.uint32))
    for zdrop, exp in ((1, (36, 16, 16)), (0, (39, 24, 24)), (5, (39, 24, 24))):
        o = gl.align(Params(algo=KSW, zdrop=zdrop), b)
        assert (o.score == exp[0]).all() and (o.q_end == exp[1]).all() and (o.t_end == exp[2]).all(), zdrop
