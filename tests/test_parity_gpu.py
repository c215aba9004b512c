"""CUDA path against the reference's own outputs (golden fixtures) and
against the oracle on larger seeded workloads.  Everything goes through the C
ABI (gb_align / the gasal_c_* storage API).  Bit-exact equality is required:
this is integer and index work."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import (Batch, Params, LOCAL, GLOBAL, SEMI_GLOBAL, BANDED, KSW, WITHOUT_START, WITH_START,
                             WITH_TB, NONE, QUERY, TARGET, BOTH)
from golden_cases import cases, case_ids
from oracle.bindings import oracle_align, ORC_ALL

pytestmark = pytest.mark.gpu

ALL = list(cases())


@pytest.fixture(scope="module", autouse=True)
def _settings():
    gl.set_reference_max_query_len(2048)  # the golden reference build's MAX_QUERY_LEN
    gl.set_reference_reverse(True)
    yield


def assert_same(got: dict, exp: dict, what: str):
    for k, v in exp.items():
        assert k in got, f"{what}: missing {k}"
        g = got[k]
        if not np.array_equal(g, v):
            bad = np.nonzero(g != v)[0]
            raise AssertionError(f"{what} {k}: {len(bad)} differ, first {bad[:5]}: got {g[bad[:5]]} want {v[bad[:5]]}")


@pytest.mark.parametrize("case", ALL, ids=case_ids())
def test_cuda_matches_reference_golden(case):
    name, p, b, exp = case
    o = gl.align(p, b, want_packed=True)
    got = o.as_dict(p)
    if name == "rc":
        got["packed_q"], got["packed_t"] = o.packed_q, o.packed_t
    assert_same(got, exp, f"{name} {p.key()}")


def _vs_oracle(p, b, **kw):
    o = gl.align(p, b)
    r = oracle_align(p, b, **kw)
    assert_same(o.as_dict(p), r.as_dict(p), p.key())


def test_workload0_full_size():
    """Workload 0 at its full size (20,000 pairs, LOCAL WITHOUT_START)."""
    _vs_oracle(Params(algo=LOCAL), W.workload0())


@pytest.mark.parametrize("p", W.WORKLOAD1_PARAMS, ids=lambda p: p.key())
def test_workload1_shape(p):
    """Workload 1's three launches on 6,000 pairs each (RC on half)."""
    parts = W.workload1(18000, seed=99)
    for pp, bb in parts:
        if pp.key() == p.key():
            _vs_oracle(pp, bb)


def test_workload2_traceback_chunked():
    """GLOBAL WITH_TB on uneven 50-1000 bp pairs, with a tiny tile budget so
    the batch runs in many chunks."""
    b = W.workload2(1500, seed=7)
    gl.set_tb_budget_mb(8)
    try:
        _vs_oracle(Params(algo=GLOBAL, start_pos=WITH_TB), b)
    finally:
        gl.set_tb_budget_mb(98304)


def test_local_traceback_and_second_best():
    b = W.workload0(3000, seed=5)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_TB, second_best=1), b)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, second_best=1, match=2, mismatch=3, gap_open=5,
                      gap_extend=2), b)


def test_ksw_long():
    b = W.workload3(400, seed=8)
    _vs_oracle(Params(algo=KSW), b)


@pytest.mark.parametrize("zdrop", [100, 20, 1])
def test_ksw_zdrop(zdrop):
    """The z-drop branch the reference leaves dead (its kernel hard-codes
    zdrop 0): a drop ends the current 8-row target tile.  Workload 3 pairs
    (250-2000 bp, 0.5-10% indels) plus unrelated pairs, where drops are
    frequent."""
    b = W.workload3(600, seed=80 + zdrop)
    _vs_oracle(Params(algo=KSW, zdrop=zdrop), b)
    u = W.workload0(600, seed=81)
    rng = np.random.default_rng(zdrop)
    u.t = u.t.copy()
    u.t[:] = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, u.t.shape[0])]
    u.seed = rng.integers(20, 61, u.n).astype(np.uint32)
    _vs_oracle(Params(algo=KSW, zdrop=zdrop), u)


@pytest.mark.parametrize("head", [NONE, QUERY, TARGET, BOTH])
@pytest.mark.parametrize("tail", [NONE, QUERY, TARGET, BOTH])
def test_semi_global_variants(head, tail):
    b = W.workload0(800, seed=head * 4 + tail)
    _vs_oracle(Params(algo=SEMI_GLOBAL, head=head, tail=tail, second_best=1), b)
    if tail in (TARGET, NONE):
        _vs_oracle(Params(algo=SEMI_GLOBAL, head=head, tail=tail, start_pos=WITH_START), b)


def test_long_queries_use_global_row_buffer():
    """Queries long enough that the row buffers leave shared memory."""
    b = W.workload3(64, seed=9)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), b)
    _vs_oracle(Params(algo=GLOBAL), b)


def test_banded():
    b = W.workload0(1000, seed=10)
    for k in (8, 24, 64):
        _vs_oracle(Params(algo=BANDED, k_band=k), b)


@pytest.mark.parametrize("head", [NONE, QUERY, TARGET, BOTH])
def test_semi_global_traceback(head):
    """Target-tail SEMI_GLOBAL WITH_TB, an extension (the reference
    instantiates it empty): forward tiles on the one-pair-per-thread kernel,
    the semi-global walk in the traceback kernel; CIGAR bytes, counts and
    starts against the oracle, with second best and in several tile chunks."""
    b = W.workload1(3000, seed=14)[2][1]
    _vs_oracle(Params(algo=SEMI_GLOBAL, start_pos=WITH_TB, head=head, tail=TARGET), b)
    gl.set_tb_budget_mb(4)
    try:
        _vs_oracle(Params(algo=SEMI_GLOBAL, start_pos=WITH_TB, head=head, tail=TARGET, second_best=1, match=2,
                          mismatch=3, gap_open=5, gap_extend=2), W.workload2(400, seed=15))
    finally:
        gl.set_tb_budget_mb(98304)
    # other tails keep the reference's outputs (no CIGAR)
    _vs_oracle(Params(algo=SEMI_GLOBAL, start_pos=WITH_TB, head=head, tail=QUERY), b)


def test_banded_with_start():
    """BANDED WITH_START, an extension (the reference's banded kernel reports
    ends only): the start pass runs the banded recurrence backwards over the
    forward band's tiles.  Against the oracle on seeded pairs (long ones on
    global row buffers too) and on hand-made pairs whose starts are known."""
    b = W.workload0(1500, seed=12)
    for k in (8, 24, 64, 512):
        _vs_oracle(Params(algo=BANDED, k_band=k, start_pos=WITH_START), b)
    _vs_oracle(Params(algo=BANDED, k_band=64, start_pos=WITH_START, match=2, mismatch=3, gap_open=5, gap_extend=2),
               W.workload3(64, seed=13))
    rng = np.random.default_rng(12)
    acgt = np.frombuffer(b"ACGT", np.uint8)

    def rs(n):
        return bytes(acgt[rng.integers(0, 4, n)])
    q = rs(100)
    pairs = [(q, q), (q, rs(40) + q + rs(30)), (q, q[:30] + rs(10) + q[30:])]
    hb = Batch.from_seqs([x for x, _ in pairs], [y for _, y in pairs])
    o = gl.align(Params(algo=BANDED, k_band=64, start_pos=WITH_START), hb)
    assert o.score.tolist() == [100, 100, 84]
    assert list(zip(o.q_start.tolist(), o.t_start.tolist())) == [(0, 0), (0, 40), (0, 0)]
    assert list(zip(o.q_end.tolist(), o.t_end.tolist())) == [(99, 99), (99, 139), (99, 109)]


def test_correct_reverse_mode():
    """With the reference-compatible reversal off, sequences are truly
    reverse-complemented; checked against the oracle's same mode."""
    b = W.workload1(3000, seed=11)[0][1]
    gl.set_reference_reverse(False)
    try:
        p = Params(algo=LOCAL, start_pos=WITH_START, reverse_complement=1)
        o = gl.align(p, b, want_packed=True)
        r = oracle_align(p, b, want_packed=True, compat=ORC_ALL & ~1)
        assert np.array_equal(o.packed_q, r.packed_q)
        assert_same(o.as_dict(p), r.as_dict(p), "rc-correct")
    finally:
        gl.set_reference_reverse(True)


def test_streams_api_per_sequence_fill():
    """The GASAL2 call sequence: init streams, gasal_host_batch_fill per
    sequence, gasal_op_fill, gasal_aln_async, poll gasal_is_aln_async_done,
    read host_res -- on two streams in flight at once."""
    p = Params(algo=LOCAL, start_pos=WITH_START, second_best=1, reverse_complement=1)
    parts = [W.workload1(2000, seed=12)[0][1], W.workload1(2000, seed=13)[0][1]]
    with gl.Streams(2, 160, 310, 1000, p) as st:
        sizes = [st.fill(i, b) for i, b in enumerate(parts)]
        for i, b in enumerate(parts):
            st.aln_async(i, sizes[i][0], sizes[i][1], b.n)
        for i, b in enumerate(parts):
            st.wait(i)
            got = st.results(i, b.n, b)
            exp = oracle_align(p, b).as_dict(p)
            assert_same(got, exp, f"stream {i}")
            assert st.is_done(i) == -2  # nothing in flight after completion


def test_streams_api_bulk_fill_repeated():
    """gasal_host_batch_fill_mt (the batch's padded blocks copied over host
    threads, after gasal_host_batch_reset) staged twice into one storage:
    both runs equal the oracle, the second after the first batch's pages
    were reused."""
    p = Params(algo=GLOBAL, start_pos=WITH_TB)
    batches = [W.workload2(3000, seed=15), W.workload2(2500, seed=16)]
    nq = max(int(b.q.shape[0]) for b in batches)
    nt = max(int(b.t.shape[0]) for b in batches)
    with gl.Streams(1, nq // 2500 + 8, nt // 2500 + 8, 3000, p) as st:
        for k, b in enumerate(batches):
            qi, ti = st.fill_bulk(0, b, threads=4)
            assert (qi, ti) == (int(b.q.shape[0]), int(b.t.shape[0]))
            st.aln_async(0, qi, ti, b.n)
            st.wait(0)
            got = st.results(0, b.n, b)
            assert_same(got, oracle_align(p, b).as_dict(p), f"bulk fill {k}")


def test_streams_api_grows_buffers():
    """A batch larger than the storage was created for is accepted after the
    host pages chain and device buffers regrow (reference behaviour)."""
    p = Params(algo=GLOBAL, start_pos=WITH_TB)
    b = W.workload2(300, seed=14)
    with gl.Streams(1, 64, 64, 300, p) as st:
        qi, ti = st.fill(0, b)
        st.aln_async(0, qi, ti, b.n)
        st.wait(0)
        got = st.results(0, b.n, b)
    exp = oracle_align(p, b).as_dict(p)
    assert_same(got, exp, "grown")


# ---- warp-cooperative path (queries of 32+ words in batches of 2048+) ----

def test_wc_local_long_pairs_all_modes():
    """Long LOCAL pairs (250-2000 bp) on the warp-cooperative kernel: forward,
    second best (two passes), start pass (reversed sweep), traceback."""
    b = W.workload3(2100, seed=41)
    _vs_oracle(Params(algo=LOCAL), b)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), b)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_TB), b)


def test_wc_global_mixed_lengths_traceback():
    """Log-uniform 50-1000 bp: short pairs on the one-thread kernel, long ones
    on the warp kernel, in one launch; GLOBAL score and CIGAR."""
    b = W.workload2(4000, seed=42)
    _vs_oracle(Params(algo=GLOBAL), b)
    _vs_oracle(Params(algo=GLOBAL, start_pos=WITH_TB), b)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), b)


def test_wc_unrelated_long_pairs():
    """Random unrelated long pairs: local maxima anywhere, including end cells
    in the first 31 query words (start pass falls back to one lane)."""
    rng = np.random.default_rng(43)
    qs = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(260, 700))).tolist()) for _ in range(2200)]
    ts = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(20, 700))).tolist()) for _ in range(2200)]
    from gasal_b200.capi import Batch
    b = Batch.from_seqs(qs, ts)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), b)
    _vs_oracle(Params(algo=GLOBAL, start_pos=WITH_TB), b)


@pytest.mark.parametrize("k", range(4))
def test_workload4_launches(k):
    """Workload 4's four launches (mixed 50-5000 bp, short- and long-read-like
    and unrelated pairs) on 4,000 pairs."""
    p, b = W.workload4(4000, seed=100)[k]
    _vs_oracle(p, b)


@pytest.mark.parametrize("head", [NONE, QUERY, TARGET, BOTH])
def test_wc_semi_global_target_tail(head):
    """Long target-tail SEMI_GLOBAL pairs (queries of 32+ words in a batch of
    2048+) on the warp-cooperative kernel: forward with second best, and the
    reversed start pass; every head mode."""
    b = W.workload2(3000, seed=60 + head)
    _vs_oracle(Params(algo=SEMI_GLOBAL, head=head, tail=TARGET, second_best=1), b)
    _vs_oracle(Params(algo=SEMI_GLOBAL, head=head, tail=TARGET, start_pos=WITH_START), b)


def test_wc_semi_global_scores_and_open_forms():
    """Other scores, a zero gap open (the shortened E chain's edge) and a
    negative one (the literal chain), on long pairs."""
    b = W.workload3(2100, seed=64)
    for sc in (dict(match=2, mismatch=3, gap_open=5, gap_extend=2), dict(gap_open=0, gap_extend=2),
               dict(gap_open=-1, gap_extend=3)):
        _vs_oracle(Params(algo=SEMI_GLOBAL, head=TARGET, tail=TARGET, start_pos=WITH_START, second_best=1, **sc), b)


def test_wc_table_and_compare_scoring_split():
    """Long pairs on the warp-cooperative kernels, a fifth of them with IUPAC
    codes outside A/C/G/T/N: those leave the table-scoring launch for the
    compare-scoring one that follows it, in the same warps as plain pairs.
    LOCAL (start and traceback), GLOBAL traceback and target-tail
    SEMI_GLOBAL against the oracle; then a mismatch penalty beyond a byte,
    where every pair takes the compare path."""
    rng = np.random.default_rng(47)
    from gasal_b200.capi import Batch
    qs, ts = [], []
    for k in range(2600):
        q = bytearray(rng.choice(list(b"ACGT"), size=int(rng.integers(260, 900))).tolist())
        t = bytearray(q)
        for _ in range(int(rng.integers(0, 10))):
            a = int(rng.integers(0, len(t)))
            t[a] = int(rng.choice(list(b"ACGT")))
        if k % 5 == 3:
            q[int(rng.integers(0, len(q)))] = ord("R")
        if k % 7 == 4:
            t[int(rng.integers(0, len(t)))] = ord("Y")
        qs.append(bytes(q))
        ts.append(bytes(t) + bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(0, 40))).tolist()))
    b = Batch.from_seqs(qs, ts)
    for p in (Params(algo=LOCAL, start_pos=WITH_START), Params(algo=LOCAL, start_pos=WITH_TB),
              Params(algo=GLOBAL, start_pos=WITH_TB),
              Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET)):
        _vs_oracle(p, b)
    # scores that leave the 16-bit row buffer (match 200 on 260-900 bp): the start passes and
    # tracebacks of such a batch run on the one-pair-per-thread kernel
    big = Params(algo=LOCAL, start_pos=WITH_START, match=200, mismatch=150, gap_open=300, gap_extend=20)
    _vs_oracle(big, b)
    # a mismatch penalty beyond a byte (scores stay far inside the 16-bit row buffer)
    _vs_oracle(Params(algo=LOCAL, start_pos=WITH_START, match=1, mismatch=200, gap_open=6, gap_extend=1), b)
    _vs_oracle(Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, match=1, mismatch=200,
                      gap_open=6, gap_extend=1), b)
