"""The oracle's definitions of the extensions the reference lacks, pinned on
hand-made pairs whose answers follow from the definitions: BANDED WITH_START
(the reference's banded kernel reports ends only)."""
import numpy as np

from gasal_b200.capi import Batch, Params, BANDED, WITH_START
from oracle.bindings import oracle_align

ACGT = np.frombuffer(b"ACGT", np.uint8)


def _rs(rng, n):
    return bytes(ACGT[rng.integers(0, 4, n)])


def test_banded_start_hand_cases():
    rng = np.random.default_rng(12)
    q = _rs(rng, 100)
    pairs = [(q, q),                                        # whole pair: start (0, 0)
             (q, _rs(rng, 40) + q + _rs(rng, 30)),          # query inside the target at 40
             (q, q[:30] + _rs(rng, 10) + q[30:]),           # a 10-base insertion in the target
             (_rs(rng, 20) + q[:60], q[:60] + _rs(rng, 50))]  # the match on diagonal -20
    b = Batch.from_seqs([x for x, _ in pairs], [y for _, y in pairs])
    o = oracle_align(Params(algo=BANDED, k_band=64, start_pos=WITH_START), b)
    assert o.score.tolist() == [100, 100, 84, 60]
    assert list(zip(o.q_start.tolist(), o.t_start.tolist())) == [(0, 0), (0, 40), (0, 0), (20, 0)]
    assert list(zip(o.q_end.tolist(), o.t_end.tolist())) == [(99, 99), (99, 139), (99, 109), (79, 59)]
    # a band too narrow for diagonal -20 (k_band 16: two words right of the diagonal) misses that match
    narrow = oracle_align(Params(algo=BANDED, k_band=16, start_pos=WITH_START), b)
    assert narrow.score[3] < 60 and narrow.score[:3].tolist() == [100, 100, 84]


def test_banded_start_ends_where_forward_scores():
    """With a band wider than every matrix, the start pass is the local
    recurrence run backwards: the alignment from (q_start, t_start) to the end
    scores the forward score, so re-aligning just that slice locally gives it
    back with the slice's own ends at its last cell."""
    rng = np.random.default_rng(3)
    qs, ts = [], []
    for _ in range(40):
        core = _rs(rng, int(rng.integers(30, 120)))
        mut = bytearray(core)
        for i in rng.integers(0, len(mut), 3):
            mut[i] = ACGT[(list(ACGT).index(mut[i]) + 1) % 4]
        qs.append(_rs(rng, int(rng.integers(0, 30))) + bytes(mut) + _rs(rng, int(rng.integers(0, 30))))
        ts.append(_rs(rng, int(rng.integers(0, 30))) + core + _rs(rng, int(rng.integers(0, 30))))
    b = Batch.from_seqs(qs, ts)
    o = oracle_align(Params(algo=BANDED, k_band=4096, start_pos=WITH_START), b)
    sq = [qs[i][o.q_start[i]:o.q_end[i] + 1] for i in range(len(qs))]
    st = [ts[i][o.t_start[i]:o.t_end[i] + 1] for i in range(len(ts))]
    s = oracle_align(Params(algo=BANDED, k_band=4096), Batch.from_seqs(sq, st))
    assert s.score.tolist() == o.score.tolist()
    assert (s.q_end == o.q_end - o.q_start).all() and (s.t_end == o.t_end - o.t_start).all()


def _rescore(ops, q, t, qs, ts, p):
    """Affine score of forward CIGAR ops [(op, n)] from (qs, ts): 0 match,
    1 mismatch (scored from the bases, N scoring 0 as in local), 2 deletion,
    3 insertion; and the bases each op kind consumed."""
    score, i, j = 0, ts, qs
    for op, n in ops:
        if op in (0, 1):
            for _ in range(n):
                a, b = q[j], t[i]
                score += 0 if (a == ord("N") or b == ord("N")) else (p.match if a == b else -p.mismatch)
                i, j = i + 1, j + 1
        elif op == 2:
            score -= p.gap_open + p.gap_extend * n
            i += n
        else:
            score -= p.gap_open + p.gap_extend * n
            j += n
    return score, i, j


def test_semi_global_traceback_walks_the_alignment():
    """Target-tail SEMI_GLOBAL WITH_TB (an extension): the CIGAR runs from
    (q_start, t_start) to (the last query base, t_end) for every head, with
    the whole query aligned unless its head is free; where the walk starts
    and ends on aligned bases inside free edges, the CIGAR re-scores to the
    reported score."""
    from gasal_b200.capi import SEMI_GLOBAL, WITH_TB, NONE, QUERY, TARGET, BOTH, cigar_ops
    rng = np.random.default_rng(7)
    qs, ts = [], []
    for _ in range(200):
        core = bytearray(_rs(rng, int(rng.integers(20, 150))))
        mut = bytearray(core)
        for _k in range(int(rng.integers(0, 6))):
            x = int(rng.integers(0, len(mut)))
            kind = int(rng.integers(0, 3))
            if kind == 0:
                mut[x] = ACGT[(list(ACGT).index(mut[x]) + 1) % 4]
            elif kind == 1:
                del mut[x:x + int(rng.integers(1, 4))]
            else:
                mut[x:x] = _rs(rng, int(rng.integers(1, 4)))
        qs.append(bytes(mut) if mut else b"A")
        ts.append(_rs(rng, int(rng.integers(0, 40))) + bytes(core) + _rs(rng, int(rng.integers(0, 40))))
    b = Batch.from_seqs(qs, ts)
    for head in (NONE, QUERY, TARGET, BOTH):
        p = Params(algo=SEMI_GLOBAL, start_pos=WITH_TB, head=head, tail=TARGET)
        o = oracle_align(p, b)
        exact = 0
        for i in range(b.n):
            ops = cigar_ops(o.cigar, o.n_cigar, b.q_off, i)
            qs_, ts_ = int(o.q_start[i]), int(o.t_start[i])
            sc, ti, qj = _rescore(ops, qs[i], ts[i], qs_, ts_, p)
            assert qj == len(qs[i]) and ti == int(o.t_end[i]) + 1, (head, i)  # ends at (t_end, last query base)
            if head in (NONE, TARGET):
                assert qs_ == 0  # the query's head is not free: all of it is aligned
            if head in (NONE, QUERY):
                assert ts_ == 0
            if head in (TARGET, BOTH) and ops and ops[0][0] in (0, 1) and qs_ == 0:
                assert sc == int(o.score[i]), (head, i, sc, int(o.score[i]))
                exact += 1
        if head in (TARGET, BOTH):
            assert exact > b.n // 2


def test_ksw_zdrop_hand_case():
    """ksw z-drop on a pair whose answers follow from ksw_extend's rules by
    hand (match 1, mismatch 4, gap 6+1, h0 20).  q = t = ACGT x4, then one
    mismatch (A against C), then GATTACA on both.  The diagonal reaches
    mx = 36 at row/column 15; row 16's best cell is the mismatch, 32, on the
    same diagonal (di = dj = 1), a drop of 4.  z-drop 1: 4 > 1, the
    extension leaves the 8-row tile, which is the last one (rows 16-23), so
    the result is (36, q_end 16, t_end 16).  z-drop 0 (off) or 5: the
    diagonal recovers to 39 at the last cell, which is also the end-to-end
    score (gscore 39 > mx - 5), giving (39, 24, 24)."""
    from gasal_b200.capi import KSW
    q = b"ACGT" * 4 + b"A" + b"GATTACA"
    t = b"ACGT" * 4 + b"C" + b"GATTACA"
    b = Batch.from_seqs([q], [t], seed=np.array([20], dtype=np.uint32))
    for zdrop, exp in ((1, (36, 16, 16)), (0, (39, 24, 24)), (5, (39, 24, 24))):
        r = oracle_align(Params(algo=KSW, zdrop=zdrop), b)
        assert (int(r.score[0]), int(r.q_end[0]), int(r.t_end[0])) == exp, zdrop
