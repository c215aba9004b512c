"""The scalar C oracle against the reference's own outputs.

The fixtures hold what the reference GASAL2 library, compiled for sm_100a and
run on a B200 through its own C++ API, returned for seeded inputs: every
algorithm, start mode, traceback, second best, the 16 semi-global head/tail
variants, banded widths, ksw seeds, reverse/complement ops on lengths 1..48,
N-rich and lower-case sequences.  Bit-exact equality is required.
"""
import numpy as np
import pytest

from golden_cases import cases, case_ids
from oracle.bindings import oracle_align

ALL = list(cases())


@pytest.mark.parametrize("case", ALL, ids=case_ids())
def test_oracle_matches_reference(case):
    name, p, b, exp = case
    o = oracle_align(p, b, want_packed=True)
    got = o.as_dict(p)
    if name == "rc":
        got["packed_q"], got["packed_t"] = o.packed_q, o.packed_t
    assert set(exp) - set(got) == set(), f"fixture has fields the oracle does not produce: {set(exp) - set(got)}"
    for k, v in exp.items():
        assert np.array_equal(got[k], v), f"{name} {p.key()} {k}: first diff at {np.nonzero(got[k] != v)[0][:5]}"


def test_fixture_coverage():
    """Every algorithm and start mode is pinned by at least one fixture."""
    seen = {(p.algo, p.start_pos) for _, p, _, _ in ALL}
    from gasal_b200.capi import LOCAL, GLOBAL, SEMI_GLOBAL, BANDED, KSW, WITHOUT_START, WITH_START, WITH_TB
    for need in [(LOCAL, WITHOUT_START), (LOCAL, WITH_START), (LOCAL, WITH_TB), (GLOBAL, WITHOUT_START),
                 (GLOBAL, WITH_TB), (SEMI_GLOBAL, WITHOUT_START), (SEMI_GLOBAL, WITH_START),
                 (BANDED, WITHOUT_START), (KSW, WITHOUT_START)]:
        assert need in seen
    heads_tails = {(p.head, p.tail) for _, p, _, _ in ALL if p.algo == SEMI_GLOBAL}
    assert len(heads_tails) == 16


def _ksw_max_off(q, t, h0, zdrop, ma=1, mi=4, o=6, e=1):
    """Pure-Python ksw extension (the reference's loop: 8-row tile breaks,
    trimmed column range), returning (score, q_end, t_end, max_off)."""
    qlen, tlen = len(q), len(t)
    H = [0] * (qlen + 2)
    E = [0] * (qlen + 2)
    H[0] = h0
    H[1] = h0 - o - e if h0 > o + e else 0
    j = 2
    while j <= qlen and H[j - 1] > e:
        H[j] = H[j - 1] - e
        j += 1
    mx, max_i, max_j, max_ie, gscore, max_off = h0, -1, -1, -1, -1, 0
    beg, end, L8 = 0, qlen, (qlen >> 3) << 3
    i = 0
    while i < tlen:
        f, m, mj = 0, 0, -1
        h1 = max(h0 - (o + e * (i + 1)), 0) if beg == 0 else 0
        for j in range(beg, end):
            M, ee = H[j], E[j]
            H[j] = h1
            s = 0 if (q[j] == 78 or t[i] == 78) else (ma if (q[j] & 15) == (t[i] & 15) else -mi)
            M = M + s if M else 0
            h = max(M, ee, f)
            h1 = h
            if h >= m:
                mj, m = j, h
            tt = max(M - o - e, 0)
            E[j] = max(ee - e, tt)
            f = max(f - e, tt)
        H[end], E[end] = h1, 0
        if max(L8, end) == qlen:
            if h1 >= gscore:
                max_ie = i
            gscore = max(gscore, h1)
        leave = m == 0
        if not leave and m > mx:
            mx, max_i, max_j = m, i, mj
            max_off = max(max_off, abs(mj - i))
        elif not leave and zdrop > 0:
            di, dj = i - max_i, mj - max_j
            leave = (mx - m - (di - dj) * e > zdrop) if di > dj else (mx - m - (dj - di) * e > zdrop)
        if leave:
            i = ((i >> 3) + 1) << 3
            continue
        j = beg
        while j < end and H[j] == 0 and E[j] == 0:
            j += 1
        beg = j
        j = end
        while j >= beg and H[j] == 0 and E[j] == 0:
            j -= 1
        end = min(j + 2, qlen)
        i += 1
    if gscore <= 0 or gscore <= mx - 5:
        return mx, max_j + 1, max_i + 1, max_off
    return gscore, qlen, max_ie + 1, max_off


def test_oracle_ksw_max_off_against_python_loop():
    """The oracle's ksw max_off (the band labels' checker) against a pure-
    Python transcription of the same loop on small related and unrelated
    pairs, z-drop 0 and 30."""
    from gasal_b200.capi import Batch, Params, KSW
    rng = np.random.default_rng(505)
    qs, ts, h0 = [], [], []
    for k in range(60):
        q = bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(5, 90))).tolist())
        if k % 3 == 2:
            t = bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(5, 90))).tolist())
        else:
            t = bytearray(q)
            for _ in range(int(rng.integers(0, 6))):
                a = int(rng.integers(0, len(t)))
                if rng.random() < 0.5:
                    del t[a:a + int(rng.integers(1, 4))]
                else:
                    t[a:a] = bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(1, 4))).tolist())
            t = bytes(t) or b"A"
        qs.append(q)
        ts.append(t)
        h0.append(int(rng.integers(5, 40)))
    b = Batch.from_seqs(qs, ts, seed=np.array(h0, dtype=np.uint32))
    for zdrop in (0, 30):
        r = oracle_align(Params(algo=KSW, zdrop=zdrop), b)
        for i in range(b.n):
            exp = _ksw_max_off(qs[i], ts[i], h0[i], zdrop)
            got = (int(r.score[i]), int(r.q_end[i]), int(r.t_end[i]), int(r.score2[i]))
            assert got == exp, (zdrop, i, got, exp)
