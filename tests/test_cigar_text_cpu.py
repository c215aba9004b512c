"""Forward CIGAR text: the oracle's restatement of the reference test
program's decode (test_prog/test_prog.cpp:382-428) on known answers, and
against a literal Python transcription of that loop on the reference's own
traceback outputs (the golden fixtures)."""
import numpy as np
import pytest

from golden_cases import cases
from oracle.bindings import oracle_cigar_text

OPS = "MXDI"


def _bytes(runs):
    """run-length bytes as the traceback stores them: last operation first"""
    return [(c << 2) | OPS.index(op) for c, op in reversed(runs)]


def test_known_answers():
    pairs = [_bytes([(5, "M"), (2, "I"), (3, "M")]),
             _bytes([(4, "D"), (63, "M"), (63, "M")]),       # neighbouring runs of one operation merge
             [],                                             # no operations
             _bytes([(1, "X")]),
             _bytes([(12, "M"), (1, "D"), (7, "I"), (1, "X"), (40, "M")])]
    q_off = np.cumsum([0] + [len(p) + 8 for p in pairs[:-1]]).astype(np.uint32)
    cig = np.zeros(int(q_off[-1]) + len(pairs[-1]) + 8, dtype=np.uint8)
    for o, p in zip(q_off, pairs):
        cig[o:o + len(p)] = p
    n_cigar = np.array([len(p) for p in pairs], dtype=np.uint32)
    txt, lens = oracle_cigar_text(cig, q_off, n_cigar, 64)
    assert txt == ["5M2I3M", "4D126M", "", "1X", "12M1D7I1X40M"]
    assert list(lens) == [6, 6, 0, 2, 12]
    txt, lens = oracle_cigar_text(cig, q_off, n_cigar, 7)   # room for 6 characters and the NUL
    assert list(lens) == [6, 6, 0, 2, -1] and txt[4] == ""


def _literal(cig, off, n):
    """test_prog.cpp:382-428 as written (for n >= 1)."""
    last_op = cig[off + n - 1] & 3
    count = cig[off + n - 1] >> 2
    out = ""
    for u in range(n - 2, -1, -1):
        cur = cig[off + u] & 3
        if cur == last_op:
            count += cig[off + u] >> 2
        else:
            out += f"{count}{OPS[last_op]}"
            count = cig[off + u] >> 2
        last_op = cur
    return out + f"{count}{OPS[last_op]}"


@pytest.mark.parametrize("case", [c for c in cases() if "cigar" in c[3]], ids=lambda c: f"{c[0]}-{c[1].key()}")
def test_matches_the_reference_decode_on_golden_tracebacks(case):
    name, p, b, exp = case
    cig = exp["cigar"].astype(np.uint8)
    n_cigar = exp["n_cigar"].astype(np.uint32)
    txt, lens = oracle_cigar_text(cig, b.q_off, n_cigar, 4096)
    for i in range(b.n):
        if n_cigar[i] == 0:
            assert txt[i] == "" and lens[i] == 0
            continue
        want = _literal(cig.astype(np.int64), int(b.q_off[i]), int(n_cigar[i]))
        assert txt[i] == want and lens[i] == len(want), (name, i)
