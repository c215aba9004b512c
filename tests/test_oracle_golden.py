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
