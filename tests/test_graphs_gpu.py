"""gasal_aln_async as a CUDA graph: relaunched for a batch of the same shape,
updated in place for a new one, captured across the warp-cooperative fork
onto the auxiliary stream and across chunked traceback.  Results must equal
the oracle's bit for bit on every path."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, LOCAL, GLOBAL, SEMI_GLOBAL, KSW, WITH_START, WITH_TB
from oracle.bindings import oracle_align

pytestmark = pytest.mark.gpu


def _same(got, exp, what):
    for k, v in exp.items():
        assert np.array_equal(got[k], v), f"{what}: {k} differs"


def _run(st, i, b):
    qi, ti = st.fill_fast(i, b)
    st.aln_async(i, qi, ti, b.n)
    st.wait(i)
    return st.results(i, b.n, b)


def _delta(a, b):
    return {k: b[k] - a[k] for k in a}


def test_graph_relaunch_and_update():
    gl.set_graphs(True)
    p = Params(algo=LOCAL, start_pos=WITH_START, second_best=1, reverse_complement=1)
    b1 = W.workload1(3000, seed=71)[0][1]
    b2 = W.workload1(2400, seed=72)[0][1]
    e1, e2 = oracle_align(p, b1).as_dict(p), oracle_align(p, b2).as_dict(p)
    with gl.Streams(1, 160, 310, 4000, p) as st:
        s0 = gl.graph_stats()
        _same(_run(st, 0, b1), e1, "first capture")
        _same(_run(st, 0, b1), e1, "same batch again")
        s1 = gl.graph_stats()
        _same(_run(st, 0, b2), e2, "another batch")
        _same(_run(st, 0, b1), e1, "first batch once more")
        s2 = gl.graph_stats()
    d1, d2 = _delta(s0, s1), _delta(s1, s2)
    assert d1["capture_refused"] == 0 and d2["capture_refused"] == 0
    assert d1["instantiated"] == 1 and d1["relaunched"] == 1
    assert d2["updated"] + d2["instantiated"] == 2


@pytest.mark.parametrize("p", [Params(algo=GLOBAL, start_pos=WITH_TB),
                               Params(algo=LOCAL, start_pos=WITH_START, second_best=1)],
                         ids=lambda p: p.key())
def test_graph_warp_cooperative_fork(p):
    """Long pairs go to the auxiliary stream inside the captured graph."""
    b = W.workload2(4000, seed=73)
    exp = oracle_align(p, b).as_dict(p)
    gl.set_graphs(True)
    with gl.Streams(1, 1008, 1100, 4000, p) as st:
        s0 = gl.graph_stats()
        _same(_run(st, 0, b), exp, "captured")
        _same(_run(st, 0, b), exp, "relaunched")
        d = _delta(s0, gl.graph_stats())
    assert d["capture_refused"] == 0 and d["relaunched"] == 1


def test_graph_chunked_traceback_matches_no_graph():
    """A traceback budget of 1 MiB splits the batch into many chunks inside
    one graph; the result equals the run without graphs and the oracle."""
    p = Params(algo=GLOBAL, start_pos=WITH_TB)
    b = W.workload2(600, seed=74)
    exp = oracle_align(p, b).as_dict(p)
    gl.set_tb_budget_mb(1)
    try:
        with gl.Streams(1, 1008, 1100, 600, p) as st:
            gl.set_graphs(False)
            plain = _run(st, 0, b)
            gl.set_graphs(True)
            s0 = gl.graph_stats()
            graphed = _run(st, 0, b)
            d = _delta(s0, gl.graph_stats())
    finally:
        gl.set_tb_budget_mb(98304)
        gl.set_graphs(True)
    _same(plain, exp, "no graph")
    _same(graphed, exp, "graph")
    assert d["capture_refused"] == 0


@pytest.mark.parametrize("p", [Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=1, tail=1),
                               Params(algo=KSW)], ids=lambda p: p.key())
def test_graph_other_algorithms(p):
    b = W.workload0(3000, seed=75) if p.algo != KSW else W.workload3(300, seed=75)
    exp = oracle_align(p, b).as_dict(p)
    with gl.Streams(2, 2048, 2100, 3000, p) as st:
        for i in range(2):
            _same(_run(st, i, b), exp, f"stream {i}")
