"""Full-size checks through a size-independent property: the batched form
(length-ordered persistent launches, warp-cooperative lane groups, warp-per-
pair ksw) and the plain full-DP form (every pair one per thread in input
order) must give bit-identical outputs.  w1 at its full 1M pairs and w2 at
its full 2M (CIGAR bytes included); ksw and the mixed workload on samples
the plain form finishes in seconds.  The oracle pins both forms at smaller
sizes (test_parity_gpu, test_tuning_gpu)."""
import functools

import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, GLOBAL, KSW, WITH_TB

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
DEV = torch.device("cuda", 0)
FIELDS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")


def _both_forms(p, b):
    from gasal_b200.band_train import DeviceBatch
    db = DeviceBatch(torch, b, DEV, outs=FIELDS)
    m = dict(db.map)
    keep = []
    if b.q_op is not None:
        keep += [torch.from_numpy(b.q_op).to(DEV), torch.from_numpy(b.t_op).to(DEV)]
        m["q_op"], m["t_op"] = keep[0].data_ptr(), keep[1].data_ptr()
    cig = torch.zeros(b.q.shape[0], dtype=torch.uint8, device=DEV)
    ncig = torch.zeros(b.n, dtype=torch.int32, device=DEV)
    m["out_cigar"], m["out_n_cigar"] = cig.data_ptr(), ncig.data_ptr()
    if not p.second_best:
        m["out_score2"] = m["out_q_end2"] = m["out_t_end2"] = None
    saved = gl.get_tuning()
    res = []
    try:
        for form in ({}, gl.PLAIN_FORM):
            for k in FIELDS:
                db.out(k).fill_(-7)
            cig.zero_()
            ncig.fill_(-7)
            gl.set_tuning(**saved)
            gl.set_tuning(**form)
            gl.align_dev(p, m, b.q_len, b.t_len, 0)
            torch.cuda.synchronize()
            res.append({k: db.out(k).clone() for k in FIELDS} | {"cigar": cig.clone(), "n_cigar": ncig.clone()})
    finally:
        gl.set_tuning(**saved)
    for k in res[0]:
        same = torch.equal(res[0][k], res[1][k])
        assert same, f"{p.key()} {k}: {int((res[0][k] != res[1][k]).sum())} differ"


@functools.lru_cache(maxsize=1)
def _w1():
    return W.workload1(1_000_000, seed=W.SEED_BASE + 1)


@pytest.mark.parametrize("k", range(3))
def test_w1_full_size(k):
    """w1 at 1M pairs: LOCAL (second best), GLOBAL, SEMI_GLOBAL with starts, RC on half."""
    p, b = _w1()[k]
    _both_forms(p, b)


def test_w2_full_size():
    """w2 at 2M pairs: GLOBAL with CIGAR, 50-1000 bp."""
    _both_forms(Params(algo=GLOBAL, start_pos=WITH_TB), W.workload2(2_000_000, seed=W.SEED_BASE + 2))


def test_ksw_sample():
    _both_forms(Params(algo=KSW, zdrop=100), W.workload3(40_000, seed=W.SEED_BASE + 3))


@pytest.mark.parametrize("k", range(4))
def test_w4_sample(k):
    p, b = W.workload4(120_000, seed=W.SEED_BASE + 4)[k]
    _both_forms(p, b)
