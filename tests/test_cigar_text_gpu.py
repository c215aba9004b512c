"""gb_cigar_text (forward CIGAR strings on the device) against the oracle's
decode, on the CUDA path's own traceback outputs: LOCAL and GLOBAL WITH_TB
on uneven 50-1000 bp pairs, slots large enough and one too small."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, LOCAL, GLOBAL, WITH_TB
from oracle.bindings import oracle_cigar_text

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
DEV = torch.device("cuda", 0)


def _device_text(cigar, q_off, n_cigar, stride):
    n = len(n_cigar)
    c = torch.from_numpy(np.ascontiguousarray(cigar, dtype=np.uint8)).to(DEV)
    qo = torch.from_numpy(np.ascontiguousarray(q_off, dtype=np.uint32).view(np.int32)).to(DEV)
    nc = torch.from_numpy(np.ascontiguousarray(n_cigar, dtype=np.uint32).view(np.int32)).to(DEV)
    text = torch.full((n * stride,), 0x55, dtype=torch.uint8, device=DEV)
    lens = torch.full((n,), -7, dtype=torch.int32, device=DEV)
    gl.cigar_text_dev(c.data_ptr(), qo.data_ptr(), nc.data_ptr(), n, text.data_ptr(), stride, lens.data_ptr(),
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    t = text.cpu().numpy()
    ln = lens.cpu().numpy()
    return [bytes(t[i * stride:i * stride + max(int(ln[i]), 0)]).decode() for i in range(n)], ln, t


@pytest.mark.parametrize("algo", [GLOBAL, LOCAL])
def test_device_text_matches_oracle(algo):
    b = W.workload2(3000, seed=140 + algo)
    p = Params(algo=algo, start_pos=WITH_TB)
    o = gl.align(p, b).as_dict(p)
    cig, ncig = o["cigar"], o["n_cigar"]
    stride = int(6 * ncig.max() + 8)
    got, glen, raw = _device_text(cig, b.q_off, ncig, stride)
    exp, elen = oracle_cigar_text(cig, b.q_off, ncig, stride)
    assert np.array_equal(glen, elen)
    assert got == exp
    assert all(raw[i * stride + glen[i]] == 0 for i in range(b.n))  # NUL-terminated
    # the text describes the alignment: M + X + I columns span the query's aligned part
    for i in range(0, b.n, 97):
        q_cols = sum(int(n) for n, op in zip(*_split(got[i])) if op in "MXI")
        assert q_cols > 0


def _split(s):
    nums, ops, cur = [], [], ""
    for ch in s:
        if ch.isdigit():
            cur += ch
        else:
            nums.append(cur)
            ops.append(ch)
            cur = ""
    return nums, ops


def test_slots_too_small_report_minus_one():
    b = W.workload2(800, seed=150)
    p = Params(algo=GLOBAL, start_pos=WITH_TB)
    o = gl.align(p, b).as_dict(p)
    got, glen, raw = _device_text(o["cigar"], b.q_off, o["n_cigar"], 9)
    exp, elen = oracle_cigar_text(o["cigar"], b.q_off, o["n_cigar"], 9)
    assert np.array_equal(glen, elen) and got == exp
    assert (glen == -1).any() and (glen >= 0).any()
    assert all(raw[i * 9] == 0 for i in np.nonzero(glen == -1)[0])
