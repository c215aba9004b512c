"""gb_align_dev_noalloc -- the entry point for callers that cannot allocate
device memory (inside stream capture, under a memory arena, or as a plugin
that must not call cudaMalloc).  It keeps its DP row buffers in a static
device array instead of allocating; this checks, through the C ABI, that two
calls in a row give exactly what the allocating entry point gb_align_dev
gives on the same inputs.  The test allocates its own buffers with torch; the
entry point under test allocates nothing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_batch(torch, b, dev):
    def t_(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt or a.dtype)).to(dev)
    keep = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
            "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32)}
    keep["pq"] = torch.zeros(b.q.shape[0] // 8, dtype=torch.int32, device=dev)
    keep["pt"] = torch.zeros(b.t.shape[0] // 8, dtype=torch.int32, device=dev)
    m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0], "q": keep["q"].data_ptr(), "t": keep["t"].data_ptr(),
         "pq": keep["pq"].data_ptr(), "pt": keep["pt"].data_ptr(), "q_off": keep["qo"].data_ptr(),
         "t_off": keep["to"].data_ptr(), "q_len": keep["ql"].data_ptr(), "t_len": keep["tl"].data_ptr()}
    if b.q_op is not None:
        keep["qop"], keep["top"] = t_(b.q_op), t_(b.t_op)
        m["q_op"], m["t_op"] = keep["qop"].data_ptr(), keep["top"].data_ptr()
    if b.seed is not None:
        keep["seed"] = t_(b.seed, np.int32)
        m["seed"] = keep["seed"].data_ptr()
    return m, keep


FIELDS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")


def _run(torch, gl, p, m, b, dev, noalloc):
    outs = {k: torch.full((b.n,), -7, dtype=torch.int32, device=dev) for k in FIELDS}
    mm = dict(m)
    for k, v in outs.items():
        mm["out_" + k] = v.data_ptr()
    gl.align_dev(p, mm, b.q_len, b.t_len, torch.cuda.current_stream().cuda_stream, noalloc=noalloc)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def _cases(W, capi):
    """(Params, Batch) for every algorithm family the entry point serves."""
    from gasal_b200.capi import (Params, LOCAL, GLOBAL, SEMI_GLOBAL, BANDED, KSW, WITH_START, WITHOUT_START,
                                 TARGET, TRUE)
    w1 = W.workload1(6000, seed=31)
    ksw = W.workload3(400, seed=33)
    return [
        ("local_start_second_rc", Params(algo=LOCAL, start_pos=WITH_START, second_best=TRUE, reverse_complement=1),
         w1[0][1]),
        ("global_long", Params(algo=GLOBAL), W.workload3(300, seed=32)),  # queries up to 2000 bp: a small grid
        ("semi_global_target_target_start", Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET,
                                                   second_best=TRUE), w1[2][1]),
        ("banded_k32", Params(algo=BANDED, k_band=32), W.workload0(3000, seed=34)),
        ("ksw_zdrop100", Params(algo=KSW, zdrop=100), ksw),
        ("ksw_zdrop0", Params(algo=KSW), ksw),
    ]


@pytest.mark.parametrize("case", ["local_start_second_rc", "global_long", "semi_global_target_target_start",
                                  "banded_k32", "ksw_zdrop100", "ksw_zdrop0"])
def test_noalloc_matches_allocating_entry_point_and_oracle(case):
    """Two calls in a row through gb_align_dev_noalloc must each equal
    gb_align_dev's output and the scalar oracle's, field for field."""
    torch = pytest.importorskip("torch")
    from gasal_b200 import lib as gl, workloads as W, capi
    from oracle.bindings import oracle_align
    dev = torch.device("cuda", 0)
    gl.set_reference_reverse(True)
    name, p, b = next(c for c in _cases(W, capi) if c[0] == case)
    m, keep = _device_batch(torch, b, dev)
    want = _run(torch, gl, p, m, b, dev, noalloc=False)
    exp = oracle_align(p, b).as_dict(p)
    for call in range(2):
        got = _run(torch, gl, p, m, b, dev, noalloc=True)
        for k in (f for f in FIELDS if f in exp):  # the arrays the reference defines for these options
            assert np.array_equal(got[k], want[k]), f"call {call} {p.key()} {k}: {np.nonzero(got[k] != want[k])[0][:5]}"
        for k, v in exp.items():
            if k in got:
                assert np.array_equal(got[k], v), f"call {call} {p.key()} {k} vs oracle: {np.nonzero(got[k] != v)[0][:5]}"
    del keep


def test_noalloc_empty_batch_is_a_no_op():
    torch = pytest.importorskip("torch")
    from gasal_b200 import lib as gl
    from gasal_b200.capi import Params, LOCAL
    import ctypes as C
    b = gl.GbDevBatch()
    b.n = 0
    o = gl.GbDevOut()
    cp = Params(algo=LOCAL).to_c()
    assert gl.lib().gb_align_dev_noalloc(C.byref(cp), C.byref(b), C.byref(o), C.c_void_p(0)) == 0
    torch.cuda.synchronize()


def test_noalloc_rejects_traceback_and_oversized_queries():
    torch = pytest.importorskip("torch")
    from gasal_b200 import lib as gl
    from gasal_b200.capi import Batch, Params, GLOBAL, LOCAL, WITH_TB
    dev = torch.device("cuda", 0)
    b = Batch.from_seqs([b"ACGTACGT"], [b"ACGTACGT"])
    m, keep = _device_batch(torch, b, dev)
    with pytest.raises(gl.GasalError):
        _run(torch, gl, Params(algo=GLOBAL, start_pos=WITH_TB), m, b, dev, noalloc=True)
    # a query so long that the static scratch cannot hold 32 row buffers
    long_q = b"A" * 300000
    bl = Batch.from_seqs([long_q], [b"ACGT"])
    ml, keep2 = _device_batch(torch, bl, dev)
    with pytest.raises(gl.GasalError, match="limit"):
        _run(torch, gl, Params(algo=LOCAL), ml, bl, dev, noalloc=True)
    del keep, keep2
