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


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    from gasal_b200 import lib as gl, workloads as W
    from gasal_b200.capi import Params, LOCAL, GLOBAL, WITH_START, TRUE
    dev = torch.device("cuda", 0)
    gl.set_reference_reverse(True)
    calls = [
        (Params(algo=LOCAL, start_pos=WITH_START, second_best=TRUE, reverse_complement=1),
         W.workload1(6000, seed=31)[0][1]),
        (Params(algo=GLOBAL), W.workload3(300, seed=32)),  # queries up to 2000 bp: a small grid
    ]
    for p, b in calls:
        m, keep = _device_batch(torch, b, dev)
        got = _run(torch, gl, p, m, b, dev, noalloc=True)
        want = _run(torch, gl, p, m, b, dev, noalloc=False)
        for k in FIELDS:
            assert np.array_equal(got[k], want[k]), f"{p.key()} {k}: {np.nonzero(got[k] != want[k])[0][:5]}"
        del keep


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
