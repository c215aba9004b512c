"""Per-pair mixed-algorithm dispatch (gb_align_dev_mixed): one device batch
whose pairs each name their own options.  Every pair must come out exactly as
gb_align_dev gives it under its kind's options alone (all result arrays,
including the ones the kind leaves untouched), and as the oracle gives it
for the arrays the reference defines.  The kinds' pairs are interleaved at
random, so the gather/scatter and the per-pair offsets are exercised."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import (Params, LOCAL, GLOBAL, SEMI_GLOBAL, BANDED, KSW, WITH_START, WITH_TB, TARGET,
                             TRUE)
from oracle.bindings import oracle_align

pytestmark = pytest.mark.gpu

FIELDS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")
FILL = -7


def _parts():
    w1 = W.workload1(3000, seed=41)
    return [
        (Params(algo=LOCAL, start_pos=WITH_START, second_best=TRUE, reverse_complement=1), w1[0][1]),
        (Params(algo=GLOBAL, start_pos=WITH_TB), W.workload2(600, seed=42)),
        (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET), w1[2][1]),
        (Params(algo=KSW, zdrop=100), W.workload3(300, seed=43)),
        (Params(algo=BANDED, k_band=32), W.workload0(800, seed=44)),
        (Params(algo=LOCAL, start_pos=WITH_TB, match=2, mismatch=3, gap_open=5, gap_extend=2),
         W.workload0(900, seed=45)),
        (Params(algo=BANDED, k_band=24, start_pos=WITH_START), W.workload0(500, seed=46)),
        (Params(algo=SEMI_GLOBAL, start_pos=WITH_TB, head=TARGET, tail=TARGET), w1[2][1]),
    ]


def _device(torch, b, dev):
    def t_(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt or a.dtype)).to(dev)
    keep = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
            "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32),
            "pq": torch.zeros(b.q.shape[0] // 8, dtype=torch.int32, device=dev),
            "pt": torch.zeros(b.t.shape[0] // 8, dtype=torch.int32, device=dev),
            "cigar": torch.zeros(b.q.shape[0], dtype=torch.uint8, device=dev),
            "ncig": torch.full((b.n,), FILL, dtype=torch.int32, device=dev)}
    keep.update({k: torch.full((b.n,), FILL, dtype=torch.int32, device=dev) for k in FIELDS})
    m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0], "q": keep["q"].data_ptr(), "t": keep["t"].data_ptr(),
         "pq": keep["pq"].data_ptr(), "pt": keep["pt"].data_ptr(), "q_off": keep["qo"].data_ptr(),
         "t_off": keep["to"].data_ptr(), "q_len": keep["ql"].data_ptr(), "t_len": keep["tl"].data_ptr(),
         "out_cigar": keep["cigar"].data_ptr(), "out_n_cigar": keep["ncig"].data_ptr()}
    for k in FIELDS:
        m["out_" + k] = keep[k].data_ptr()
    if b.q_op is not None:
        keep["qop"], keep["top"] = t_(b.q_op), t_(b.t_op)
        m["q_op"], m["t_op"] = keep["qop"].data_ptr(), keep["top"].data_ptr()
    if b.seed is not None:
        keep["seed"] = t_(b.seed, np.int32)
        m["seed"] = keep["seed"].data_ptr()
    return m, keep


def _host(keep):
    d = {k: keep[k].cpu().numpy() for k in FIELDS}
    d["n_cigar"] = keep["ncig"].cpu().numpy()
    d["cigar"] = keep["cigar"].cpu().numpy()
    return d


def _cigars(d, q_off, rows):
    return [bytes(d["cigar"][int(q_off[r]):int(q_off[r]) + int(d["n_cigar"][r])]) for r in rows]


def test_mixed_matches_single_kind_calls_and_oracle():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    gl.set_reference_reverse(True)
    parts = _parts()
    kinds, b, kind, idx = W.concat_parts(parts, shuffle_seed=5)
    m, keep = _device(torch, b, dev)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # a second call reuses the per-stream buffers
        gl.align_dev_mixed(kinds, kind, m, b.q_len, b.t_len, stream)
        torch.cuda.synchronize()
        got = _host(keep)
        for k, (p, pb) in enumerate(parts):
            rows = np.nonzero(kind == k)[0]
            src = idx[rows]
            pm, pkeep = _device(torch, pb, dev)
            gl.align_dev(p, pm, pb.q_len, pb.t_len, stream)
            torch.cuda.synchronize()
            one = _host(pkeep)
            what = f"call {call} kind {k} {p.key()}"
            for f in FIELDS + ("n_cigar",):
                g, w = got[f][rows], one[f][src]
                bad = np.nonzero(g != w)[0]
                assert bad.size == 0, f"{what} {f}: {bad.size} differ from gb_align_dev, first rows {rows[bad[:5]]}"
            exp = oracle_align(p, pb).as_dict(p)
            for f, v in exp.items():
                if f == "cigar":
                    assert _cigars(got, b.q_off, rows) == [bytes(v[int(pb.q_off[i]):int(pb.q_off[i]) +
                                                                int(exp["n_cigar"][i])]) for i in src], what
                    continue
                bad = np.nonzero(got[f][rows] != v[src])[0]
                assert bad.size == 0, f"{what} {f}: {bad.size} differ from the oracle"


def test_mixed_kind_without_pairs_and_empty_batch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    parts = _parts()[:2]
    kinds, b, kind, idx = W.concat_parts(parts, shuffle_seed=6)
    kinds = kinds + [Params(algo=KSW)]  # a third kind no pair names (and no seeds needed)
    m, keep = _device(torch, b, dev)
    m.pop("seed", None)
    gl.align_dev_mixed(kinds, kind, m, b.q_len, b.t_len, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = _host(keep)
    for k, (p, pb) in enumerate(parts):
        rows = np.nonzero(kind == k)[0]
        exp = oracle_align(p, pb).as_dict(p)
        for f, v in exp.items():
            if f != "cigar":
                assert np.array_equal(got[f][rows], v[idx[rows]]), f"kind {k} {f}"
    empty = dict(m)
    gl.align_dev_mixed(kinds, np.zeros(0, np.uint8), empty, np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                       torch.cuda.current_stream().cuda_stream)


def test_release_workspaces_between_calls():
    """gb_release_workspaces frees the per-stream buffers of gb_align_dev and
    the mixed dispatch; the next calls grow them again and give the same
    results (a traceback kind included)."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    parts = _parts()[:2]  # LOCAL WITH_START (second best, RC) and GLOBAL WITH_TB
    kinds, b, kind, idx = W.concat_parts(parts, shuffle_seed=8)
    m, keep = _device(torch, b, dev)
    stream = torch.cuda.current_stream().cuda_stream
    runs = []
    for _ in range(2):
        gl.align_dev_mixed(kinds, kind, m, b.q_len, b.t_len, stream)
        p, pb = parts[1]
        pm, pkeep = _device(torch, pb, dev)
        gl.align_dev(p, pm, pb.q_len, pb.t_len, stream)
        torch.cuda.synchronize()
        runs.append((_host(keep), _host(pkeep)))
        gl.release_workspaces()
    for f in FIELDS + ("n_cigar",):
        assert np.array_equal(runs[0][0][f], runs[1][0][f]), f
        assert np.array_equal(runs[0][1][f], runs[1][1][f]), f
