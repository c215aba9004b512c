"""Launch tuning and the autotuner: results never depend on the block size,
the warp-cooperative threshold or the ordering threshold, and gb_autotune
installs the fastest candidate it timed."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, LOCAL, GLOBAL, SEMI_GLOBAL, WITH_START, WITH_TB, TARGET, QUERY, NONE
from oracle.bindings import oracle_align

pytestmark = pytest.mark.gpu

FIELDS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")


def _device(torch, b, dev):
    def t_(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a).view(dt or a.dtype)).to(dev)
    keep = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
            "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32),
            "pq": torch.zeros(b.q.shape[0] // 8, dtype=torch.int32, device=dev),
            "pt": torch.zeros(b.t.shape[0] // 8, dtype=torch.int32, device=dev)}
    keep.update({k: torch.full((b.n,), -7, dtype=torch.int32, device=dev) for k in FIELDS})
    m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0]}
    for k, src in (("q", "q"), ("t", "t"), ("pq", "pq"), ("pt", "pt"), ("q_off", "qo"), ("t_off", "to"),
                   ("q_len", "ql"), ("t_len", "tl")):
        m[k] = keep[src].data_ptr()
    for k in FIELDS:
        m["out_" + k] = keep[k].data_ptr()
    return m, keep


@pytest.mark.parametrize("tuning", [dict(block=32, wc_min_qregs=32, min_order_pairs=0),
                                    dict(block=128, wc_min_qregs=64, min_order_pairs=1 << 30),
                                    dict(block=64, wc_min_qregs=40, min_order_pairs=100)],
                         ids=["b32_wc32_order_all", "b128_wc64_no_order", "b64_wc40"])
def test_results_independent_of_tuning(tuning):
    saved = gl.get_tuning()
    b = W.workload2(3000, seed=61)
    try:
        gl.set_tuning(**tuning)
        for p in (Params(algo=GLOBAL, start_pos=WITH_TB), Params(algo=LOCAL, start_pos=WITH_START, second_best=1)):
            got = gl.align(p, b).as_dict(p)
            exp = oracle_align(p, b).as_dict(p)
            for k, v in exp.items():
                assert np.array_equal(got[k], v), f"{tuning} {p.key()} {k}"
    finally:
        gl.set_tuning(**saved)


def test_autotune_installs_fastest_and_keeps_results():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    saved = gl.get_tuning()
    p = Params(algo=LOCAL, start_pos=WITH_START, second_best=1)
    b = W.workload2(4000, seed=62)
    m, keep = _device(torch, b, dev)
    try:
        best = gl.autotune(p, m, b.q_len, b.t_len, torch.cuda.current_stream().cuda_stream, reps=1)
        torch.cuda.synchronize()
        assert best["block"] in (32, 64, 128) and best["wc_min_qregs"] in (16, 32, 48, 64)
        assert best["wc_group"] in (0, 8, 16, 32) and best["wc_min_qregs"] >= best["wc_group"]
        assert best["ms"] > 0
        cur = gl.get_tuning()
        assert (cur["block"], cur["wc_min_qregs"], cur["wc_group"]) == \
            (best["block"], best["wc_min_qregs"], best["wc_group"])
        exp = oracle_align(p, b).as_dict(p)
        for k, v in exp.items():
            assert np.array_equal(keep[k].cpu().numpy(), v), k
    finally:
        gl.set_tuning(**saved)


@pytest.mark.parametrize("split", [0, 1])
def test_start_pass_split_keeps_results(split):
    """Start passes in the forward launch or as their own score-ordered
    launch give the same starts (batches of 2048+ pairs; the w2 batch also
    has warp-cooperative long pairs, whose starts the split leaves alone)."""
    saved = gl.get_tuning()
    try:
        gl.set_tuning(split_start=split)
        cases = [(Params(algo=LOCAL, start_pos=WITH_START, second_best=1, reverse_complement=1),
                  W.workload1(9000, seed=66)[0][1]),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, reverse_complement=1),
                  W.workload1(9000, seed=67)[2][1]),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=QUERY, tail=NONE), W.workload0(3000, seed=68)),
                 (Params(algo=LOCAL, start_pos=WITH_START), W.workload2(3000, seed=69)),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET), W.workload2(3000, seed=70))]
        for p, b in cases:
            got = gl.align(p, b).as_dict(p)
            exp = oracle_align(p, b).as_dict(p)
            for k, v in exp.items():
                assert np.array_equal(got[k], v), f"split={split} {p.key()} {k}"
    finally:
        gl.set_tuning(**saved)


def test_plain_form_matches_oracle():
    """The plain full-DP form (every pair one per thread in input order, no
    device work counter, no ordering, no warp kernels) gives the same results:
    it is the baseline the batched form is measured against."""
    from gasal_b200.capi import KSW, WITH_TB as TB
    saved = gl.get_tuning()
    try:
        gl.set_tuning(**gl.PLAIN_FORM)
        assert gl.get_tuning()["persistent"] == 0
        cases = [(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), W.workload2(2500, seed=71)),
                 (Params(algo=GLOBAL, start_pos=TB), W.workload2(2500, seed=72)),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, second_best=1),
                  W.workload1(3000, seed=73)[2][1]),
                 (Params(algo=KSW, zdrop=100), W.workload3(300, seed=74))]
        for p, b in cases:
            got = gl.align(p, b).as_dict(p)
            exp = oracle_align(p, b).as_dict(p)
            for k, v in exp.items():
                assert np.array_equal(got[k], v), f"plain {p.key()} {k}"
    finally:
        gl.set_tuning(**saved)


@pytest.mark.parametrize("group", [0, 8, 16, 32, 64])
def test_wc_lane_groups_match_oracle(group):
    """Warp-cooperative kernels with 32/group pairs per warp: every mode on
    mixed 50-1000 bp pairs with the cut at `group` words (so the shortest
    warp-cooperative pairs just meet the ring's bound), unrelated long pairs
    (start regions narrower than the group fall back to one lane), and batch
    sizes that leave groups of the last warp without a pair.  Group 0 picks
    the group per launch."""
    saved = gl.get_tuning()
    try:
        gl.set_tuning(wc_group=group, wc_min_qregs=group or 32)
        rng = np.random.default_rng(80 + group)
        from gasal_b200.capi import Batch
        qs = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(260, 700))).tolist()) for _ in range(2101)]
        ts = [bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(20, 700))).tolist()) for _ in range(2101)]
        unrelated = Batch.from_seqs(qs, ts)
        cases = [(Params(algo=LOCAL, start_pos=WITH_START, second_best=1), W.workload2(3003, seed=81)),
                 (Params(algo=LOCAL, start_pos=WITH_TB, second_best=1), W.workload2(2053, seed=82)),
                 (Params(algo=GLOBAL, start_pos=WITH_TB), W.workload2(3001, seed=83)),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, second_best=1),
                  W.workload2(3005, seed=84)),
                 (Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=QUERY, tail=TARGET), W.workload3(2051, seed=85)),
                 (Params(algo=LOCAL, start_pos=WITH_START, second_best=1), unrelated),
                 (Params(algo=GLOBAL), unrelated)]
        for p, b in cases:
            got = gl.align(p, b).as_dict(p)
            exp = oracle_align(p, b).as_dict(p)
            for k, v in exp.items():
                bad = np.nonzero(got[k] != v)[0]
                assert len(bad) == 0, f"group {group} {p.key()} {k}: {len(bad)} differ, first {bad[:5]}"
    finally:
        gl.set_tuning(**saved)


def test_long_prefix_runs_its_own_wc_launch():
    """Warp-cooperative pairs of 127+ query words (the length order's prefix)
    run as their own launch with their own lane group; mixed 50-5000 bp
    batches cover both launches, with traceback chunks of a small tile
    budget splitting the prefix across chunks."""
    saved = gl.get_tuning()
    try:
        gl.set_tuning(wc_group=0)
        parts = W.workload4(12000, seed=101)[:3]  # each launch above the ordering threshold
        for p, b in parts:
            assert int((b.q_len >= 1009).sum()) > 0 and int(((b.q_len >= 249) & (b.q_len < 1009)).sum()) > 0
            exp = oracle_align(p, b).as_dict(p)
            got = gl.align(p, b).as_dict(p)
            for k, v in exp.items():
                assert np.array_equal(got[k], v), f"{p.key()} {k}"
        p, b = parts[1]
        gl.set_tb_budget_mb(8)
        try:
            got = gl.align(p, b).as_dict(p)
        finally:
            gl.set_tb_budget_mb(98304)
        exp = oracle_align(p, b).as_dict(p)
        for k, v in exp.items():
            assert np.array_equal(got[k], v), f"chunked {p.key()} {k}"
    finally:
        gl.set_tuning(**saved)


@pytest.mark.parametrize("group", [0, 8, 16, 32, 64])
def test_wc_boundary_shapes(group):
    """Shapes at the edges of the warp-cooperative split, per lane group:
    queries of exactly 249/256 bases (the 32-word cut) and 1009/1016 bases
    (the 127-word cut of the separate long launch), targets of 0, 1 and 7
    bases, and a batch size that leaves groups of the last warp empty."""
    from gasal_b200.capi import Batch
    saved = gl.get_tuning()
    rng = np.random.default_rng(160 + group)

    def seq(n):
        return bytes(np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, n)])
    qs, ts = [], []
    for i in range(2081):
        ql = [249, 256, 1009, 1016, 300, 5000][i % 6]
        q = seq(ql)
        k = i % 5
        if k == 0:
            t = b""
        elif k == 1:
            t = seq(1)
        elif k == 2:
            t = seq(7)
        else:
            t = bytearray(q[: int(rng.integers(1, ql))])
            for _ in range(len(t) // 30 + 1):
                t[int(rng.integers(0, len(t)))] = b"ACGT"[int(rng.integers(0, 4))]
            t = bytes(t)
        qs.append(q)
        ts.append(t)
    b = Batch.from_seqs(qs, ts)
    try:
        gl.set_tuning(wc_group=group, wc_min_qregs=32)
        for p in (Params(algo=LOCAL, start_pos=WITH_START, second_best=1), Params(algo=GLOBAL, start_pos=WITH_TB),
                  Params(algo=LOCAL, start_pos=WITH_TB),
                  Params(algo=SEMI_GLOBAL, start_pos=WITH_START, head=TARGET, tail=TARGET, second_best=1)):
            got = gl.align(p, b).as_dict(p)
            exp = oracle_align(p, b).as_dict(p)
            for k, v in exp.items():
                if p.algo == GLOBAL and k == "score":
                    keep = b.t_len > 0  # the reference leaves empty-target GLOBAL scores undefined
                    assert np.array_equal(got[k][keep], v[keep]), f"group {group} {p.key()} {k}"
                elif k in ("cigar",):
                    continue
                else:
                    assert np.array_equal(got[k], v), f"group {group} {p.key()} {k}"
    finally:
        gl.set_tuning(**saved)
