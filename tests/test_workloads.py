"""The seeded workload generators produce the shapes the benchmark lines
name (lengths, mixes, launch splits) and are reproducible."""
import numpy as np

from gasal_b200 import workloads as W
from gasal_b200.capi import KSW, LOCAL, SEMI_GLOBAL, WITH_TB


def _check_layout(b):
    assert (b.q_off % 8 == 0).all() and (b.t_off % 8 == 0).all()
    assert int(b.q_off[-1]) + int(b.q_len[-1]) <= b.q.shape[0]
    assert int(b.t_off[-1]) + int(b.t_len[-1]) <= b.t.shape[0]


def test_workload1_shape():
    parts = W.workload1(3000, seed=5)
    assert [p.algo for p, _ in parts] == [p.algo for p in W.WORKLOAD1_PARAMS]
    for _, b in parts:
        _check_layout(b)
        assert (b.q_len == 150).all() and b.t_len.min() >= 150 and b.t_len.max() <= 300
        assert 0.4 < (b.q_op != 0).mean() < 0.6


def test_workload3_shape():
    b = W.workload3(2000, seed=6)
    _check_layout(b)
    assert b.q_len.min() >= 250 and b.q_len.max() <= 2000
    assert b.seed.min() >= 20 and b.seed.max() <= 60


def test_workload4_mix_and_split():
    parts = W.workload4(20000, seed=7)
    assert [(p.algo, p.start_pos) for p, _ in parts] == [(p.algo, p.start_pos) for p in W.WORKLOAD4_PARAMS]
    n = sum(b.n for _, b in parts)
    assert n == 20000
    tb = [b.n for p, b in parts if p.start_pos == WITH_TB][0]
    assert abs(tb / n - 0.20) < 0.01
    allq = np.concatenate([b.q_len for _, b in parts])
    assert allq.min() >= 50 and allq.max() <= 5000
    assert 200 < np.median(allq) < 300
    for _, b in parts:
        _check_layout(b)
    again = W.workload4(20000, seed=7)
    assert all(np.array_equal(a.q, c.q) and np.array_equal(a.t, c.t) for (_, a), (_, c) in zip(parts, again))


def test_pairs_do_not_depend_on_threads_or_batch_size():
    """Each pair has its own xoshiro256** stream keyed by (seed, pair index)."""
    a = W.generate(4, 3000, seed=11, threads=1)[0]
    b = W.generate(4, 3000, seed=11, threads=4)[0]
    assert np.array_equal(a.q, b.q) and np.array_equal(a.t, b.t) and np.array_equal(a.seed, b.seed)
    big = W.generate(4, 5000, seed=11)[0]
    for i in (0, 1, 1234, 2999):
        assert a.seq(i, "q") == big.seq(i, "q") and a.seq(i, "t") == big.seq(i, "t")
    other = W.generate(4, 3000, seed=12)[0]
    assert not np.array_equal(a.q_len, other.q_len)


def test_workload_shapes_and_padding():
    b0 = W.workload0(4000, seed=3)
    _check_layout(b0)
    assert b0.q_len.min() >= 100 and b0.q_len.max() <= 150
    assert (b0.t_len >= b0.q_len - 10).all()
    for b in (b0, W.workload2(2000, seed=4)):
        for i in (0, 17, b.n - 1):
            o, n = int(b.q_off[i]), int(b.q_len[i])
            assert (b.q[o + n:o + ((n + 7) // 8) * 8] == ord("N")).all()
    b2 = W.workload2(4000, seed=4)
    assert b2.q_len.min() >= 50 and b2.q_len.max() <= 1000 and b2.t_len.min() >= 1
    # unrelated pairs exist in workload 4: identity near 1/4 for some pairs
    p, b4 = W.workload4(4000, seed=9)[0]
    ident = []
    for i in range(200):
        q, t = b4.seq(i, "q"), b4.seq(i, "t")
        m = min(len(q), len(t))
        ident.append(np.mean(np.frombuffer(q[:m], np.uint8) == np.frombuffer(t[:m], np.uint8)))
    assert min(ident) < 0.4 and max(ident) > 0.9
