"""Host side of the mixed dispatch: the argument check of gb_align_dev_mixed
(gb_mixed_check, no CUDA call) and the batch concatenation helper."""
import numpy as np
import pytest

from gasal_b200 import lib as gl
from gasal_b200 import workloads as W
from gasal_b200.capi import Params, LOCAL, GLOBAL, KSW, WITH_START
from gasal_b200.lib import GasalError


def test_mixed_check_counts_and_rejects():
    kinds = [Params(algo=LOCAL, start_pos=WITH_START), Params(algo=KSW), Params(algo=GLOBAL)]
    kind = np.array([0, 1, 2, 2, 1, 0, 0], np.uint8)
    assert gl.mixed_check(kinds, kind).tolist() == [3, 2, 2]
    with pytest.raises(GasalError):
        gl.mixed_check(kinds, np.array([0, 3], np.uint8))  # kind index out of range
    with pytest.raises(GasalError):
        gl.mixed_check(kinds, np.array([1], np.uint8), has_seed=False)  # ksw pairs need seeds
    assert gl.mixed_check(kinds, np.array([0, 2], np.uint8), has_seed=False).tolist() == [1, 0, 1]
    with pytest.raises(GasalError):
        gl.mixed_check([Params(algo=4)], np.zeros(1, np.uint8))  # no such algorithm
    with pytest.raises(GasalError):
        gl.mixed_check(kinds * 3, np.zeros(1, np.uint8))  # more than 8 kinds
    assert gl.mixed_check(kinds, np.zeros(0, np.uint8)).tolist() == [0, 0, 0]


def test_concat_parts_keeps_every_pair():
    parts = W.workload1(900, seed=3)
    kinds, b, kind, idx = W.concat_parts(parts, shuffle_seed=1)
    assert [k.key() for k in kinds] == [p.key() for p, _ in parts]
    assert b.n == sum(pb.n for _, pb in parts)
    assert np.bincount(kind).tolist() == [pb.n for _, pb in parts]
    for j in range(b.n):
        pb = parts[int(kind[j])][1]
        i = int(idx[j])
        assert b.q_len[j] == pb.q_len[i] and b.t_len[j] == pb.t_len[i]
        assert np.array_equal(b.q[b.q_off[j]:b.q_off[j] + b.q_len[j]], pb.q[pb.q_off[i]:pb.q_off[i] + pb.q_len[i]])
        assert np.array_equal(b.t[b.t_off[j]:b.t_off[j] + b.t_len[j]], pb.t[pb.t_off[i]:pb.t_off[i] + pb.t_len[i]])
        if pb.q_op is not None:
            assert b.q_op[j] == pb.q_op[i] and b.t_op[j] == pb.t_op[i]
    # every pair's offset is distinct and 8-aligned, so CIGAR bytes land apart
    assert len(set(b.q_off.tolist())) == b.n and not (b.q_off % 8).any()
