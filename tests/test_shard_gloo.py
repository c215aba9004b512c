"""The multi-GPU path's host logic on CPU: two gloo ranks each build their
own shard, align it with the scalar oracle, and agree on the job time as the
maximum over ranks.  No GPU and no data-path collective are involved."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from gasal_b200 import shard, workloads as W
    from oracle.bindings import oracle_align
    r, w, lr = shard.rank_info()
    assert (r, w, lr) == (rank, world, rank)
    parts = W.workload1(600, seed=shard.shard_seed(W.SEED_BASE + 1, r))
    scores = np.concatenate([oracle_align(p, b, threads=1).score for p, b in parts])
    my_ms = 10.0 * (rank + 1)
    job_ms = shard.max_over_ranks(my_ms, dist)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), scores=scores, job_ms=job_ms,
             q0=parts[0][1].q[:64])
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"r{k}.npz") for k in (0, 1))
    assert float(r0["job_ms"]) == float(r1["job_ms"]) == 20.0          # max over ranks
    assert len(r0["scores"]) == len(r1["scores"]) == 600                # weak scaling: full shard per rank
    assert not np.array_equal(r0["q0"], r1["q0"])                       # ranks hold different pairs
    from gasal_b200 import shard
    assert shard.job_throughput(600, 2, 1, 20.0) == pytest.approx(60000.0)


def test_shard_range_partitions():
    from gasal_b200 import shard
    for n in (0, 1, 7, 1000):
        for w in (1, 2, 3, 8):
            spans = [shard.shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_cell_shard_range_balances_work():
    from gasal_b200 import shard, workloads as W
    parts = W.workload4(40000, seed=3)
    cells = np.concatenate([b.q_len.astype(np.int64) * b.t_len for _, b in parts])
    for w in (1, 2, 3, 4, 8):
        spans = [shard.cell_shard_range(cells, r, w) for r in range(w)]
        assert spans[0][0] == 0 and spans[-1][1] == len(cells)
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        work = [cells[lo:hi].sum() for lo, hi in spans]
        # every slice within one pair's worth of the even share
        assert max(work) - min(work) <= 2 * cells.max(), (w, work)
    assert shard.cell_shard_range(np.zeros(0), 0, 2) == (0, 0)
    assert [shard.cell_shard_range(np.zeros(5), r, 2) for r in range(2)] == [(0, 3), (3, 5)]


def _strong_main(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from gasal_b200 import shard, workloads as W
    from oracle.bindings import oracle_align
    b = W.workload2(900, seed=17)                      # one batch, the same on every rank
    cells = b.q_len.astype(np.int64) * b.t_len
    lo, hi = shard.cell_shard_range(cells, rank, world)
    from gasal_b200.capi import Params, GLOBAL
    mine = b.subset(np.arange(lo, hi))
    scores = oracle_align(Params(algo=GLOBAL), mine, threads=1).score
    np.savez(os.path.join(out_dir, f"s{rank}.npz"), lo=lo, hi=hi, scores=scores, work=cells[lo:hi].sum())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_strong_split_of_one_batch(tmp_path):
    """A strong split: two ranks take cell-balanced slices of one batch; the
    concatenated results equal the whole batch aligned at once."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_strong_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    s0, s1 = (np.load(tmp_path / f"s{k}.npz") for k in (0, 1))
    assert int(s0["lo"]) == 0 and int(s0["hi"]) == int(s1["lo"]) and int(s1["hi"]) == 900
    from gasal_b200 import workloads as W
    from gasal_b200.capi import Params, GLOBAL
    from oracle.bindings import oracle_align
    whole = oracle_align(Params(algo=GLOBAL), W.workload2(900, seed=17), threads=1).score
    assert np.array_equal(np.concatenate([s0["scores"], s1["scores"]]), whole)
    w0, w1 = float(s0["work"]), float(s1["work"])
    assert abs(w0 - w1) / (w0 + w1) < 0.05
