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
