"""Multi-rank host logic on CPU (gloo, world size 2): every rank runs its own replica, the
reported time is the maximum over ranks, and the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        skipped = bench.run_reference(type("A", (), {})(), rank) if rank != 0 else None
        out.put((rank, t, skipped))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]          # both ranks see the slowest rank's time
    assert res[1][2] == 0                                # rank 1 leaves the reference arm without work


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5


def test_balance_splits_cases_by_work():
    from water_flow_simulation_b200.batch import balance
    work = [19.1, 4.1, 13.2, 12.7, 6.6, 4.7, 12.0, 7.0, 8.1, 13.6, 8.1, 4.1]
    for parts in (1, 2, 3, 8):
        split = balance(work, parts)
        assert sorted(i for s in split for i in s) == list(range(len(work)))   # each case exactly once
        loads = [sum(work[i] for i in s) for s in split]
        assert max(loads) - min(loads) <= max(work)                            # greedy bound
    assert balance(work, 1) == [list(range(len(work)))]
    assert balance([5.0, 5.0, 1.0], 2) == [[0, 2], [1]]                        # ties go to the lowest index
    with pytest.raises(ValueError):
        balance(work, 0)
