"""The multi-GPU path is replicas: every rank solves its own rows, and the
only collectives are the measurement's barrier and max-over-ranks.  This
runs that plumbing (gpusim2grid_b200.replicas, used by bench.py) as two
gloo ranks on the CPU."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from gpusim2grid_b200 import replicas
    info = replicas.init("gloo", timeout_s=60)
    replicas.barrier(device_sync=False)
    mx = replicas.max_over_ranks(10.0 + 3 * rank)
    total = replicas.sum_over_ranks(100 * (rank + 1))
    b, e = replicas.shard_rows(11, info.rank, info.world)
    replicas.finish()
    q.put((info.rank, info.world, mx, total, b, e))


def test_two_gloo_ranks_reduce_and_shard():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 13.0 for o in out)      # the slowest rank's time
    assert all(o[3] == 300.0 for o in out)
    assert [(o[4], o[5]) for o in out] == [(0, 6), (6, 11)]


def test_shard_rows_covers_every_row_once():
    from gpusim2grid_b200.replicas import shard_rows
    for n in (0, 1, 7, 2847):
        for world in (1, 2, 3, 8):
            spans = [shard_rows(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_rows(5, 2, 2)


def test_single_process_needs_no_group():
    from gpusim2grid_b200 import replicas
    assert replicas.max_over_ranks(4.5) == 4.5
    assert replicas.rank_info().world >= 1
