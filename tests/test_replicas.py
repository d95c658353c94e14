"""The bench's replica path on two gloo ranks on the CPU: each rank takes its own seeded tiles and
the job's figures combine as the max time and the summed paths."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as tdist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _, steps, _ = bench.workload("road", rank, 8, 1000)
        timing = dict(kernel_ms=10.0 * (rank + 1), wall_s=0.5 + rank, paint_ms=9.0 * (rank + 1))
        total = bench.combine_ranks(timing, 100 + rank, "cpu")
        out.put((rank, total, timing, len(steps)))
    finally:
        tdist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_combine_max_time_and_summed_paths():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, timing, n_steps in results:
        assert total == 201
        assert timing == dict(kernel_ms=20.0, wall_s=1.5, paint_ms=18.0)
        assert n_steps == 1

