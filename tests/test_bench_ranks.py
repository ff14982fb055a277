"""CPU: the multi-GPU bench harness (N independent replicas, one process per
GPU) on two gloo ranks: the job time is the slowest rank's, and the per-solve
figure divides the work of all ranks by it.  No GPU is touched."""
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
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, local = bench.dist_env()
    got = bench.max_over_ranks(100.0 + 50.0 * rank, w)
    out[rank] = (r, w, local, got, bench.job_ms_per_solve(got, 5, w))
    tdist.barrier()
    tdist.destroy_process_group()


def test_two_rank_job_time_is_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        for p in procs:  # a rank stuck in a collective must not outlive the test
            if p.is_alive():
                p.terminate()
                p.join(10)
        assert codes == [0, 0], codes
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (r, w, local, got, per) in res.items():
        assert (r, w, local) == (rank, 2, rank)
        assert got == 150.0
        assert per == pytest.approx(150.0 / 10)


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_ms_per_solve(35.0, 5, 1) == 7.0
