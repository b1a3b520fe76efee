"""The multi-rank path of bench.py (one independent lattice per rank): the
max-over-ranks timing reduction and the whole-job throughput, run as two
gloo ranks on the CPU (the GPU run uses the same calls over NCCL)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = [3.0, 5.0][rank]  # the slower rank sets the job's time
        ms_max = bench.max_over_ranks(ms, dist, device="cpu")
        e2e = bench.max_over_ranks([0.2, 0.1][rank], dist, device="cpu")
        dist.barrier()
        out.put((rank, ms_max, e2e, bench.whole_job_mlups(4096 * 1024, 100, world, ms_max * 1e-3)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_rank_and_the_whole_job():
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
    for rank, ms_max, e2e, mlups in res:
        assert ms_max == 5.0 and e2e == 0.2
        assert mlups == pytest.approx(4096 * 1024 * 100 * 2 / 5e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.whole_job_mlups(10, 4, 1, 2.0) == pytest.approx(20e-6)
