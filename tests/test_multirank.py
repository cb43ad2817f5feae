"""Multi-GPU sharding logic, as world_size-2 gloo process groups on the CPU: the problems
of a batch and the requests of a serving stream are independent, so each rank takes a
deterministic share (no data-path collective) and only the per-rank results are gathered."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from fmm_gen_b200 import serve, tuner  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # batch problems
        shapes = tuner.random_batch_shapes(512, seed=0)
        choices, _ = tuner.BatchTuner().model_choice(shapes)
        mine = tuner.shard_problems(shapes, choices, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        # serving requests: each rank serves its share on a simulated GPU
        from tests.test_serve import SimClock, SimExecutor

        reqs = serve.poisson_requests(serve.Mix(rate=2000.0), 0.2, seed=9)
        share = serve.shard_requests(reqs, world)[rank]
        clk = SimClock()
        rep = serve.Server(SimExecutor(clk), clock=clk, sleep=clk.sleep).run(share, 0.2)
        stats = {"rids": sorted(r.rid for r in share), "lat": rep.latencies, "completed": rep.completed,
                 "offered": rep.offered}
        all_stats = [None] * world
        dist.all_gather_object(all_stats, stats)
        if rank == 0:
            out.put((got, all_stats))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_batch_and_requests_without_overlap():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got, stats = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = sorted(i for part in got for i in part)
    assert flat == list(range(512))
    shapes = tuner.random_batch_shapes(512, seed=0)
    choices, _ = tuner.BatchTuner().model_choice(shapes)
    m = tuner.B200Model()
    work = [sum(tuner.model_time(m, choices[i], *shapes[i]) for i in part) for part in got]
    assert max(work) / min(work) < 1.02
    rids = sorted(r for s in stats for r in s["rids"])
    reqs = serve.poisson_requests(serve.Mix(rate=2000.0), 0.2, seed=9)
    assert rids == [r.rid for r in reqs]
    assert sum(s["offered"] for s in stats) == len(reqs)
    lat = [x for s in stats for x in s["lat"]]
    assert len(lat) == sum(s["completed"] for s in stats) > 0
