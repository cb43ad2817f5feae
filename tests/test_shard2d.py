"""One GEMM split 2-D over ranks (fmm_gen_b200.shard), as gloo process groups on the CPU:
each rank starts with one k slice of its A row panel and of its B column panel, gathers both
panels over its grid row / column (or, in k chunks, receives each chunk from its owner while the
previous chunk computes), and computes its C block; the assembled C equals C0 + A*B.  The local GEMM here is torch's FP64 CPU matmul (on GPUs it is the library's FMM)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from fmm_gen_b200 import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cm(x):
    """A column-major copy (stride(0) == 1), as the library's operands are laid out."""
    return x.t().contiguous().t()


def _worker(rank, world, port, shape, out, pipelined=False):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, n, k = shape
        g = torch.Generator().manual_seed(11)
        A = torch.rand(m, k, generator=g, dtype=torch.float64) * 2 - 1
        B = torch.rand(k, n, generator=g, dtype=torch.float64) * 2 - 1
        C0 = torch.rand(m, n, generator=g, dtype=torch.float64) * 2 - 1
        gm = shard.Gemm2D(m, n, k)
        b = gm.blk
        (r0, r1), (c0, c1) = b.rows, b.cols
        A_own = _cm(A[r0:r1, b.a_k[0]:b.a_k[1]])
        B_own = _cm(B[b.b_k[0]:b.b_k[1], c0:c1])
        C_own = _cm(C0[r0:r1, c0:c1])

        def local(Ap, Bp, Cp):
            assert Ap.stride(0) == 1 and Bp.stride(0) == 1
            Cp += Ap @ Bp

        (gm.run_pipelined if pipelined else gm.run)(A_own, B_own, C_own, local)
        blocks = [None] * world
        dist.all_gather_object(blocks, (b.rows, b.cols, C_own.clone()))
        if rank == 0:
            C = torch.empty(m, n, dtype=torch.float64)
            seen = torch.zeros(m, n, dtype=torch.int32)
            for (ra, rb), (ca, cb), blk in blocks:
                C[ra:rb, ca:cb] = blk
                seen[ra:rb, ca:cb] += 1
            want = C0 + A @ B
            out.put((bool((seen == 1).all()), float((C - want).abs().max()), gm.pr, gm.pc))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("pipelined", [False, True], ids=["gathered", "k_chunks"])
@pytest.mark.parametrize("world,shape", [(2, (300, 520, 260)), (4, (384, 700, 333))])
def test_2d_split_assembles_the_whole_product(world, shape, pipelined):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, shape, q, pipelined)) for r in range(world)]
    for p in procs:
        p.start()
    covered, err, pr, pc = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert covered  # every C element computed exactly once
    assert err < 1e-12
    assert pr * pc == world and pr <= pc


def test_grid_and_ranges():
    assert shard.process_grid(1) == (1, 1)
    assert shard.process_grid(2) == (1, 2)
    assert shard.process_grid(4) == (2, 2)
    assert shard.process_grid(8) == (2, 4)
    r = shard.split_range(16384, 4, 768)
    assert r[0][0] == 0 and r[-1][1] == 16384
    assert all(a % 768 == 0 for a, _ in r)
    assert all(b > a for a, b in r)
    small = shard.split_range(3, 4, 128)  # fewer elements than parts: some ranges are empty
    assert sum(b - a for a, b in small) == 3 and small[0][0] == 0 and small[-1][1] == 3
