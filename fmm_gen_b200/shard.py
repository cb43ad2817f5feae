"""One large FMM GEMM over several GPUs: a 2-D split of C over a pr x pc process grid.

The reference's only parallel split is the OpenMP range of each product's rows inside one
process (meta/abc_gen_mix.py:357, common/dgemm/bl_dgemm_util.c:189-280).  Across GPUs the
natural split of C += A*B is over C: rank (i, j) of the grid owns C[I_i, J_j] and computes
C[I_i, J_j] += A[I_i, :] * B[:, J_j] as an FMM call of its own (with its own partition and
fringes, so its rounding differs from a single-GPU call of the whole problem, within the same
error bound).  No reduction is needed; the exchange is one all-gather per operand:

  * A starts distributed as blocks A[I_i, K^a_j] (rank (i, j) holds the j-th of pc slices of
    its row panel's k range); an all-gather over the ranks of grid row i assembles A[I_i, :].
  * B starts as blocks B[K^b_i, J_j] (the i-th of pr slices of its column panel's k range);
    an all-gather over grid column j assembles B[:, J_j].

Row and column ranges fall on multiples of a unit (128 x the plan's block rows / columns), so
every local FMM call's sub-blocks are whole 128-row tiles where the size allows.  Every rank
takes the same collective steps in the same order (group creation included).  With NCCL the
gathered panels land in each GPU's own memory; the local call then reads only local memory.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Sequence, Tuple


def process_grid(world: int) -> Tuple[int, int]:
    """pr x pc = world with pr <= pc and pr as large as possible (near square)."""
    pr = int(math.isqrt(world))
    while world % pr:
        pr -= 1
    return pr, world // pr


def split_range(total: int, parts: int, unit: int) -> List[Tuple[int, int]]:
    """`parts` consecutive ranges covering [0, total), edges on multiples of `unit` where the
    size allows (the last range takes the remainder); empty ranges only when total < parts."""
    edges = [0]
    for p in range(1, parts):
        e = total * p // parts
        if total // parts >= unit:
            e -= e % unit
        edges.append(max(edges[-1], min(e, total)))
    edges.append(total)
    return [(edges[p], edges[p + 1]) for p in range(parts)]


@dataclass
class Block2D:
    """What rank (i, j) of a pr x pc grid owns and computes."""
    i: int
    j: int
    rows: Tuple[int, int]     # I_i: rows of A and C
    cols: Tuple[int, int]     # J_j: columns of B and C
    a_k: Tuple[int, int]      # K^a_j: the k slice of A[I_i, :] this rank starts with
    b_k: Tuple[int, int]      # K^b_i: the k slice of B[:, J_j] this rank starts with
    a_ks: List[Tuple[int, int]]  # every rank of grid row i's slice of k (gather order)
    b_ks: List[Tuple[int, int]]  # every rank of grid column j's slice of k


def block_of(rank: int, world: int, m: int, n: int, k: int, unit_m: int = 128, unit_n: int = 128) -> Block2D:
    pr, pc = process_grid(world)
    i, j = divmod(rank, pc)
    rows = split_range(m, pr, unit_m)[i]
    cols = split_range(n, pc, unit_n)[j]
    a_ks = split_range(k, pc, 8)
    b_ks = split_range(k, pr, 8)
    return Block2D(i, j, rows, cols, a_ks[j], b_ks[i], a_ks, b_ks)


class Gemm2D:
    """C += A*B of an m x n x k problem split over `world` ranks (torch.distributed must be
    initialised; NCCL on GPUs, gloo on CPUs).  Construct on every rank in the same order: it
    creates the grid's row and column groups."""

    def __init__(self, m: int, n: int, k: int, dims: Sequence[int] = (1, 1, 1)):
        import torch.distributed as dist

        self.dist = dist
        self.world, self.rank = dist.get_world_size(), dist.get_rank()
        self.m, self.n, self.k = m, n, k
        self.pr, self.pc = process_grid(self.world)
        self.blk = block_of(self.rank, self.world, m, n, k, 128 * dims[0], 128 * dims[2])
        self.row_group = self.col_group = None
        for i in range(self.pr):  # every rank creates every group, in the same order
            g = dist.new_group([i * self.pc + j for j in range(self.pc)])
            if i == self.blk.i:
                self.row_group = g
        for j in range(self.pc):
            g = dist.new_group([i * self.pc + j for i in range(self.pr)])
            if j == self.blk.j:
                self.col_group = g

    def gather_a(self, A_own):
        """A[I_i, K^a_j] (column-major, |I_i| x |K^a_j|) -> A[I_i, :] (column-major)."""
        import torch

        if self.pc == 1:  # one rank in the grid row: its slice is the whole panel
            return A_own
        rows = self.blk.rows[1] - self.blk.rows[0]
        width = max(b - a for a, b in self.blk.a_ks)
        # column-major |I| x w is row-major w x |I|: pieces stack along k
        buf = torch.zeros((width, rows), dtype=A_own.dtype, device=A_own.device)
        kk = A_own.shape[1]
        buf[:kk].copy_(A_own.t())
        parts = [buf]
        if self.pc > 1:
            parts = [torch.empty_like(buf) for _ in range(self.pc)]
            self.dist.all_gather(parts, buf, group=self.row_group)
        full = torch.cat([p[: b - a] for p, (a, b) in zip(parts, self.blk.a_ks)], dim=0)
        return full.t()  # |I| x k, column-major view

    def gather_b(self, B_own):
        """B[K^b_i, J_j] (column-major, |K^b_i| x |J_j|) -> B[:, J_j] (column-major)."""
        import torch

        if self.pr == 1:
            return B_own
        cols = self.blk.cols[1] - self.blk.cols[0]
        width = max(b - a for a, b in self.blk.b_ks)
        buf = torch.zeros((cols, width), dtype=B_own.dtype, device=B_own.device)  # row-major |J| x w
        kk = B_own.shape[0]
        buf[:, :kk].copy_(B_own.t())
        parts = [buf]
        if self.pr > 1:
            parts = [torch.empty_like(buf) for _ in range(self.pr)]
            self.dist.all_gather(parts, buf, group=self.col_group)
        full = torch.cat([p[:, : b - a] for p, (a, b) in zip(parts, self.blk.b_ks)], dim=1).contiguous()
        return full.t()  # k x |J|, column-major view

    def run(self, A_own, B_own, C_own, local_gemm: Callable) -> None:
        """C[I_i, J_j] += A[I_i, :] * B[:, J_j]: gather both panels, then local_gemm(A, B, C)."""
        A = self.gather_a(A_own)
        B = self.gather_b(B_own)
        if C_own.numel():
            local_gemm(A, B, C_own)

    def k_chunks(self) -> List[Tuple[int, int]]:
        """The k range cut at every edge of both starting distributions: each chunk lies in one
        rank's A slice (of this grid row) and in one rank's B slice (of this grid column)."""
        edges = sorted({e for ab in (self.blk.a_ks, self.blk.b_ks) for r in ab for e in r})
        return [(e0, e1) for e0, e1 in zip(edges, edges[1:]) if e1 > e0]

    def run_pipelined(self, A_own, B_own, C_own, local_gemm: Callable) -> None:
        """C[I_i, J_j] += A[I_i, :] * B[:, J_j] in k chunks (a SUMMA order): the owner of a chunk's
        A[I_i, K_q] broadcasts it over the grid row and the owner of B[K_q, J_j] over the grid
        column, and chunk q + 1's broadcasts are in flight while chunk q's local GEMM runs.  The
        exchange then hides behind the compute; each chunk is a GEMM of its own, so the rounding
        differs from run()'s (within the same error bound)."""
        import torch

        dist, blk = self.dist, self.blk
        rows = blk.rows[1] - blk.rows[0]
        cols = blk.cols[1] - blk.cols[0]
        chunks = self.k_chunks()
        owner_a = [next(j for j, (a, b) in enumerate(blk.a_ks) if a <= k0 and k1 <= b) for k0, k1 in chunks]
        owner_b = [next(i for i, (a, b) in enumerate(blk.b_ks) if a <= k0 and k1 <= b) for k0, k1 in chunks]

        def fetch(q):
            k0, k1 = chunks[q]
            w = k1 - k0
            works = []
            # A[I, K_q]: a column-major view of this rank's slice when the grid row is this rank
            # alone, else a row-major (w, rows) buffer (= column-major rows x w) broadcast by its owner
            if self.pc == 1:
                a = A_own[:, k0 - blk.a_k[0]:k1 - blk.a_k[0]]
            else:
                if owner_a[q] == blk.j:
                    buf = A_own[:, k0 - blk.a_k[0]:k1 - blk.a_k[0]].t().contiguous()
                else:
                    buf = torch.empty((w, rows), dtype=A_own.dtype, device=A_own.device)
                works.append(dist.broadcast(buf, src=blk.i * self.pc + owner_a[q], group=self.row_group, async_op=True))
                a = buf.t()
            # B[K_q, J] likewise (row-major (cols, w) buffer = column-major w x cols)
            if self.pr == 1:
                b = B_own[k0 - blk.b_k[0]:k1 - blk.b_k[0], :]
            else:
                if owner_b[q] == blk.i:
                    buf = B_own[k0 - blk.b_k[0]:k1 - blk.b_k[0], :].t().contiguous()
                else:
                    buf = torch.empty((cols, w), dtype=B_own.dtype, device=B_own.device)
                works.append(dist.broadcast(buf, src=owner_b[q] * self.pc + blk.j, group=self.col_group, async_op=True))
                b = buf.t()
            return a, b, works

        nxt = fetch(0) if chunks else None
        for q in range(len(chunks)):
            a, b, works = nxt
            for wk in works:
                wk.wait()
            nxt = fetch(q + 1) if q + 1 < len(chunks) else None
            if C_own.numel():
                local_gemm(a, b, C_own)
