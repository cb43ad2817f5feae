"""Test driver of a generated configuration: one FMM C += A*B and the classical GEMM on
the GPU, printed as the reference's generated driver prints it
(meta/misc_gen.py:147-261): `m n k GFLOPS_fmm GFLOPS_gemm` (min over repeats), plus the
relative Frobenius difference between the two results.

    python -m fmm_gen_b200.testdriver 222-1_333-1_abc 4096 4096 4096 [--reps 3]

Two more modes of this project (no counterpart in the reference):
    --split           FP32 inputs through the split-BF16 tensor-core path (the job's pack
                      type is ignored); the line adds the relative error of both results
                      against an FP64 product of the same inputs.
    --batch COUNT     COUNT problems with m, n, k log-uniform in [256, m] (seed 0) in one
                      batch launch, every problem on the job's plan; prints the batch's
                      effective GFLOPS and the all-classical batch's.
"""
from __future__ import annotations

import argparse
import re


def parse_job(job: str):
    """'222-1_333-1_abc' -> (['222', '333'], [1, 1], 'abc')"""
    parts = job.split("_")
    pack = parts[-1]
    algs, levels = [], []
    for p in parts[:-1]:
        m = re.fullmatch(r"(.+)-(\d+)", p)
        if not m:
            raise ValueError(f"bad job name {job!r}")
        algs.append(m.group(1))
        levels.append(int(m.group(2)))
    return algs, levels, pack


def main(argv=None):
    import torch

    from . import runtime as rt

    ap = argparse.ArgumentParser()
    ap.add_argument("job")
    ap.add_argument("m", type=int)
    ap.add_argument("n", type=int)
    ap.add_argument("k", type=int)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--split", action="store_true")
    ap.add_argument("--batch", type=int, default=0)
    a = ap.parse_args(argv)
    algs, levels, pack = parse_job(a.job)
    plan = rt.Plan.from_levels(algs, levels)
    if a.split:
        return split_mode(a, plan)
    if a.batch:
        return batch_mode(a, plan)
    g = torch.Generator(device="cuda").manual_seed(0)
    A = rt.colmajor(a.m, a.k, device="cuda").uniform_(0, 1, generator=g)
    B = rt.colmajor(a.k, a.n, device="cuda").uniform_(0, 1, generator=g)
    C = rt.colmajor(a.m, a.n, device="cuda").zero_()
    Cr = rt.colmajor(a.m, a.n, device="cuda").zero_()

    def best(fn):
        ts = []
        for _ in range(a.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return min(ts)

    t_fmm = best(lambda: rt.fmm_gemm(plan, A, B, C, pack))
    t_gemm = best(lambda: rt.plain_gemm(A, B, Cr))
    diff = ((C - Cr).norm() / Cr.norm()).item()
    gf = 2.0 * a.m * a.n * a.k / 1e9
    print(f"{a.m:5d}\t {a.n:5d}\t {a.k:5d}\t {gf / t_fmm:5.2f}\t {gf / t_gemm:5.2f}\t rel_diff={diff:.2e}", flush=True)


def _best(torch, fn, reps):
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
    return min(ts)


def split_mode(a, plan):
    import torch

    from . import runtime as rt

    g = torch.Generator(device="cuda").manual_seed(0)
    A = rt.colmajor(a.m, a.k, dtype=torch.float32, device="cuda").normal_(generator=g)
    B = rt.colmajor(a.k, a.n, dtype=torch.float32, device="cuda").normal_(generator=g)
    C = rt.colmajor(a.m, a.n, device="cuda").zero_()
    Cr = rt.colmajor(a.m, a.n, device="cuda").zero_()
    t_fmm = _best(torch, lambda: (C.zero_(), rt.split_gemm(plan, A, B, C)), a.reps)
    t_gemm = _best(torch, lambda: (Cr.zero_(), rt.split_gemm(None, A, B, Cr)), a.reps)
    ref = A.double() @ B.double()
    e1 = ((C - ref).norm() / ref.norm()).item()
    e2 = ((Cr - ref).norm() / ref.norm()).item()
    gf = 2.0 * a.m * a.n * a.k / 1e9
    print(f"{a.m:5d}\t {a.n:5d}\t {a.k:5d}\t {gf / t_fmm:5.2f}\t {gf / t_gemm:5.2f}\t "
          f"rel_err_fmm={e1:.2e} rel_err_gemm={e2:.2e}", flush=True)


def batch_mode(a, plan):
    import torch

    from . import runtime as rt
    from .tuner import random_batch_shapes

    shapes = random_batch_shapes(a.batch, lo=256, hi=max(a.m, 256), seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    As = [rt.colmajor(m, k, device="cuda").uniform_(0, 1, generator=g) for (m, n, k) in shapes]
    Bs = [rt.colmajor(k, n, device="cuda").uniform_(0, 1, generator=g) for (m, n, k) in shapes]
    Cs = [rt.colmajor(m, n, device="cuda").zero_() for (m, n, k) in shapes]
    fmm_b = rt.Batch(shapes, [plan] * len(shapes))
    cls_b = rt.Batch(shapes)
    t_fmm = _best(torch, lambda: fmm_b.run(As, Bs, Cs), a.reps)
    t_gemm = _best(torch, lambda: cls_b.run(As, Bs, Cs), a.reps)
    gf = sum(2.0 * m * n * k for (m, n, k) in shapes) / 1e9
    print(f"batch {len(shapes)} (dims log-uniform in [256, {max(a.m, 256)}])\t {gf / t_fmm:5.2f}\t "
          f"{gf / t_gemm:5.2f}", flush=True)


if __name__ == "__main__":
    main()
