"""Test driver of a generated configuration: one FMM C += A*B and the classical GEMM on
the GPU, printed as the reference's generated driver prints it
(meta/misc_gen.py:147-261): `m n k GFLOPS_fmm GFLOPS_gemm` (min over repeats), plus the
relative Frobenius difference between the two results.

    python -m fmm_gen_b200.testdriver 222-1_333-1_abc 4096 4096 4096 [--reps 3]
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
    a = ap.parse_args(argv)
    algs, levels, pack = parse_job(a.job)
    plan = rt.Plan.from_levels(algs, levels)
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


if __name__ == "__main__":
    main()
