"""Sweep runner: the reference's three experiment families on one GPU, measured beside the
performance model, written as CSV.

The reference writes one SLURM job per configuration whose script loops the generated test
driver over a size range (meta/sbatch_util.py:122-157) and compares the curves with its model
by eye (meta/model_gen.py:132-175).  The same families here, in one process:

    square   m = n = k = s
    rankk    m = n = 14400, k = s
    fixk     m = n = s,     k = 1024
    s = start, start + step, ..., end   (the reference: 240 .. 12000 step 240)

    python -m fmm_gen_b200.sweep square --algs 222-1,222-2,333-1 --start 2048 --end 8192 --step 2048 \
        --out square.csv

One row per (size, algorithm): effective GFLOPS of the FMM (ABC), of the classical kernel, the
B200 model's single-problem prediction for both (tuner.model_time_single), and the relative
difference between the two results.
"""
from __future__ import annotations

import argparse
import csv
import sys
from typing import Iterable, List, Sequence, Tuple

from . import tuner

FAMILIES = ("square", "rankk", "fixk")


def shapes(family: str, sizes: Iterable[int]) -> List[Tuple[int, int, int]]:
    if family == "square":
        return [(s, s, s) for s in sizes]
    if family == "rankk":
        return [(14400, 14400, s) for s in sizes]
    if family == "fixk":
        return [(s, s, 1024) for s in sizes]
    raise ValueError(f"unknown family {family!r} (one of {', '.join(FAMILIES)})")


def model_gflops(alg: str, m: int, n: int, k: int, model: tuner.B200Model) -> float:
    return 2.0 * m * n * k / tuner.model_time_single(model, alg, m, n, k) / 1e9


HEADER = ["family", "algorithm", "m", "n", "k", "gflops_fmm", "gflops_gemm", "model_gflops_fmm",
          "model_gflops_gemm", "rel_diff"]


def run(family: str, algs: Sequence[str], sizes: Sequence[int], reps: int = 3, out=None) -> List[dict]:
    import torch

    from . import runtime as rt

    model = tuner.B200Model()
    writer = csv.DictWriter(out, fieldnames=HEADER) if out is not None else None
    if writer:
        writer.writeheader()
    plans = {a: rt.Plan.from_levels(*tuner.candidate_levels(a)) for a in algs}
    g = torch.Generator(device="cuda").manual_seed(0)

    def best(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return min(ts)

    rows = []
    for (m, n, k) in shapes(family, sizes):
        A = rt.colmajor(m, k, device="cuda").uniform_(0, 1, generator=g)
        B = rt.colmajor(k, n, device="cuda").uniform_(0, 1, generator=g)
        Cr = rt.colmajor(m, n, device="cuda").zero_()
        t_gemm = best(lambda: rt.plain_gemm(A, B, Cr))
        Cr.zero_()
        rt.plain_gemm(A, B, Cr)
        gf = 2.0 * m * n * k / 1e9
        for a in algs:
            C = rt.colmajor(m, n, device="cuda").zero_()
            t_fmm = best(lambda: rt.fmm_gemm(plans[a], A, B, C, "abc"))
            C.zero_()
            rt.fmm_gemm(plans[a], A, B, C, "abc")
            diff = ((C - Cr).norm() / Cr.norm()).item()
            row = {"family": family, "algorithm": a, "m": m, "n": n, "k": k, "gflops_fmm": gf / t_fmm,
                   "gflops_gemm": gf / t_gemm, "model_gflops_fmm": model_gflops(a, m, n, k, model),
                   "model_gflops_gemm": model_gflops("classical", m, n, k, model), "rel_diff": diff}
            rows.append(row)
            if writer:
                writer.writerow(row)
                out.flush()
            del C
        del A, B, Cr
        torch.cuda.empty_cache()
    return rows


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("family", choices=FAMILIES)
    ap.add_argument("--algs", default="222-1", help="comma-separated, e.g. 222-1,222-2,222-1_333-1")
    ap.add_argument("--start", type=int, default=240)
    ap.add_argument("--end", type=int, default=12000)
    ap.add_argument("--step", type=int, default=240)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default="-")
    a = ap.parse_args(argv)
    sizes = list(range(a.start, a.end + 1, a.step))
    algs = [x for x in a.algs.split(",") if x]
    if a.out == "-":
        run(a.family, algs, sizes, a.reps, sys.stdout)
    else:
        with open(a.out, "w", newline="") as fh:
            run(a.family, algs, sizes, a.reps, fh)


if __name__ == "__main__":
    main()
