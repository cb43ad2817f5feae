#!/usr/bin/env python
"""Benchmark of the generated FMM GEMM on B200: effective TFLOPS = 2mnk/t.

Workload (one step): the two-level hybrid 222-1 x 333-1 (Strassen x Smirnov <3,3,3;23>),
pack type abc, FP64 column-major C += A*B on the three shapes of that configuration:
16384^3, 14400x14400x480 (rank-k) and 4000x16000x2000, with A, B, C ~ U(-1,1) from a
seed.  Inputs stay resident in HBM; every step touches ~8.5 GB, far more than the
126 MB L2, so no extra L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`e2e` is the same metric through the host C ABI (fmm_dgemm_host, pinned host buffers, every
copy inside the timed region), the step's three calls issued from three host threads so that
one call's copies overlap another's compute; `e2e.serial_value` issues them one after another.

One JSON line on rank 0.  Under torchrun (N > 1) every rank runs the same workload on
its own inputs (independent replicas: a single GEMM is not split across GPUs), and the
value is the sum over ranks divided by the slowest rank's device time.
`--impl reference` times the reference's own generated multithreaded code for this job on
the host cores instead (oracle/_ref/fmm, built from an fmm-gen checkout by
oracle/build_ref_fmm.py; the oracle, its CPU restatement, where those libraries are absent),
on rank 0 only.
"""
from __future__ import annotations

import argparse
import csv
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALGS, LEVELS, PACK = ["222", "333"], [1, 1], "abc"
SHAPES = [(16384, 16384, 16384), (14400, 14400, 480), (4000, 16000, 2000)]
WORKLOAD = "222-1x333-1 abc FP64 C+=A*B over 16384^3, 14400x14400x480, 4000x16000x2000"
METRIC = "effective TFLOPS (2mnk/t), 222-1x333-1 abc FP64"
UNIT = "TFLOP/s"
# DRAM traffic of the FMM products kernel per executed core flop, from a one-pass ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the products launch of a smaller case of
# the same algorithm, 222-1 x 333-1 at 6144^3: 11.62 GB over 3.46e11 executed flops (its
# algorithmic bytes: 11.4 GB).  roofline.traffic scales it to the average products launch.
TRAFFIC_BYTES_PER_FLOP = 11.62e9 / 3.46e11
TRAFFIC_SOURCE = "scaled by executed flops from one capture of the 222-1x333-1 6144^3 products launch"


def effective_flops(shapes):
    return sum(2.0 * m * n * k for (m, n, k) in shapes)


def core_flops(plan, shapes):
    from fmm_gen_b200 import algebra

    tot = 0.0
    for (m, n, k) in shapes:
        p = algebra.partition(m, n, k, plan.dims)
        tot += plan.rank * 2.0 * p.ms * p.ns * p.ks
    return tot


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            with open(self.path) as fh:
                for r in csv.reader(fh):
                    if len(r) >= 9:
                        rows.append([x.strip() for x in r])
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = [num(r[2]) for r in rows if num(r[2]) is not None]
        power = [num(r[3]) for r in rows if num(r[3]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(power) if power else None}


REF_PRODUCTS_PER_STEP = 8  # products of the 16384^3 call's FMM core timed per CPU step


class _CpuWorkload:
    """This bench's workload on the host cores, with every input made (seeded) and every
    table or library loaded before anything is timed.

    One step runs the 14400x14400x480 and 4000x16000x2000 calls whole, and samples the
    16384^3 call: its FMM core (16368 x 16368 x 16380; the fringe strips are 0.2 % of its
    flops) run over REF_PRODUCTS_PER_STEP of its 161 products, a different group each step
    (all 161 after 21 steps), credited that share of the core's 2mnk.  A whole 16384^3 call
    takes tens of seconds on 16 cores; the sample keeps a step at a few seconds.  step()
    returns the credited effective flops and the seconds spent in the timed calls alone."""

    kind = ""

    def __init__(self, seed: int = 99):
        import numpy as np

        from fmm_gen_b200 import algebra

        plan = algebra.make_plan(ALGS, LEVELS)
        self.plan = plan
        self.R = plan.rank
        rng = np.random.default_rng(seed)
        self.mats = []
        for (m, n, k) in SHAPES:
            A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
            B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
            C = self._c_buffer(m, n)
            C[:] = rng.uniform(-1, 1, (m, n))
            self.mats.append((A, B, C))
        m, n, k = SHAPES[0]
        self.core = algebra.partition(m, n, k, plan.dims)
        P = REF_PRODUCTS_PER_STEP
        ngroups = (self.R + P - 1) // P
        self.groups = [[(g * P + i) % self.R for i in range(P)] for g in range(ngroups)]
        self.step_no = 0

    def _c_buffer(self, m, n):
        import numpy as np

        return np.zeros((m, n), order="F")

    def step(self):
        pc = self.core
        secs, flops = 0.0, 0.0
        for (m, n, k), (A, B, C) in zip(SHAPES[1:], self.mats[1:]):
            t0 = time.perf_counter()
            self._whole(A, B, C)
            secs += time.perf_counter() - t0
            flops += 2.0 * m * n * k
        A, B, C = self.mats[0]
        g = self.step_no % len(self.groups)
        Ac, Bc, Cc = A[:pc.md, :pc.kd], B[:pc.kd, :pc.nd], C[:pc.md, :pc.nd]
        t0 = time.perf_counter()
        self._sample(g, Ac, Bc, Cc)
        secs += time.perf_counter() - t0
        flops += 2.0 * pc.md * pc.nd * pc.kd * REF_PRODUCTS_PER_STEP / self.R
        self.step_no += 1
        return flops, secs

    def _sample_text(self, steps):
        return (f"per step 14400x14400x480 and 4000x16000x2000 whole plus {REF_PRODUCTS_PER_STEP} of the 161 "
                f"products of the 16384^3 call's FMM core (16368x16368x16380), rotating, credited "
                f"{REF_PRODUCTS_PER_STEP}/161 of its 2mnk; {steps} steps; inputs generated before timing")


class ReferenceWorkload(_CpuWorkload):
    """The reference's own generated multithreaded code (oracle/build_ref_fmm.py: the
    222-1_333-1 abc job emitted by its generator and compiled with its runtime and
    -D_PARALLEL_), on every host core the process may use (BLISLAB_IC_NT).  The sample of the
    16384^3 call runs one of the job's 8-product libraries: the same generated code for those
    products.  C is laid out as the reference's driver allocates it (32-byte aligned)."""

    kind = "reference"

    def __init__(self, seed: int = 99):
        from oracle import build_ref_fmm, cpu

        self.cpu = cpu
        paths = build_ref_fmm.library_paths()
        self.cores = len(os.sched_getaffinity(0))
        cpu.set_ref_threads(self.cores)
        self.full = cpu.RefFMMLib(paths["full"])
        self.libs = [cpu.RefFMMLib(p) for p in paths["groups"]]
        super().__init__(seed)
        assert len(self.libs) == len(self.groups)

    def _c_buffer(self, m, n):
        return self.cpu.aligned_colmajor(m, n)

    def _whole(self, A, B, C):
        self.full(A, B, C)

    def _sample(self, g, A, B, C):
        self.libs[g](A, B, C)

    def describe(self, steps):
        return (f"the reference's generated 222-1_333-1 abc code (its generator + runtime, -D_PARALLEL_, "
                f"oracle/_ref/fmm) on {self.cores} host threads; " + self._sample_text(steps))


class OracleWorkload(_CpuWorkload):
    """The oracle -- the CPU restatement of the reference's generated abc code, OpenMP over
    the host cores -- where the reference's own libraries were not built."""

    kind = "port"

    def __init__(self, seed: int = 99):
        from fmm_gen_b200 import runtime
        from oracle import cpu

        self.cpu = cpu
        super().__init__(seed)
        dims, nterms, rows, cols, coefs = runtime.plan_tables(self.plan)
        self.tables = (dims, self.R, nterms, rows, cols, coefs)
        self.subsets = [cpu.product_subset(self.tables, grp) for grp in self.groups]
        self.cores = cpu.num_threads()

    def _whole(self, A, B, C):
        self.cpu.fmm(self.tables, PACK, A, B, C)

    def _sample(self, g, A, B, C):
        self.cpu.fmm(self.subsets[g], PACK, A, B, C)

    def describe(self, steps):
        return (f"oracle/fmm_oracle.c (the reference's abc arithmetic) on {self.cores} host threads; "
                + self._sample_text(steps))


def cpu_workload():
    """The reference's own libraries where they were built, else the oracle port."""
    from oracle import build_ref_fmm

    paths = build_ref_fmm.library_paths()
    if all(os.path.exists(p) for p in [paths["full"]] + paths["groups"]):
        return ReferenceWorkload()
    return OracleWorkload()


def run_reference(args, rank):
    """--impl reference: the reference's own code for the path (or the oracle), timed on the host."""
    if rank != 0:
        return
    wl = cpu_workload()
    for _ in range(args.warmup):
        wl.step()
    flops, secs = 0.0, 0.0
    for _ in range(args.steps):
        f, t = wl.step()
        flops += f
        secs += t
    value = flops / secs / 1e12
    sample = wl.describe(args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "algorithm": "222-1_333-1", "pack_type": PACK,
                   "shapes": [list(s) for s in SHAPES], "inputs": "A,B,C ~ U(-1,1), seeded",
                   "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": wl.cores, "kind": wl.kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def split_bf16_8192(rt, torch, dev, steps=3):
    """Split-BF16 FMM (222-2, 8192^3): FP32 inputs in two sets (N(0,1); log-uniform
    magnitudes 2^-10..2^10 with random sign), FP64 C; time, effective TFLOPS against the
    project's plain FP64 GEMM on the same values, and the relative Frobenius error against
    an FP64 classical GEMM (cuBLAS) of the same inputs."""
    n = 8192
    p2 = rt.Plan.from_levels(["222"], [2])
    g = torch.Generator(device=dev).manual_seed(8192)
    out = {"algorithm": "222-2", "shape": [n, n, n], "products": "6 bf16 plane products, FP32 accumulate, FP64 scatter"}

    def loguniform():
        e = torch.empty((n, n), device=dev).uniform_(-10, 10, generator=g)
        s = torch.empty((n, n), device=dev).uniform_(-1, 1, generator=g).sign()
        return rt.colmajor(n, n, dtype=torch.float32, device=dev).copy_(s * torch.exp2(e))

    sets = {
        "normal": lambda: rt.colmajor(n, n, dtype=torch.float32, device=dev).normal_(generator=g),
        "loguniform": loguniform,
    }
    C = rt.colmajor(n, n, device=dev)
    f = 2.0 * n ** 3
    for name, make in sets.items():
        A, B = make(), make()
        C.zero_()
        rt.split_gemm(p2, A, B, C)
        torch.cuda.synchronize()
        ref = A.double() @ B.double()
        err = ((C - ref).norm() / ref.norm()).item()
        del ref
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            rt.split_gemm(p2, A, B, C)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms": ms, "tflops_effective": f / (ms * 1e-3) / 1e12, "rel_fro_err": err}
        del A, B
    # the plain FP64 comparator on FP64 operands of the same size
    Ad = rt.colmajor(n, n, device=dev).uniform_(-1, 1, generator=g)
    Bd = rt.colmajor(n, n, device=dev).uniform_(-1, 1, generator=g)
    rt.plain_gemm(Ad, Bd, C)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        rt.plain_gemm(Ad, Bd, C)
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / steps
    out["plain_fp64_ms"] = plain_ms
    out["speedup_vs_plain_fp64"] = {k: plain_ms / out[k]["ms"] for k in sets}
    with rt.KernelTimer() as kt:
        rt.split_gemm(p2, Ad.float(), Bd.float(), C)
    out["kernel_ms"] = {k: v for k, v in kt.ms.items() if kt.count[k]}
    peak, peak_src = _measured_peak("bf16_tflops")
    gemm_ms = kt.ms.get("fmm_split_gemm_kernel", 0.0)
    if gemm_ms > 0:
        bf16_flops = 49 * 6 * 2.0 * (n // 4) ** 3
        ach = bf16_flops / (gemm_ms * 1e-3) / 1e12
        out["roofline"] = {"bound": "tensor", "kernel": "fmm_split_gemm_kernel", "achieved": ach, "peak": peak,
                           "unit": "TFLOP/s", "frac": ach / peak if peak else None,
                           "peak_source": peak_src + ", burst"}
    del Ad, Bd, C
    torch.cuda.empty_cache()
    return out


def strassen_2048(rt, torch, dev, steps=5):
    """222-1 abc at 2048^3 (the minimum slice: A, B ~ U(-1,1), C = 0): effective TFLOPS beside
    the plain kernel, and the relative error against an FP64 classical GEMM (cuBLAS)."""
    n = 2048
    g = torch.Generator(device=dev).manual_seed(2048)
    A = rt.colmajor(n, n, device=dev).uniform_(-1, 1, generator=g)
    B = rt.colmajor(n, n, device=dev).uniform_(-1, 1, generator=g)
    C = rt.colmajor(n, n, device=dev).zero_()
    p1 = rt.Plan.from_levels(["222"], [1])
    rt.fmm_gemm(p1, A, B, C, "abc")
    ref = A @ B
    torch.cuda.synchronize()
    err = ((C - ref).norm() / ref.norm()).item()

    def t(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    f = 2.0 * n ** 3
    ms_f = t(lambda: rt.fmm_gemm(p1, A, B, C, "abc"))
    ms_p = t(lambda: rt.plain_gemm(A, B, C))
    return {"algorithm": "222-1", "pack_type": "abc", "shape": [n, n, n], "ms": ms_f,
            "tflops_effective": f / (ms_f * 1e-3) / 1e12, "plain_tflops": f / (ms_p * 1e-3) / 1e12,
            "rel_fro_err_vs_cublas": err}


# Peaks measured earlier on this pool's B200s, used when the per-pod MEASURED_PEAKS.json is
# absent: dense bf16 GEMM burst (TFLOP/s) and a copy's HBM bandwidth (GB/s).
FALLBACK_PEAKS = {"bf16_tflops": 1590.0, "hbm_gbs": 6650.0}


def _measured_peak(key):
    """(peak, source): MEASURED_PEAKS.json's value, else the fallback measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)[key]), f"MEASURED_PEAKS.json {key} (of measured)"
    except Exception:
        return FALLBACK_PEAKS.get(key), f"{key} = {FALLBACK_PEAKS.get(key)} (of fallback: no MEASURED_PEAKS.json)"


def batch_512(rt, torch, dev, steps=3):
    """512 FP64 problems, m, n, k log-uniform in [256, 4096] from the seed, entries U(-1,1),
    C += A*B in one persistent launch (captured in a CUDA graph and replayed); per-problem
    algorithm from the tuner (model seed, then measured refinement)."""
    from fmm_gen_b200 import tuner

    shapes = tuner.random_batch_shapes(512, seed=0)
    g = torch.Generator(device=dev).manual_seed(512)
    As, Bs, Cs = [], [], []
    for (m, n, k) in shapes:
        As.append(rt.colmajor(m, k, device=dev).uniform_(-1, 1, generator=g))
        Bs.append(rt.colmajor(k, n, device=dev).uniform_(-1, 1, generator=g))
        Cs.append(rt.colmajor(m, n, device=dev).uniform_(-1, 1, generator=g))
    flops = sum(2.0 * m * n * k for (m, n, k) in shapes)
    measure = tuner.batch_timer(rt, shapes, As, Bs, Cs, reps=2)
    t0 = time.perf_counter()
    tn = tuner.BatchTuner()
    rep = tn.tune(shapes, measure)
    tune_s = time.perf_counter() - t0
    model_ms = sum(tuner.model_time(tn.model, c, *s) for c, s in zip(rep.choices, shapes)) * 1e3
    classical_ms = measure(["classical"] * len(shapes))
    for c in set(rep.choices) - {"classical"} - set(measure.plans):
        measure.plans[c] = rt.Plan.from_levels(*tuner.candidate_levels(c))
    plans = [None if c == "classical" else measure.plans[c] for c in rep.choices]
    batch = rt.Batch(shapes, plans, tiles=rep.tiles)
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        batch.run(As, Bs, Cs, stream=s)
    torch.cuda.current_stream(dev).wait_stream(s)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    n0 = rt.kernel_launch_count()
    with torch.cuda.graph(graph):
        batch.run(As, Bs, Cs)
    launches_per_replay = rt.kernel_launch_count() - n0  # kernels the library put into the graph
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    del graph
    batch.close()
    out = {"problems": len(shapes), "dims": "log-uniform [256, 4096], seed 0", "total_flop": flops,
           "ms": ms, "tflops_effective": flops / (ms * 1e-3) / 1e12,
           "all_classical_ms": classical_ms, "model_ms": model_ms,
           "choices": rep.counts(), "choices_key": "algorithm/tile rows", "tune_s": tune_s,
           "tune_trials": rep.trials,
           "launches_per_replay": launches_per_replay}
    del As, Bs, Cs
    torch.cuda.empty_cache()
    return out


# operands of admitted requests live in one allocation made before the window (the rest of
# the 160 GB budget is the library's workspaces, from its own stream-ordered pool)
SERVE_ARENA_BYTES = 120e9


def serving_2000(rt, torch, dev, window=1.0, rank=0, world=1):
    """Continuous-batching request loop: Poisson arrivals at 2000 req/s for `window` s
    (80% FP64 with m, n, k log-uniform in [256, 4096]; 10% FP64 rank-k 16000x16000x256;
    10% split-BF16 222-2 8192^3), operands device-resident from admission in an arena made
    up front, 160 GB HBM budget; p50/p99 latency and effective TFLOPS over the window.  With N GPUs each rank
    serves its deterministic share of the stream."""
    from fmm_gen_b200 import serve

    reqs = serve.poisson_requests(serve.Mix(rate=2000.0), window, seed=0)
    if world > 1:
        reqs = serve.shard_requests(reqs, world)[rank]
    torch.cuda.empty_cache()
    ex = serve.GpuExecutor(seed=0, arena_bytes=SERVE_ARENA_BYTES)
    ex.warm(reqs)  # first-use costs (plans, workspace pool growth) outside the window
    rep = serve.Server(ex, budget_bytes=160e9).run(reqs, window)
    out = rep.summary()
    out["arrivals"] = "Poisson 2000 req/s, seed 0" + (f", share of rank {rank}/{world}" if world > 1 else "")
    out["budget_gb"] = 160
    out["operand_arena_gb"] = SERVE_ARENA_BYTES / 1e9
    out["policy"] = ("admission in arrival order by HBM budget, backfill past a waiting request for up to 50 ms, "
                     "bounded queue 4096; FP64 requests batched per launch")
    del ex
    torch.cuda.empty_cache()
    return out


def run_split2d(args, world, rank, local):
    """--split2d: each of the workload's three GEMMs split 2-D over the ranks (strong scaling:
    the total work stays the workload's).  A step per shape: the A row panel and the B column
    panel arrive over the process grid in k chunks (NCCL broadcasts from each chunk's owner, the
    next chunk in flight while the local FMM call of this one runs on this rank's C block).
    value = the workload's effective flops / the slowest rank's time."""
    import datetime

    import torch
    import torch.distributed as dist

    from fmm_gen_b200 import runtime as rt, shard

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        dist.init_process_group("gloo", store=dist.HashStore(), rank=0, world_size=1)
    dev = torch.device("cuda", local)
    plan = rt.Plan.from_levels(ALGS, LEVELS)
    g = torch.Generator(device=dev).manual_seed(2000 + rank)
    work = []
    for (m, n, k) in SHAPES:
        gm = shard.Gemm2D(m, n, k, plan.algebra.dims)
        b = gm.blk
        rows, cols = b.rows[1] - b.rows[0], b.cols[1] - b.cols[0]
        A_own = rt.colmajor(rows, b.a_k[1] - b.a_k[0], device=dev).uniform_(-1, 1, generator=g)
        B_own = rt.colmajor(b.b_k[1] - b.b_k[0], cols, device=dev).uniform_(-1, 1, generator=g)
        C_own = rt.colmajor(rows, cols, device=dev).uniform_(-1, 1, generator=g)
        work.append((gm, A_own, B_own, C_own))

    def local_gemm(A, B, C):
        rt.fmm_gemm(plan, A, B, C, PACK)

    def step():
        for gm, A_own, B_own, C_own in work:
            gm.run_pipelined(A_own, B_own, C_own, local_gemm)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev if world > 1 else "cpu")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = effective_flops(SHAPES) * args.steps / (ms * 1e-3) / 1e12
    if rank == 0:
        pr, pc = shard.process_grid(world)
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "algorithm": "222-1_333-1", "pack_type": PACK,
                       "parallelism": f"2-D C split over a {pr}x{pc} grid, panels broadcast in k chunks (SUMMA order)"}}),
              flush=True)
    dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the split-BF16 and batch measurements")
    ap.add_argument("--split2d", action="store_true",
                    help="split each GEMM 2-D over the ranks (strong scaling) instead of replicas")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.split2d:
        run_split2d(args, world, rank, local)
        return

    import torch

    from fmm_gen_b200 import algebra, runtime as rt

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_

        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_
    dev = torch.device("cuda", local)
    plan = rt.Plan.from_levels(ALGS, LEVELS)
    g = torch.Generator(device=dev).manual_seed(1000 + rank)
    mats = []
    for (m, n, k) in SHAPES:
        A = rt.colmajor(m, k, device=dev).uniform_(-1, 1, generator=g)
        B = rt.colmajor(k, n, device=dev).uniform_(-1, 1, generator=g)
        C = rt.colmajor(m, n, device=dev).uniform_(-1, 1, generator=g)
        mats.append((A, B, C))
    stream = torch.cuda.current_stream(dev)

    def step():
        for (A, B, C) in mats:
            rt.fmm_gemm(plan, A, B, C, PACK, stream=stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- timed region ----
    launches0 = rt.kernel_launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        with rt.KernelTimer() as kt:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
    barrier()
    launches = rt.kernel_launch_count() - launches0
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    eff = effective_flops(SHAPES)
    value = world * eff * args.steps / (ms_max * 1e-3) / 1e12
    clk = clocks.summary()

    # ---- dominant kernel roofline (FP64 DMMA bound) ----
    # the FMM products launches: the direct variant (pre-summed operands) or the folding kernel
    kinds = [k for k in ("fmm_gemm_direct_kernel[fmm products]", "fmm_gemm_kernel[fmm products]") if kt.count.get(k)]
    core_name = max(kinds, key=lambda k: kt.ms[k]) if kinds else "fmm_gemm_direct_kernel[fmm products]"
    core_ms = sum(kt.ms[k] for k in kinds)
    core_launches = sum(kt.count[k] for k in kinds)
    cflops = core_flops(plan.algebra, SHAPES) * args.steps
    achieved = cflops / (core_ms * 1e-3) / 1e12 if core_ms > 0 else None

    # measured FP64 tensor peak: cuBLAS DGEMM 8192^3 on this GPU, this run
    a = torch.rand(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.rand(8192, 8192, dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        torch.matmul(a, b, out=c)
        s1.record()
        torch.cuda.synchronize()
        best = min(best, s0.elapsed_time(s1))
    peak = 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12
    del a, b, c

    # ---- correctness of this run's result against a classical FP64 GEMM; workspace per call ----
    errs, ws_bytes = {}, {}
    for (m, n, k), (A, B, C) in zip(SHAPES, mats):
        C0 = rt.colmajor(m, n, device=dev).copy_(C)
        ref = torch.addmm(C0, A, B)
        rt.fmm_gemm(plan, A, B, C0, PACK)
        torch.cuda.synchronize()
        ws_bytes[f"{m}x{n}x{k}"] = rt.last_workspace_bytes()
        errs[f"{m}x{n}x{k}"] = ((C0 - ref).norm() / ref.norm()).item()
        del C0, ref
    torch.cuda.empty_cache()

    # ---- comparators: the project's plain FP64 GEMM, and 222-1 at 16384^3 ----
    def time_call(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(reps):
            fn()
        s1.record()
        torch.cuda.synchronize()
        return s0.elapsed_time(s1) / reps

    plain_ms = sum(time_call(lambda A=A, B=B, C=C: rt.plain_gemm(A, B, C)) for (A, B, C) in mats)
    plain_tflops = eff / (plain_ms * 1e-3) / 1e12
    A16, B16, C16 = mats[0]
    p1 = rt.Plan.from_levels(["222"], [1])
    s222 = time_call(lambda: rt.fmm_gemm(p1, A16, B16, C16, "abc"))
    ws222 = rt.last_workspace_bytes()
    s_plain16 = time_call(lambda: rt.plain_gemm(A16, B16, C16))
    f16 = 2.0 * 16384 ** 3
    # the per-shape rate of the workload's algorithm beside the plain kernel
    per_shape = {}
    for (m, n, k), (A, B, C) in zip(SHAPES, mats):
        tf = time_call(lambda A=A, B=B, C=C: rt.fmm_gemm(plan, A, B, C, PACK))
        tp = time_call(lambda A=A, B=B, C=C: rt.plain_gemm(A, B, C))
        per_shape[f"{m}x{n}x{k}"] = {"fmm_tflops": 2.0 * m * n * k / (tf * 1e-3) / 1e12,
                                     "plain_tflops": 2.0 * m * n * k / (tp * 1e-3) / 1e12, "ratio": tp / tf}

    # ---- end to end through the host C ABI (pinned host buffers, copies in the timed region) ----
    host = []
    for (A, B, C) in mats:
        hs = []
        for X in (A, B, C):
            h = torch.empty(X.shape[1], X.shape[0], dtype=torch.float64, pin_memory=True).t()
            h.copy_(X)
            hs.append(h.numpy())
        host.append(hs)
    h2d = sum(8 * (m * k + k * n + m * n) for (m, n, k) in SHAPES)
    d2h = sum(8 * m * n for (m, n, k) in SHAPES)
    # One step = the workload's three calls, issued from three host threads (the library is
    # reentrant per thread: each call runs on its thread's own stream), so that one call's PCIe
    # copies overlap another's compute; the serial figure (one call after the other) beside it.
    from concurrent.futures import ThreadPoolExecutor

    def call(h):
        torch.cuda.set_device(dev)
        rt.fmm_gemm_host(plan, h[0], h[1], h[2], PACK)

    pool = ThreadPoolExecutor(max_workers=len(host))
    list(pool.map(call, host))  # warm the host path (workspace pool, every thread's stream)
    for h in host:
        call(h)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        list(pool.map(call, host))
    e2e_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for h in host:
            call(h)
    e2e_serial_s = time.perf_counter() - t0
    pool.shutdown()
    te = torch.tensor([e2e_s, e2e_serial_s], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * eff * args.steps / float(te[0].item()) / 1e12
    e2e_serial = world * eff * args.steps / float(te[1].item()) / 1e12
    del host

    extra = {}
    if not args.no_extra:
        del mats
        torch.cuda.empty_cache()
        extra["strassen_222_1_2048"] = strassen_2048(rt, torch, dev)
        extra["split_bf16_222_2_8192"] = split_bf16_8192(rt, torch, dev)
        extra["batch_512_fp64"] = batch_512(rt, torch, dev)
        del A16, B16, C16
        torch.cuda.empty_cache()
        extra["serving_2000rps"] = serving_2000(rt, torch, dev, rank=rank, world=world)

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        wl = cpu_workload()
        wl.step()  # warm-up
        cf, cs = 0.0, 0.0
        for _ in range(3):
            f, t = wl.step()
            cf += f
            cs += t
        cpu_baseline = {"value": cf / cs / 1e12, "unit": UNIT, "cores": wl.cores, "kind": wl.kind,
                        "sample": wl.describe(3) + f", {cs:.1f} s"}
        del wl

    if rank == 0:
        per_launch_flops = cflops / max(core_launches, 1)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "algorithm": "222-1_333-1", "pack_type": PACK,
                       "shapes": [list(s) for s in SHAPES], "inputs": "A,B,C ~ U(-1,1), seeded",
                       "l2": "inputs larger than L2 (8.5 GB per step), no flush",
                       "parallelism": f"replicas{world}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "fmm_dgemm_host (C ABI, pinned host buffers); the step's three calls from three host "
                           "threads", "serial_value": e2e_serial},
            "roofline": {"bound": "tensor", "kernel": core_name, "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                         "peak_source": "measured cuBLAS DGEMM 8192^3 on this GPU in this run (FP64 tensor)",
                         "traffic": (TRAFFIC_BYTES_PER_FLOP * per_launch_flops) if TRAFFIC_BYTES_PER_FLOP else None,
                         "traffic_source": TRAFFIC_SOURCE,
                         "launches": core_launches, "avg_launch_ms": core_ms / max(core_launches, 1),
                         "executed_flops_per_launch": per_launch_flops},
            "kernel_ms": kt.ms, "kernel_launches": kt.count,
            "gpu_launches": launches,
            "clocks": clk,
            "cpu_baseline": cpu_baseline,
            "plain_fp64": {"tflops": plain_tflops, "fmm_over_plain": value / world / plain_tflops},
            "strassen_222_1_16384": {"fmm_tflops": f16 / (s222 * 1e-3) / 1e12,
                                     "plain_tflops": f16 / (s_plain16 * 1e-3) / 1e12,
                                     "ratio": s_plain16 / s222, "workspace_bytes": ws222},
            "per_shape": per_shape,
            "workspace": {"limit_bytes": rt.set_workspace_limit(0), "per_call_bytes": ws_bytes,
                          "note": "pre-summed operand workspace; calls above the limit run their products in groups"},
            "rel_fro_err_vs_cublas": errs,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
