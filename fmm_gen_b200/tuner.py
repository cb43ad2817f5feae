"""Per-problem algorithm selection for batches: a B200 performance model seeds the
choice, batch-level measurements refine it.

The reference ranks algorithms with an analytic model (meta/model_coefficient.py:36-100
counts, per product, the nonzeros of U, V, W; meta/model_gen.py:65-102 turns them into
time = actual_flops * tau + memops * alpha for its CPU blocking MC/KC/NC).  The same
structure is re-derived here for this implementation on B200:

  * compute: every product of a job is a sub-GEMM tiled 128 x 128 with k steps of 8.
    A k step costs `kstep_s` on one SM at the plain kernel's rate.  A product whose
    operand sums are folded while staging costs `1 + fold_per_term * (T - 1)` times that
    (T = the larger of its A and B term counts) on whole tiles; pre-summed products (and
    classical jobs) run in the direct kernel variant, cost 1, and their edge tiles count
    only the 16-row / 32-column fragments they compute.
  * memory: the pre-sum pass reads every U/V term and writes each summed operand once
    (HBM bytes / bandwidth, a separate pass).  The multi-destination epilogue reads and
    writes one C tile per W nonzero: in the direct variant it overlaps the products'
    MMAs (the job takes the longer of the two, the C traffic counted `c_direct` times its
    HBM time); in the folded kernel it does not (`c_exposed` times, added).
  * partition: the same fringe split as the library (algebra.partition); the strips
    are classical jobs.
`model_time` is the batch's throughput view: SM-seconds / SMs plus the exposed memory
time (a batch keeps every SM busy, so wave quantisation of a single problem does not
apply).  `model_time_single` is one problem on its own: every launch (pre-sum pass, FMM
products, each fringe strip) takes whole waves of work units over the SMs plus a launch
latency.

The tuner takes the model's best candidate per problem, then measures the whole batch
and re-assigns groups of problems (by the model's choice and margin) while that makes the
measured batch faster.  The only tile shape of the FP64 kernel is 128 x 128; the other
scheduling parameter, products per work unit, is chosen by the batch itself.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import algebra

CANDIDATES: Tuple[str, ...] = ("classical", "222-1", "232-1", "333-1", "222-2")
TILE = 128
KSTEP = 8


@dataclass
class B200Model:
    """Constants of the model; defaults are this implementation's measurements on B200.

    plain FP64 kernel 34.5 TFLOP/s; folded 222-1 products at 1.7x a plain k step; 6.5 TB/s
    copy bandwidth; `c_exposed` fitted to the folded kernel (the epilogue on the consumer
    warps, 1.5 x its HBM time); `c_direct`, `wave_unit_s` and `launch_s` fitted to 17
    single-problem measurements of the direct variant (222-1, 222-2, 222-1 x 333-1 and
    classical, 1024^3 to 16384^3 and the rank-k shapes): `model_time_single` is within
    9 % RMS (log ratio) of them, 3-5 % on the large shapes."""

    sms: int = 148
    plain_tflops: float = 34.5
    hbm_gbs: float = 6500.0
    fold_per_term: float = 0.7
    c_exposed: float = 1.5
    c_direct: float = 1.6
    unit_overhead_s: float = 1.5e-6  # pipeline fill + epilogue latency per work unit (batch view)
    wave_unit_s: float = 8e-6        # the same seen by one problem (its last epilogue is exposed)
    launch_s: float = 20e-6          # per launch of one problem

    @property
    def kstep_s(self) -> float:
        per_sm = self.plain_tflops * 1e12 / self.sms
        return 2.0 * TILE * TILE * KSTEP / per_sm


def candidate_levels(name: str) -> Tuple[List[str], List[int]]:
    algs, levels = [], []
    for part in name.split("_"):
        a, lv = part.split("-")
        algs.append(a)
        levels.append(int(lv))
    return algs, levels


_PLANS: Dict[str, algebra.FMMPlan] = {}


def plan_of(name: str) -> Optional[algebra.FMMPlan]:
    if name == "classical":
        return None
    if name not in _PLANS:
        _PLANS[name] = algebra.make_plan(*candidate_levels(name))
    return _PLANS[name]


def model_counts(plan: algebra.FMMPlan) -> List[int]:
    """[R, A additions, B additions, C updates]: the reference's comp_counter
    (model_coefficient.py:36-100), from the composed U, V, W."""
    nu = np.count_nonzero(plan.U, axis=0)
    nv = np.count_nonzero(plan.V, axis=0)
    return [plan.rank, int((nu - 1).sum()), int((nv - 1).sum()), int(np.count_nonzero(plan.W))]


def _presummed(plan: algebra.FMMPlan, ms: int, ns: int, ks: int) -> bool:
    """The library's rule for forming operand sums in HBM before the products."""
    return plan.rank > 1 and ms * ns >= (1 << 17) and ks >= 64


def _tiles(ms: int, ns: int) -> int:
    return math.ceil(ms / TILE) * math.ceil(ns / TILE)


def _tile_work(ms: int, ns: int) -> float:
    """Tiles of an ms x ns sub-block in the direct variant, an edge tile counted by the
    fragments it computes: 16-row fragments at the bottom edge, 32-column groups at the
    right edge, the cheaper of the two at the corner."""
    fr, rr = divmod(ms, TILE)
    fc, rc = divmod(ns, TILE)
    rf = math.ceil(rr / 16) / 8 if rr else 0.0
    cf = math.ceil(rc / 32) / 4 if rc else 0.0
    return fr * fc + fc * rf + fr * cf + (min(rf, cf) if rr and rc else 0.0)


def _classical_job(model: B200Model, m: int, n: int, k: int) -> Tuple[float, float, int]:
    if m <= 0 or n <= 0 or k <= 0:
        return 0.0, 0.0, 0
    return _tile_work(m, n) * math.ceil(k / KSTEP) * model.kstep_s, 0.0, _tiles(m, n)


def _core(model: B200Model, plan: algebra.FMMPlan, p) -> Dict[str, float]:
    """The FMM products of one problem: SM-seconds, work units, pre-sum seconds, C epilogue
    seconds and whether the epilogue overlaps the MMAs."""
    tiles = _tiles(p.ms, p.ns)
    ksteps = math.ceil(p.ks / KSTEP)
    nu = np.count_nonzero(plan.U, axis=0)
    nv = np.count_nonzero(plan.V, axis=0)
    c_s = 16.0 * int(np.count_nonzero(plan.W)) * p.ms * p.ns / (model.hbm_gbs * 1e9)
    if _presummed(plan, p.ms, p.ns, p.ks):
        na, nb = int((nu > 1).sum()), int((nv > 1).sum())
        bytes_ = 8.0 * (nu[nu > 1].sum() * p.ms * p.ks + na * p.ms * p.ks +
                        nv[nv > 1].sum() * p.ks * p.ns + nb * p.ks * p.ns)
        return {"sm_s": _tile_work(p.ms, p.ns) * ksteps * model.kstep_s * plan.rank, "units": tiles * plan.rank,
                "presum_s": bytes_ / (model.hbm_gbs * 1e9), "c_s": model.c_direct * c_s, "overlap": True}
    T = np.maximum(nu, nv)
    factor = float((1.0 + model.fold_per_term * (T - 1)).sum())
    return {"sm_s": tiles * ksteps * model.kstep_s * factor, "units": tiles * plan.rank, "presum_s": 0.0,
            "c_s": model.c_exposed * c_s, "overlap": False}


def _strips(p, m: int, n: int, k: int):
    return ((p.md, p.nd, p.kr), (m, p.nr, k), (p.mr, p.nd, k))


def job_costs(model: B200Model, name: str, m: int, n: int, k: int) -> Dict[str, float]:
    """Modelled SM-seconds, exposed HBM seconds (`mem_s`), HBM seconds that overlap the
    MMAs (`ovl_s`) and work units of one problem."""
    plan = plan_of(name)
    if plan is None:
        sm, mem, units = _classical_job(model, m, n, k)
        return {"sm_s": sm + units * model.unit_overhead_s, "mem_s": mem, "ovl_s": 0.0, "units": units}
    p = algebra.partition(m, n, k, plan.dims)
    sm = mem = ovl = 0.0
    units = 0
    if p.ms > 0 and p.ns > 0 and p.ks > 0:
        c = _core(model, plan, p)
        sm += c["sm_s"]
        units += c["units"]
        mem += c["presum_s"]
        if c["overlap"]:
            ovl += c["c_s"]
        else:
            mem += c["c_s"]
    for (mm, nn, kk) in _strips(p, m, n, k):
        s2, _, u2 = _classical_job(model, mm, nn, kk)
        sm += s2
        units += u2
    sm += units * model.unit_overhead_s
    return {"sm_s": sm, "mem_s": mem, "ovl_s": ovl, "units": units}


def model_time(model: B200Model, name: str, m: int, n: int, k: int) -> float:
    """Throughput view (one problem of a batch that keeps every SM busy)."""
    c = job_costs(model, name, m, n, k)
    return max(c["sm_s"] / model.sms, c["ovl_s"]) + c["mem_s"]


def model_time_single(model: B200Model, name: str, m: int, n: int, k: int) -> float:
    """One problem on its own: whole waves of work units per launch plus launch latency."""

    def launch(sm_s: float, units: int) -> float:
        if units <= 0:
            return 0.0
        return math.ceil(units / model.sms) * (sm_s / units + model.wave_unit_s) + model.launch_s

    def classical(mm: int, nn: int, kk: int) -> float:
        s, _, u = _classical_job(model, mm, nn, kk)
        return launch(s, u)

    plan = plan_of(name)
    if plan is None:
        return classical(m, n, k)
    p = algebra.partition(m, n, k, plan.dims)
    t = 0.0
    if p.ms > 0 and p.ns > 0 and p.ks > 0:
        c = _core(model, plan, p)
        if c["presum_s"] > 0:
            t += c["presum_s"] + model.launch_s
        if c["overlap"]:
            t += max(launch(c["sm_s"], c["units"]), c["c_s"])
        else:
            t += launch(c["sm_s"], c["units"]) + c["c_s"]
    for (mm, nn, kk) in _strips(p, m, n, k):
        t += classical(mm, nn, kk)
    return t


def rank_candidates(model: B200Model, shape: Sequence[int],
                    candidates: Sequence[str] = CANDIDATES) -> List[Tuple[str, float]]:
    m, n, k = shape
    return sorted(((c, model_time(model, c, m, n, k)) for c in candidates), key=lambda t: t[1])


@dataclass
class TuneReport:
    choices: List[str]
    model_choices: List[str]
    trials: List[Tuple[str, float]] = field(default_factory=list)  # (description, measured ms)
    tiles: List[int] = field(default_factory=list)  # tile height per problem (128 or 64 rows)

    def counts(self) -> Dict[str, int]:
        """Problems per (algorithm, tile height), e.g. {"classical/128": 500, "222-1/64": 3}."""
        out: Dict[str, int] = {}
        tiles = self.tiles or [TILE] * len(self.choices)
        for c, t in zip(self.choices, tiles):
            key = f"{c}/{t}"
            out[key] = out.get(key, 0) + 1
        return out


class BatchTuner:
    """Chooses an algorithm per problem of a batch.

    `measure(choices) -> milliseconds` times a whole batch with the given per-problem
    algorithm names (the caller owns the operands; see `batch_timer`).  Without it the
    model's choice is returned."""

    def __init__(self, model: Optional[B200Model] = None, candidates: Sequence[str] = CANDIDATES):
        self.model = model or B200Model()
        self.candidates = tuple(candidates)

    def model_choice(self, shapes: Sequence[Sequence[int]]) -> Tuple[List[str], List[List[Tuple[str, float]]]]:
        ranked = [rank_candidates(self.model, s, self.candidates) for s in shapes]
        return [r[0][0] for r in ranked], ranked

    def tune(self, shapes: Sequence[Sequence[int]], measure=None, rounds: int = 2) -> TuneReport:
        choices, ranked = self.model_choice(shapes)
        rep = TuneReport(list(choices), list(choices))
        if measure is None:
            return rep
        best = measure(choices)
        rep.trials.append(("model choice", best))
        for _ in range(rounds):
            improved = False
            # groups: problems the model gives to one FMM candidate; try each group on its
            # runner-up, then on classical
            for cand in self.candidates:
                if cand == "classical":
                    continue
                idx = [i for i, c in enumerate(choices) if c == cand]
                if not idx:
                    continue
                for alt_rank in (1, None):
                    trial = list(choices)
                    for i in idx:
                        if alt_rank is None:
                            trial[i] = "classical"
                        else:
                            trial[i] = ranked[i][alt_rank][0]
                    if trial == choices:
                        continue
                    t = measure(trial)
                    what = f"{cand} group ({len(idx)}) -> " + ("classical" if alt_rank is None else "runner-up")
                    rep.trials.append((what, t))
                    if t < best * 0.995:
                        best, choices, improved = t, trial, True
                        break
            # problems the model sends to classical by a small margin: try their runner-up
            close = [i for i, r in enumerate(ranked)
                     if choices[i] == "classical" and len(r) > 1 and r[1][1] <= 1.05 * r[0][1]]
            if close:
                trial = list(choices)
                for i in close:
                    trial[i] = ranked[i][1][0] if ranked[i][0][0] == "classical" else ranked[i][0][0]
                t = measure(trial)
                rep.trials.append((f"near-tie classical ({len(close)}) -> FMM", t))
                if t < best * 0.995:
                    best, choices, improved = t, trial, True
            if not improved:
                break
        rep.choices = list(choices)
        # tile height: 64-row tiles halve a problem's unit length (twice the units); they help
        # where a problem's units are long and few, so the batch's last units finish late.  The
        # model ranks problems by unit length over unit count; the measurement decides.
        rep.tiles = [TILE] * len(shapes)
        order = sorted(range(len(shapes)), key=lambda i: -self.tile_pressure(choices[i], shapes[i]))
        for frac in (0.05, 0.25, 1.0):
            sel = order[:max(1, int(round(frac * len(order))))]
            trial = list(rep.tiles)
            for i in sel:
                trial[i] = TILE // 2
            t = measure(choices, trial)
            rep.trials.append((f"64-row tiles for {len(sel)} problems", t))
            if t < best * 0.995:
                best, rep.tiles = t, trial
        return rep

    def tile_pressure(self, name: str, shape: Sequence[int]) -> float:
        """k steps per unit over units: large for problems with long, few units."""
        m, n, k = shape
        plan = plan_of(name)
        if plan is None:
            ms, ns, ks, R = m, n, k, 1
        else:
            p = algebra.partition(m, n, k, plan.dims)
            ms, ns, ks, R = max(p.ms, 1), max(p.ns, 1), max(p.ks, 1), plan.rank
        units = _tiles(ms, ns) * R
        return (ks / KSTEP) / max(units, 1)


def random_batch_shapes(count: int = 512, lo: int = 256, hi: int = 4096, seed: int = 0) -> List[Tuple[int, int, int]]:
    """m, n, k each round(exp(U(ln lo, ln hi))) from the seed (the batching workload)."""
    rng = np.random.default_rng(seed)
    d = np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), size=(count, 3)))).astype(int)
    return [tuple(int(v) for v in row) for row in d]


def batch_timer(runtime, shapes, As, Bs, Cs, reps: int = 3, warmup: int = 1):
    """measure(choices, tiles=None) for BatchTuner: builds a Batch with the named plans (and
    per-problem tile heights) and returns the best of `reps` device-timed runs in
    milliseconds.  The runs add into Cs."""
    import torch

    plans: Dict[str, object] = {}

    def plan(name):
        if name == "classical":
            return None
        if name not in plans:
            plans[name] = runtime.Plan.from_levels(*candidate_levels(name))
        return plans[name]

    def measure(choices: Sequence[str], tiles: Optional[Sequence[int]] = None) -> float:
        b = runtime.Batch(shapes, [plan(c) for c in choices], tiles=tiles)
        try:
            for _ in range(warmup):
                b.run(As, Bs, Cs)
            times = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                b.run(As, Bs, Cs)
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            return min(times)
        finally:
            torch.cuda.synchronize()
            b.close()

    measure.plans = plans
    return measure


def shard_problems(shapes: Sequence[Sequence[int]], choices: Sequence[str], world: int,
                   model: Optional[B200Model] = None) -> List[List[int]]:
    """Independent problems to GPUs: longest modelled problem first, each to the GPU with
    the least modelled work so far (LPT).  Deterministic, so every rank computes the same
    assignment without an exchange; returns the problem indices per rank."""
    model = model or B200Model()
    cost = [model_time(model, c, *s) for s, c in zip(shapes, choices)]
    order = sorted(range(len(shapes)), key=lambda i: (-cost[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        g = min(range(world), key=lambda r: (load[r], r))
        load[g] += cost[i]
        out[g].append(i)
    return [sorted(x) for x in out]
