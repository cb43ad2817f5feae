"""Serving: a continuous-batching request loop for mixed-shape, mixed-precision GEMMs.

The reference has no serving layer (its entry point is one synchronous call per GEMM,
meta/abc_gen_mix.py:448-472); this module is the loop that keeps a B200 busy with a stream
of such calls:

  * arrivals   - requests arrive on their own clock (a seeded Poisson stream in the
                 benchmark); each is an FP64 C += A*B of some shape, or an FP32-accurate
                 split-BF16 one.
  * admission  - a request is admitted when its device bytes (operands plus workspace)
                 fit in the HBM budget beside everything admitted and not yet finished;
                 until then it waits in a bounded queue (arrivals beyond it are rejected).
                 Requests behind one that does not fit yet may be admitted past it
                 (backfill) while it has waited less than `head_wait` seconds; after that
                 admission stops until it fits, so a large request cannot starve.
                 Admission brings its operands into device memory, where they stay until
                 it finishes.
  * batching   - every admitted FP64 request not yet dispatched joins the next FP64 batch:
                 one persistent launch over all of their work units (fmm_batch_submit,
                 per-request algorithm from the tuner's model).  Split-BF16 requests run on
                 a second stream.  Up to `inflight` launches per stream are queued on the
                 device, so requests that arrive while others run are admitted and
                 dispatched as memory and launch slots free up, and their work overlaps.
  * completion - an event per launch; when it completes, its requests' latencies are
                 recorded and their memory returns to the budget.

Results do not depend on the mix: a batch gives each problem exactly the arithmetic of a
single call with the same algorithm, and the algorithm depends on the shape only.

The executor is pluggable: GpuExecutor runs on the device through the library;
tests drive the same loop with a simulated executor on the CPU.
"""
from __future__ import annotations

import bisect
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import tuner

FP64, SPLIT = "fp64", "split"


@dataclass
class Request:
    rid: int
    kind: str                      # FP64 or SPLIT
    shape: Tuple[int, int, int]    # (m, n, k)
    algorithm: str                 # tuner candidate name ("classical", "222-1", ...)
    arrival: float                 # seconds from the start of the run
    admitted: Optional[float] = None
    dispatched: Optional[float] = None
    done: Optional[float] = None
    nbytes: int = 0
    handle: object = None          # executor state (operands)

    @property
    def flops(self) -> float:
        m, n, k = self.shape
        return 2.0 * m * n * k

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


def request_bytes(kind: str, shape: Sequence[int], algorithm: str) -> int:
    """Device bytes a request holds while admitted: operands, C and workspaces."""
    m, n, k = shape
    if kind == SPLIT:
        plan = tuner.plan_of(algorithm)
        R = plan.rank if plan is not None else 1
        dims = plan.dims if plan is not None else (1, 1, 1)
        ms, ks, ns = m // dims[0], k // dims[1], n // dims[2]
        kpad = -(-ks // 64) * 64
        mws = 8 * R * ms * ns if R > 1 else 0  # product tiles before the combine pass
        return 4 * (m * k + k * n) + 8 * m * n + 6 * R * (ms + ns) * kpad + mws
    ws = 0
    plan = tuner.plan_of(algorithm)
    if plan is not None:
        p = tuner.algebra.partition(m, n, k, plan.dims)
        if tuner._presummed(plan, p.ms, p.ns, p.ks):
            nu = np.count_nonzero(plan.U, axis=0)
            nv = np.count_nonzero(plan.V, axis=0)
            ws = 8 * (int((nu > 1).sum()) * p.ms * p.ks + int((nv > 1).sum()) * (p.ks + 1) * p.ns)
    pitch = 8 * ((m + 1) * k if m & 1 else 0) + 8 * ((k + 1) * n if k & 1 else 0)
    return 8 * (m * k + k * n + m * n) + ws + pitch


@dataclass
class Mix:
    """The offered load: Poisson arrivals at `rate` per second; a fraction `f_rank_k` of
    rank-k FP64 requests, `f_split` of split-BF16 ones, the rest FP64 with m, n, k each
    log-uniform in [lo, hi]."""

    rate: float = 2000.0
    f_rank_k: float = 0.10
    f_split: float = 0.10
    lo: int = 256
    hi: int = 4096
    rank_k_shape: Tuple[int, int, int] = (16000, 16000, 256)
    split_shape: Tuple[int, int, int] = (8192, 8192, 8192)
    split_algorithm: str = "222-2"


def poisson_requests(mix: Mix, window: float, seed: int = 0,
                     model: Optional[tuner.B200Model] = None) -> List[Request]:
    rng = np.random.default_rng(seed)
    model = model or tuner.B200Model()
    out: List[Request] = []
    t, rid = 0.0, 0
    cache: Dict[Tuple[int, int, int], str] = {}
    while True:
        t += rng.exponential(1.0 / mix.rate)
        if t >= window:
            break
        u = rng.random()
        if u < mix.f_split:
            kind, shape, alg = SPLIT, mix.split_shape, mix.split_algorithm
        else:
            kind = FP64
            if u < mix.f_split + mix.f_rank_k:
                shape = mix.rank_k_shape
            else:
                d = np.rint(np.exp(rng.uniform(math.log(mix.lo), math.log(mix.hi), size=3))).astype(int)
                shape = (int(d[0]), int(d[1]), int(d[2]))
            if shape not in cache:
                cache[shape] = tuner.rank_candidates(model, shape)[0][0]
            alg = cache[shape]
        out.append(Request(rid, kind, shape, alg, t, nbytes=request_bytes(kind, shape, alg)))
        rid += 1
    return out


class FreeList:
    """First-fit placement in one address range [0, size): an address-ordered list of free
    (offset, length) runs, neighbours merged on release.  Offsets and lengths are multiples of
    `align`.  alloc() returns None when no run is long enough (the caller waits)."""

    def __init__(self, size: int, align: int = 256):
        self.align = align
        self.size = size - size % align
        self.runs: List[Tuple[int, int]] = [(0, self.size)] if self.size else []
        self.used = 0

    def rounded(self, nbytes: int) -> int:
        return -(-max(nbytes, 1) // self.align) * self.align

    def alloc(self, nbytes: int) -> Optional[int]:
        n = self.rounded(nbytes)
        for i, (off, ln) in enumerate(self.runs):
            if ln >= n:
                if ln == n:
                    del self.runs[i]
                else:
                    self.runs[i] = (off + n, ln - n)
                self.used += n
                return off
        return None

    def release(self, off: int, nbytes: int) -> None:
        n = self.rounded(nbytes)
        i = bisect.bisect_left(self.runs, (off, 0))
        if (i < len(self.runs) and self.runs[i][0] < off + n) or (i > 0 and sum(self.runs[i - 1]) > off):
            raise ValueError("release of a range that is (partly) free")
        self.used -= n
        if i > 0 and sum(self.runs[i - 1]) == off:  # merge with the run before
            off, n = self.runs[i - 1][0], self.runs[i - 1][1] + n
            i -= 1
            del self.runs[i]
        if i < len(self.runs) and self.runs[i][0] == off + n:  # ... and the run after
            n += self.runs[i][1]
            del self.runs[i]
        self.runs.insert(i, (off, n))

    def largest(self) -> int:
        return max((ln for _, ln in self.runs), default=0)


class DeviceArena:
    """Request operands carved out of one device allocation made up front, so that the loop
    calls no allocator while it runs (a cudaMalloc of a large block costs the single host
    thread about a millisecond, a cudaFree waits for the device).  A range returns to the
    free list only after the launch that used it has completed, so any stream may reuse it."""

    def __init__(self, nbytes: int, align: int = 256):
        import torch

        self.free = FreeList(nbytes, align)
        self.buf = torch.empty(self.free.size, dtype=torch.uint8, device="cuda")

    def alloc(self, nbytes: int):
        off = self.free.alloc(nbytes)
        return None if off is None else (off, self.buf[off:off + nbytes])

    def release(self, off: int, nbytes: int) -> None:
        self.free.release(off, nbytes)


class Launch:
    """Requests dispatched together, and how to tell that they finished."""

    def __init__(self, kind: str, reqs: List[Request], token):
        self.kind, self.reqs, self.token = kind, reqs, token


@dataclass
class Report:
    window: float
    offered: int
    completed: int
    rejected: int
    backlog: int                  # arrived in the window, not finished at its end
    latencies: List[float] = field(default_factory=list)
    flops_done: float = 0.0
    by_kind: Dict[str, Dict[str, float]] = field(default_factory=dict)
    launches: Dict[str, int] = field(default_factory=dict)
    peak_bytes: int = 0
    run_s: float = 0.0            # the loop's duration (window plus the drain of admitted work)
    stream_busy_s: Dict[str, float] = field(default_factory=dict)  # per stream: device time of its launches
    host_s: Dict[str, float] = field(default_factory=dict)  # host time in admission, launches, completions
    declined: int = 0             # admissions the executor declined (no room for the operands yet)

    def percentile(self, q: float) -> Optional[float]:
        return float(np.percentile(self.latencies, q)) if self.latencies else None

    def summary(self) -> Dict[str, object]:
        return {
            "window_s": self.window, "offered": self.offered, "completed": self.completed,
            "rejected": self.rejected, "backlog_at_end": self.backlog,
            "p50_ms": None if not self.latencies else 1e3 * self.percentile(50),
            "p99_ms": None if not self.latencies else 1e3 * self.percentile(99),
            "tflops_effective": self.flops_done / self.window / 1e12,
            "by_kind": self.by_kind, "launches": self.launches, "peak_admitted_gb": self.peak_bytes / 1e9,
            "run_s": self.run_s,
            "host_s": self.host_s,
            "declined": self.declined,
            "stream_busy_s": self.stream_busy_s,
            "stream_busy_frac": {k: v / self.run_s for k, v in self.stream_busy_s.items()} if self.run_s else {},
        }


class Server:
    """The request loop.  `executor` provides admit(req) (bring operands to the device; False
    when there is no room for them yet, and the request waits as if the budget were full),
    launch(kind, reqs) -> token, done(token) -> bool, release(req) and sync()."""

    def __init__(self, executor, budget_bytes: float = 160e9, max_queue: int = 4096, max_batch: int = 512,
                 inflight: int = 2, clock: Callable[[], float] = time.perf_counter,
                 sleep: Callable[[float], None] = time.sleep, backfill: bool = True, head_wait: float = 0.05,
                 scan: int = 64):
        self.ex = executor
        self.budget = budget_bytes
        self.max_queue = max_queue
        self.max_batch = max_batch
        self.inflight = inflight
        self.clock = clock
        self.sleep = sleep
        self.backfill = backfill    # admit past a head request that does not fit yet
        self.head_wait = head_wait  # ... only while it has waited less than this (seconds)
        self.scan = scan            # queue entries looked at per admission pass

    def run(self, requests: Sequence[Request], window: float, drain: bool = True) -> Report:
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue: List[Request] = []
        ready: Dict[str, deque] = {FP64: deque(), SPLIT: deque()}
        running: Dict[str, deque] = {FP64: deque(), SPLIT: deque()}
        in_use = peak = 0
        rejected = declined = 0
        nxt = 0
        launches = {FP64: 0, SPLIT: 0}
        host = {"admit": 0.0, "launch": 0.0, "complete": 0.0}
        can_hold = getattr(self.ex, "can_hold", lambda r: True)  # could it ever be placed?
        t0 = self.clock()
        now = 0.0
        while True:
            now = self.clock() - t0
            open_ = now < window
            if open_:
                # arrivals up to now
                while nxt < len(reqs) and reqs[nxt].arrival <= now:
                    if (len(queue) >= self.max_queue or reqs[nxt].nbytes > self.budget
                            or not can_hold(reqs[nxt])):
                        rejected += 1
                    else:
                        queue.append(reqs[nxt])
                    nxt += 1
                # admission in arrival order while memory allows; past a request that does not
                # fit yet (backfill) only while that request has waited less than head_wait
                i = 0
                while i < len(queue) and i < self.scan:
                    r = queue[i]
                    if in_use + r.nbytes <= self.budget:
                        ta = self.clock()
                        placed = self.ex.admit(r) is not False  # False: no room for its operands yet
                        if placed:
                            del queue[i]
                            r.admitted = self.clock() - t0
                            host["admit"] += r.admitted + t0 - ta
                            in_use += r.nbytes
                            peak = max(peak, in_use)
                            ready[r.kind].append(r)
                            continue
                        host["admit"] += self.clock() - ta
                        declined += 1
                    if not self.backfill or now - queue[0].arrival > self.head_wait:
                        break
                    i += 1
            # dispatch: all ready FP64 requests form one batch; split requests one by one
            for kind in (FP64, SPLIT):
                while ready[kind] and len(running[kind]) < self.inflight:
                    take = self.max_batch if kind == FP64 else 1
                    group = [ready[kind].popleft() for _ in range(min(take, len(ready[kind])))]
                    tnow = self.clock() - t0
                    for r in group:
                        r.dispatched = tnow
                    running[kind].append(Launch(kind, group, self.ex.launch(kind, group)))
                    host["launch"] += self.clock() - t0 - tnow
                    launches[kind] += 1
            # completions (launches on one stream finish in order)
            progressed = False
            for kind in (FP64, SPLIT):
                while running[kind] and self.ex.done(running[kind][0].token):
                    lch = running[kind].popleft()
                    tdone = self.clock() - t0
                    for r in lch.reqs:
                        r.done = tdone
                        self.ex.release(r)
                        in_use -= r.nbytes
                    host["complete"] += self.clock() - t0 - tdone
                    progressed = True
            busy = any(running.values()) or any(ready.values())
            if not open_ and (not drain or not busy):
                break  # what still waits in the queue is the backlog
            if nxt == len(reqs) and not queue and not busy:
                break  # every request has arrived and finished
            if progressed:
                continue
            if not busy and not queue and open_:
                nxt_t = reqs[nxt].arrival if nxt < len(reqs) else window
                self.sleep(min(max(0.0, min(nxt_t, window) - now), 1e-3))
            else:
                self.sleep(2e-5)
        self.ex.sync()
        run_s = self.clock() - t0
        arrived = [r for r in reqs if r.arrival < window]
        done_in = [r for r in arrived if r.done is not None and r.done <= window]
        rep = Report(window=window, offered=len(arrived), completed=len(done_in), rejected=rejected,
                     backlog=sum(1 for r in arrived if r.done is None or r.done > window) - rejected,
                     latencies=[r.latency for r in done_in], flops_done=sum(r.flops for r in done_in),
                     launches=launches, peak_bytes=peak, run_s=run_s, host_s=host, declined=declined,
                     stream_busy_s=self.ex.busy_seconds() if hasattr(self.ex, "busy_seconds") else {})
        for kind in (FP64, SPLIT):
            ks = [r for r in done_in if r.kind == kind]
            if ks:
                lat = [r.latency for r in ks]
                rep.by_kind[kind] = {"completed": len(ks), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                                     "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                                     "flops_done": sum(r.flops for r in ks),
                                     "tflops_effective": sum(r.flops for r in ks) / window / 1e12}
        return rep


class GpuExecutor:
    """Runs requests on the current CUDA device through the library.  Operands are made on
    the device from a per-request seed (A, B ~ U(-1,1) for FP64; A ~ N(0,1), B log-uniform
    2^-10..2^10 with random sign for split-BF16; C = 0), so a request can be re-run alone
    with the same inputs; keep=True keeps every result for such comparisons."""

    def __init__(self, seed: int = 0, keep: bool = False, arena_bytes: int = 0):
        import torch

        from . import runtime as rt

        self.torch, self.rt = torch, rt
        self.seed, self.keep = seed, keep
        # operands from one up-front allocation (DeviceArena) when arena_bytes > 0, else from
        # torch's caching allocator
        self.arena = DeviceArena(int(arena_bytes)) if arena_bytes else None
        self.blocks: Dict[int, Tuple[int, int]] = {}  # rid -> (offset, bytes) in the arena
        self.streams = {FP64: torch.cuda.Stream(), SPLIT: torch.cuda.Stream()}
        self.plans: Dict[str, object] = {}
        self.results: Dict[int, object] = {}
        self.marks: Dict[str, list] = {FP64: [], SPLIT: []}  # (start, end) timing events per launch
        self.gen = torch.Generator(device="cuda")

    def plan(self, name: str):
        if name == "classical":
            return None
        if name not in self.plans:
            self.plans[name] = self.rt.Plan.from_levels(*tuner.candidate_levels(name))
        return self.plans[name]

    def operands(self, r: Request):
        """A, B, C of a request in one device allocation (column-major views, each starting on
        256 bytes), filled from the request's seed with few calls: at thousands of requests
        per second the host side of admission is part of the loop's budget.  None when the
        arena has no room for them yet."""
        torch = self.torch
        m, n, k = r.shape
        el = 8 if r.kind == FP64 else 4
        pad = lambda x: -(-x // 256) * 256  # noqa: E731  (bytes)
        ob = pad(el * m * k)
        oc = ob + pad(el * k * n)
        total = self.operand_bytes(r)
        if self.arena is not None:
            got = self.arena.alloc(total)
            if got is None:
                return None
            self.blocks[r.rid] = (got[0], total)
            buf = got[1]
        else:
            buf = torch.empty(total, dtype=torch.uint8, device="cuda")
        g = self.gen
        g.manual_seed(self.seed * 1000003 + r.rid)
        dt = torch.float64 if r.kind == FP64 else torch.float32
        ab = buf[:oc].view(dt)
        if r.kind == FP64:
            ab.uniform_(-1, 1, generator=g)
        else:
            ab[:ob // el].normal_(generator=g)
            b = ab[ob // el:]
            b.uniform_(-20, 20, generator=g)  # sign * 2^U(-10, 10): the sign from the draw's sign
            b.copy_(torch.sign(b) * torch.exp2(b.abs() - 10))
        A = ab[:m * k].view(k, m).t()
        B = ab[ob // el:ob // el + k * n].view(n, k).t()
        C = buf[oc:total].view(torch.float64).zero_().view(n, m).t()  # FP64 in both kinds
        return A, B, C

    def operand_bytes(self, r: Request) -> int:
        m, n, k = r.shape
        el = 8 if r.kind == FP64 else 4
        pad = lambda x: -(-x // 256) * 256  # noqa: E731
        return pad(el * m * k) + pad(el * k * n) + 8 * m * n

    def can_hold(self, r: Request) -> bool:
        return self.arena is None or self.arena.free.rounded(self.operand_bytes(r)) <= self.arena.free.size

    def admit(self, r: Request):
        with self.torch.cuda.stream(self.streams[r.kind]):
            r.handle = self.operands(r)
        return r.handle is not None

    def launch(self, kind: str, reqs: List[Request]):
        torch, rt = self.torch, self.rt
        st = self.streams[kind]
        with torch.cuda.stream(st):
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            if kind == FP64:
                rt.batch_submit([self.plan(r.algorithm) for r in reqs], [r.handle[0] for r in reqs],
                                [r.handle[1] for r in reqs], [r.handle[2] for r in reqs], stream=st)
            else:
                for r in reqs:
                    rt.split_gemm(self.plan(r.algorithm), *r.handle, stream=st)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(st)
        self.marks[kind].append((e0, ev))
        return ev

    def busy_seconds(self) -> Dict[str, float]:
        """Device time each stream spent in its launches (after sync()): a launch's events
        bracket its work on its stream, and launches of one stream run one after another."""
        return {k: sum(a.elapsed_time(b) for a, b in v) / 1e3 for k, v in self.marks.items() if v}

    def done(self, token) -> bool:
        return token.query()

    def release(self, r: Request) -> None:
        if self.keep:
            self.results[r.rid] = r.handle[2].cpu()
        r.handle = None
        self.free_operands(r.rid)  # the launch that used them has completed

    def free_operands(self, rid: int) -> None:
        """Return a request's arena range (no-op without an arena: torch frees the tensors)."""
        blk = self.blocks.pop(rid, None)
        if blk is not None:
            self.arena.release(*blk)

    def sync(self) -> None:
        self.torch.cuda.synchronize()

    def warm(self, requests: Sequence[Request]) -> None:
        """First-use costs outside any timed window: every (kind, algorithm) of `requests` runs
        once alone (its plan's tables are uploaded, the workspace pool grows to the largest
        of them), and one FP64 request once through a batch launch."""
        largest: Dict[Tuple[str, str], Request] = {}
        for r in requests:
            key = (r.kind, r.algorithm)
            if key not in largest or r.flops > largest[key].flops:
                largest[key] = r
        for r in largest.values():
            self.run_alone(r)
        fp = next((r for r in requests if r.kind == FP64), None)
        if fp is not None:
            ops = self.operands(fp)
            if ops is not None:
                A, B, C = ops
                self.rt.batch_submit([self.plan(fp.algorithm)], [A], [B], [C], stream=self.streams[FP64])
                self.torch.cuda.synchronize()
                self.free_operands(fp.rid)

    def run_alone(self, r: Request):
        """The request by itself (same inputs, same algorithm), for comparison."""
        ops = self.operands(r)
        if ops is None:
            raise RuntimeError("no room in the arena for the request's operands")
        A, B, C = ops
        if r.kind == FP64:
            p = self.plan(r.algorithm)
            if p is None:
                self.rt.plain_gemm(A, B, C)
            else:
                self.rt.fmm_gemm(p, A, B, C, "abc")
        else:
            self.rt.split_gemm(self.plan(r.algorithm), A, B, C)
        self.torch.cuda.synchronize()
        out = C.cpu()
        self.free_operands(r.rid)
        return out


def shard_requests(requests: Sequence[Request], world: int, model: Optional[tuner.B200Model] = None) -> List[List[Request]]:
    """Requests to GPUs for a multi-GPU server: in arrival order, each request goes to the
    GPU with the least modelled outstanding work (work drains at one GPU-second per second;
    among idle GPUs, the one given the least work so far), the same deterministic answer
    on every rank without any exchange."""
    model = model or tuner.B200Model()
    load = [0.0] * world   # modelled work still queued on each GPU
    total = [0.0] * world  # work given to each GPU so far (breaks ties between idle GPUs)
    last = 0.0
    out: List[List[Request]] = [[] for _ in range(world)]
    for r in sorted(requests, key=lambda q: q.arrival):
        dt = r.arrival - last
        last = r.arrival
        load = [max(0.0, x - dt) for x in load]
        cost = model_cost(model, r)
        g = min(range(world), key=lambda i: (load[i], total[i], i))
        load[g] += cost
        total[g] += cost
        out[g].append(r)
    return out


def model_cost(model: tuner.B200Model, r: Request) -> float:
    m, n, k = r.shape
    if r.kind == SPLIT:
        # bf16 plane products at about half the measured dense bf16 rate, six per product
        plan = tuner.plan_of(r.algorithm)
        frac = plan.rank / float(np.prod(plan.dims)) if plan is not None else 1.0
        return 6 * frac * r.flops / 0.8e15
    return tuner.model_time(model, r.algorithm, m, n, k)
