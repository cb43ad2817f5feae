"""The serving loop's scheduling on the CPU: a simulated executor whose launches take
their modelled time on a simulated clock, so admission, batching, overlap and the
window accounting are checked exactly and quickly.  (GPU runs: tests/test_gpu_serve.py.)"""
import numpy as np
import pytest

from fmm_gen_b200 import serve, tuner


class SimClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class SimExecutor:
    """One simulated GPU: launches (from either stream) run back to back, each taking the
    modelled time of its requests (a batch: the sum, as one persistent launch shares the
    SMs among them)."""

    def __init__(self, clock, speed=1.0):
        self.clock, self.speed = clock, speed
        self.gpu_free = 0.0
        self.admitted, self.released, self.batches = [], [], []
        self.model = tuner.B200Model()

    def admit(self, r):
        self.admitted.append(r.rid)

    def launch(self, kind, reqs):
        cost = sum(serve.model_cost(self.model, r) for r in reqs) / self.speed
        start = max(self.clock(), self.gpu_free)
        self.gpu_free = start + cost
        self.batches.append((kind, [r.rid for r in reqs]))
        return start + cost

    def done(self, token):
        return self.clock() >= token

    def release(self, r):
        self.released.append(r.rid)

    def sync(self):
        pass


def run(reqs, window, **kw):
    clk = SimClock()
    ex = SimExecutor(clk, kw.pop("speed", 1.0))
    srv = serve.Server(ex, clock=clk, sleep=clk.sleep, **kw)
    return srv.run(reqs, window), ex


def test_poisson_stream_is_seeded_and_has_the_mix():
    mix = serve.Mix(rate=2000.0)
    a = serve.poisson_requests(mix, 1.0, seed=3)
    b = serve.poisson_requests(mix, 1.0, seed=3)
    assert [(r.shape, r.arrival) for r in a] == [(r.shape, r.arrival) for r in b]
    assert 1800 < len(a) < 2200
    kinds = [r.kind for r in a]
    assert abs(kinds.count(serve.SPLIT) / len(a) - 0.10) < 0.03
    rk = sum(1 for r in a if r.shape == (16000, 16000, 256))
    assert abs(rk / len(a) - 0.10) < 0.03
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)


def test_light_load_serves_everything_with_service_time_latency():
    mix = serve.Mix(rate=50.0, f_rank_k=0.0, f_split=0.0, lo=256, hi=512)
    reqs = serve.poisson_requests(mix, 0.5, seed=1)
    rep, ex = run(reqs, 0.5)
    assert rep.completed + rep.backlog == rep.offered and rep.rejected == 0
    assert rep.completed >= rep.offered - 2
    assert max(rep.latencies) < 0.01      # no queueing at 50 req/s of small GEMMs
    assert sorted(ex.released) == sorted(ex.admitted)


def test_requests_arriving_during_a_launch_join_the_next_batch():
    mix = serve.Mix(rate=4000.0, f_rank_k=0.0, f_split=0.0, lo=1024, hi=2048)
    reqs = serve.poisson_requests(mix, 0.05, seed=2)
    rep, ex = run(reqs, 0.05, inflight=1)
    fp = [ids for kind, ids in ex.batches if kind == serve.FP64]
    assert len(fp) < len(reqs) and max(len(ids) for ids in fp) > 1
    # batches are formed in arrival order
    flat = [i for ids in fp for i in ids]
    assert flat == sorted(flat)


def test_admission_respects_the_budget_and_the_queue_bounds_overload():
    mix = serve.Mix(rate=2000.0)
    reqs = serve.poisson_requests(mix, 0.2, seed=4)
    budget = 20e9
    rep, ex = run(reqs, 0.2, budget_bytes=budget, max_queue=64)
    assert rep.peak_bytes <= budget
    assert rep.rejected > 0                      # overload: the bounded queue sheds
    assert rep.backlog > 0
    assert rep.completed + rep.backlog + rep.rejected == rep.offered
    assert all(r.done is None or r.done >= r.arrival for r in reqs)


def test_split_and_fp64_streams_overlap():
    mix = serve.Mix(rate=400.0, f_rank_k=0.0, f_split=0.5, lo=256, hi=1024)
    reqs = serve.poisson_requests(mix, 0.1, seed=5)
    rep, ex = run(reqs, 0.1)
    assert {k for k, _ in ex.batches} == {serve.FP64, serve.SPLIT}
    assert rep.by_kind[serve.FP64]["p50_ms"] < rep.by_kind[serve.SPLIT]["p50_ms"]


def test_sharding_is_deterministic_and_balanced():
    reqs = serve.poisson_requests(serve.Mix(rate=2000.0), 0.5, seed=6)
    a = serve.shard_requests(reqs, 4)
    b = serve.shard_requests(reqs, 4)
    assert [[r.rid for r in s] for s in a] == [[r.rid for r in s] for s in b]
    assert sorted(r.rid for s in a for r in s) == [r.rid for r in reqs]
    model = tuner.B200Model()
    work = [sum(serve.model_cost(model, r) for r in s) for s in a]
    assert max(work) / min(work) < 1.3


def _req(rid, kind, shape, alg, t, nbytes):
    return serve.Request(rid, kind, shape, alg, t, nbytes=int(nbytes))


def test_backfill_admits_past_a_request_that_does_not_fit_yet():
    """A large request that must wait for memory does not hold back the small ones behind it
    (they are admitted past it), and with head_wait it is admitted once memory frees."""
    big = [_req(0, serve.FP64, (4096, 4096, 4096), "classical", 0.0, 8e9),
           _req(1, serve.SPLIT, (8192, 8192, 8192), "222-2", 1e-4, 5e9)]
    small = [_req(2 + i, serve.FP64, (256, 256, 256), "classical", 2e-4 + 1e-5 * i, 1e7) for i in range(20)]
    reqs = big + small

    def fresh():
        return [serve.Request(r.rid, r.kind, r.shape, r.algorithm, r.arrival, nbytes=r.nbytes) for r in reqs]

    rep_fifo, ex_fifo = run(fresh(), 0.5, budget_bytes=10e9, backfill=False)
    rep_bf, ex_bf = run(fresh(), 0.5, budget_bytes=10e9, backfill=True, head_wait=1.0)
    # FIFO: every small request is admitted after the split request (which waits for the
    # first one's memory); with backfill they are admitted before it
    assert ex_fifo.admitted.index(1) < min(ex_fifo.admitted.index(2 + i) for i in range(20))
    assert ex_bf.admitted.index(1) > max(ex_bf.admitted.index(2 + i) for i in range(20))
    assert rep_bf.completed == rep_fifo.completed == len(reqs)
    small_lat = lambda rep: np.median([r for r in rep.latencies])  # noqa: E731
    assert small_lat(rep_bf) < small_lat(rep_fifo)


def test_backfill_stops_when_the_waiting_request_has_waited_long_enough():
    """A steady stream of small requests that keeps the budget busy cannot starve a large one:
    past head_wait nothing is admitted past it, so it gets the memory as launches finish."""
    first = _req(0, serve.FP64, (4096, 4096, 4096), "classical", 0.0, 6e9)
    big = _req(1, serve.SPLIT, (8192, 8192, 8192), "222-2", 1e-4, 6e9)
    small = [_req(2 + i, serve.FP64, (1024, 1024, 1024), "classical", 2e-4 + 2e-4 * i, 2e9) for i in range(400)]
    rep, ex = run([first, big] + small, 0.2, budget_bytes=10e9, backfill=True, head_wait=0.005)
    assert 1 in ex.admitted
    pos = ex.admitted.index(1)
    assert pos < len(ex.admitted) - 1  # admitted while small requests were still arriving


def test_free_list_places_first_fit_and_merges_neighbours():
    fl = serve.FreeList(10 * 256, align=256)
    a = fl.alloc(256)
    b = fl.alloc(300)            # rounded up to 512
    c = fl.alloc(256)
    assert (a, b, c) == (0, 256, 768) and fl.used == 1024
    assert fl.alloc(7 * 256) is None  # 6 blocks left
    fl.release(b, 300)
    assert fl.alloc(512) == 256  # first fit reuses the hole
    fl.release(256, 512)
    fl.release(a, 256)
    fl.release(c, 256)           # all three merge back with the tail
    assert fl.runs == [(0, 10 * 256)] and fl.used == 0
    with pytest.raises(ValueError):
        fl.release(0, 256)       # already free


def test_free_list_random_sequence_matches_a_bitmap():
    rng = np.random.default_rng(7)
    size, align = 4096, 16
    fl = serve.FreeList(size, align)
    taken = np.zeros(size // align, dtype=bool)
    live = []
    for _ in range(3000):
        if live and rng.random() < 0.45:
            off, n = live.pop(int(rng.integers(len(live))))
            fl.release(off, n)
            taken[off // align:(off + fl.rounded(n)) // align] = False
        else:
            n = int(rng.integers(1, 400))
            off = fl.alloc(n)
            blocks = fl.rounded(n) // align
            # first fit: the lowest free run that is long enough
            want = None
            run = 0
            for i, t in enumerate(taken):
                run = 0 if t else run + 1
                if run == blocks:
                    want = (i - blocks + 1) * align
                    break
            assert off == want
            if off is not None:
                assert not taken[off // align:off // align + blocks].any()
                taken[off // align:off // align + blocks] = True
                live.append((off, n))
        free_runs = sum(ln for _, ln in fl.runs)
        assert free_runs == size - int(taken.sum()) * align == size - fl.used
        assert all(fl.runs[i][0] + fl.runs[i][1] < fl.runs[i + 1][0] for i in range(len(fl.runs) - 1))


class ArenaSimExecutor(SimExecutor):
    """The simulated GPU with an operand arena: admission is declined while the arena has no
    room for the request's operands, whatever the budget says."""

    def __init__(self, clock, arena_bytes):
        super().__init__(clock)
        self.fl = serve.FreeList(arena_bytes, 256)
        self.where = {}

    def admit(self, r):
        off = self.fl.alloc(r.nbytes)
        if off is None:
            return False
        self.where[r.rid] = off
        return super().admit(r)

    def release(self, r):
        self.fl.release(self.where.pop(r.rid), r.nbytes)
        super().release(r)


def test_requests_wait_while_the_executor_declines_them():
    mix = serve.Mix(rate=400.0, f_rank_k=0.5, f_split=0.0, lo=256, hi=1024)
    reqs = serve.poisson_requests(mix, 0.3, seed=4)
    big = max(r.nbytes for r in reqs)
    clk = SimClock()
    ex = ArenaSimExecutor(clk, 3 * big)      # room for about three rank-k requests at once
    rep = serve.Server(ex, budget_bytes=1e15, clock=clk, sleep=clk.sleep).run(reqs, 0.3)
    assert rep.declined > 0                  # the budget alone would have admitted them
    assert sorted(ex.released) == sorted(ex.admitted)
    assert ex.fl.used == 0 and ex.fl.runs == [(0, ex.fl.size)]
    assert rep.completed + rep.backlog + rep.rejected == rep.offered
