"""The serving loop on the GPU: a short Poisson stream of mixed FP64 (several shapes,
FMM and classical) and split-BF16 requests under a small HBM budget, so requests queue,
batch and overlap.  Every result must be bit-identical to the same request run alone
(same inputs, same algorithm), and correct against an FP64 reference: relative
Frobenius error <= 1e-13 for FP64 requests, <= 1e-6 for split-BF16 ones.  Run with operands
from torch's caching allocator and from the executor's arena (smaller than the budget, so some
admissions are declined until a range frees up)."""
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import build, runtime as rt, serve  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    rt.load_library()


@pytest.mark.parametrize("arena_bytes", [0, 0.5e9], ids=["torch_allocator", "arena"])
def test_results_are_the_same_alone_and_in_the_mix(arena_bytes):
    mix = serve.Mix(rate=600.0, f_rank_k=0.1, f_split=0.2, lo=200, hi=1500, rank_k_shape=(3000, 3000, 256),
                    split_shape=(1024, 1024, 1024), split_algorithm="222-1")
    reqs = serve.poisson_requests(mix, 0.15, seed=11)
    # make sure an FMM algorithm is exercised inside a batch
    for r in reqs[:6]:
        if r.kind == serve.FP64:
            r.algorithm = "222-1"
    ex = serve.GpuExecutor(seed=5, keep=True, arena_bytes=arena_bytes)
    for kind in (serve.FP64, serve.SPLIT):  # first-use costs (plans, kernels) outside the loop
        ex.run_alone(next(r for r in reqs if r.kind == kind))
    # all arrivals come in the first 0.15 s; the window is long enough for every request
    rep = serve.Server(ex, budget_bytes=0.6e9, max_queue=10_000, max_batch=16).run(reqs, 30.0)
    done = [r for r in reqs if r.done is not None]
    assert len(done) == len(reqs) and rep.rejected == 0
    assert rep.launches[serve.FP64] < sum(1 for r in reqs if r.kind == serve.FP64)  # batched
    assert rt.load_library().fmm_device_status(1) == 0
    for r in done:
        alone = ex.run_alone(r)
        assert torch.equal(ex.results[r.rid], alone), (r.rid, r.kind, r.shape, r.algorithm)
    # correctness of a sample against FP64 classical products of the same inputs
    for r in [q for q in done if q.kind == serve.SPLIT][:3] + [q for q in done if q.kind == serve.FP64][:5]:
        A, B, C = ex.operands(r)
        ref = (A.double() @ B.double()).cpu()
        torch.cuda.synchronize()
        ex.free_operands(r.rid)
        err = ((ex.results[r.rid] - ref).norm() / ref.norm()).item()
        assert err <= (1e-6 if r.kind == serve.SPLIT else 1e-13), (r.kind, r.shape, err)
