"""Oracle parity at the benchmark configurations' own shapes.

The CUDA path (through the C ABI) against the oracle -- the bit-exact CPU restatement of
the reference's generated code, pinned by the golden vectors -- on the same seeded
inputs, at the full sizes of every configuration:

  * one-level Strassen 222-1 abc, 2048^3, C = 0 (`control.py 1 222 1 abc`);
  * the two-level hybrid 222-1 x 333-1 abc at 14400 x 14400 x 480, 4000 x 16000 x 2000
    and 16384^3 (A, B, C ~ U(-1, 1));
  * the first problems of the 512-problem batch (m, n, k log-uniform in [256, 4096]
    from seed 0), one persistent batch launch with an algorithm per problem;
  * the split-BF16 222-2 FMM at 8192^3 against the oracle's classical FP64 product of the
    same FP32 inputs, both input sets.

Tolerances (the same as the small-size parity tests):
  * FP64 paths: relative Frobenius difference to the oracle <= RTOL = 1e-13 and max-norm
    difference <= 2 * algebra.error_bound(...).  The oracle adds each KC = 256 chunk into C
    with a separate multiply and add, the GPU accumulates the whole k range with fused
    multiply-adds, so results agree to rounding, not bits.
  * split-BF16: relative Frobenius error of the update against the FP64 oracle
    <= RTOL_SPLIT = 1e-6.
The reference's own check of a run is the same comparison against its plain GEMM at the
run's shape (meta/misc_gen.py:224, bl_compare_error in common/dgemm/bl_dgemm_util.c:300-314).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import algebra, build, runtime as rt, tuner  # noqa: E402
from tests.golden_util import inputs  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-13
RTOL_SPLIT = 1e-6
DEV = "cuda"


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    rt.load_library()


def to_dev(x: np.ndarray):
    dt = torch.float32 if x.dtype == np.float32 else torch.float64
    t = rt.colmajor(x.shape[0], x.shape[1], dtype=dt, device=DEV)
    t.copy_(torch.from_numpy(np.ascontiguousarray(x)))
    return t


def tables(plan):
    dims, nterms, rows, cols, coefs = rt.plan_tables(plan)
    return (dims, plan.rank, nterms, rows, cols, coefs)


def rel_fro(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def check_against_oracle(oracle_lib, plan, A, B, C, got):
    m, k = A.shape
    n = B.shape[1]
    want = C.copy(order="F")
    oracle_lib.fmm(tables(plan.algebra), "abc", A, B, want)
    rel = rel_fro(got, want)
    bound = algebra.error_bound(plan.algebra, m, n, k, np.abs(A).max(), np.abs(B).max(),
                                max(np.abs(C).max(), 1e-300))
    diff = float(np.abs(got - want).max())
    assert rel <= RTOL, (m, n, k, rel)
    assert diff <= 2 * bound, (m, n, k, diff, bound)
    return rel


def test_config1_strassen_2048_c_zero(oracle_lib):
    """222-1 abc, 2048^3, A, B ~ U(-1, 1), C = 0: C += A*B."""
    m = n = k = 2048
    A, B, _ = inputs(2048, m, n, k)
    C = np.zeros((m, n), order="F")
    plan = rt.Plan.from_levels(["222"], [1])
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.fmm_gemm(plan, dA, dB, dC, "abc")
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    check_against_oracle(oracle_lib, plan, A, B, C, dC.cpu().numpy())


@pytest.mark.parametrize("shape", [(14400, 14400, 480), (4000, 16000, 2000), (16384, 16384, 16384)],
                         ids=lambda s: "x".join(map(str, s)))
def test_config2_hybrid_222x333_full_shapes(oracle_lib, shape):
    """222-1 x 333-1 abc at the three shapes of the hybrid configuration, A, B, C ~ U(-1, 1)."""
    m, n, k = shape
    A, B, C = inputs(m + 3 * n + 7 * k, m, n, k)
    plan = rt.Plan.from_levels(["222", "333"], [1, 1])
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.fmm_gemm(plan, dA, dB, dC, "abc")
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    got = dC.cpu().numpy()
    del dA, dB, dC
    torch.cuda.empty_cache()
    check_against_oracle(oracle_lib, plan, A, B, C, got)


BATCH_HEAD = 12  # problems of the 512-problem batch checked against the oracle


def test_config4_batch_head_against_oracle(oracle_lib):
    """The first problems of the 512-problem batch in one persistent launch, each problem on
    one of the tuner's candidate algorithms in turn; every result against the oracle."""
    shapes = tuner.random_batch_shapes(512, seed=0)[:BATCH_HEAD]
    names = [tuner.CANDIDATES[i % len(tuner.CANDIDATES)] for i in range(len(shapes))]
    plans = {}
    for nm in set(names) - {"classical"}:
        plans[nm] = rt.Plan.from_levels(*tuner.candidate_levels(nm))
    host = [inputs(1000 + i, m, n, k) for i, (m, n, k) in enumerate(shapes)]
    As = [to_dev(h[0]) for h in host]
    Bs = [to_dev(h[1]) for h in host]
    Cs = [to_dev(h[2]) for h in host]
    batch = rt.Batch(shapes, [plans.get(nm) for nm in names])
    batch.run(As, Bs, Cs)
    torch.cuda.synchronize()
    batch.close()
    assert rt.load_library().fmm_device_status(1) == 0
    for (m, n, k), nm, (A, B, C), dC in zip(shapes, names, host, Cs):
        got = dC.cpu().numpy()
        if nm == "classical":
            want = C.copy(order="F")
            oracle_lib.bl_dgemm(A, B, want)
            assert rel_fro(got, want) <= RTOL, (m, n, k, nm)
        else:
            check_against_oracle(oracle_lib, plans[nm], A, B, C, got)


def _split_operand(rng, n, which):
    if which == "normal":
        return np.asfortranarray(rng.standard_normal((n, n)).astype(np.float32))
    sign = np.where(rng.random((n, n)) < 0.5, -1.0, 1.0)
    return np.asfortranarray((sign * np.exp2(rng.uniform(-10, 10, (n, n)))).astype(np.float32))


@pytest.mark.parametrize("which", ["normal", "loguniform"])
def test_config3_split_bf16_8192_against_fp64_oracle(oracle_lib, which):
    """222-2 split-BF16 FMM, 8192^3, FP32 inputs (N(0, 1); sign * 2^U(-10, 10)), C = 0: the
    relative Frobenius error against the oracle's classical FP64 product is <= 1e-6."""
    n = 8192
    rng = np.random.default_rng(8192 + (0 if which == "normal" else 1))
    A, B = _split_operand(rng, n, which), _split_operand(rng, n, which)
    C = np.zeros((n, n), order="F")
    plan = rt.Plan.from_levels(["222"], [2])
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.split_gemm(plan, dA, dB, dC)
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    got = dC.cpu().numpy()
    del dA, dB, dC
    torch.cuda.empty_cache()
    want = np.zeros((n, n), order="F")
    oracle_lib.bl_dgemm(np.asfortranarray(A.astype(np.float64)), np.asfortranarray(B.astype(np.float64)), want)
    assert rel_fro(got, want) <= RTOL_SPLIT
