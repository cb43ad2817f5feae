"""Split-BF16 FMM on the tensor cores (fmm_split_gemm_dev) through the C ABI.

FP32 A and B, FP64 C.  The oracle is the classical FP64 product of the same FP32 inputs
(oracle.cpu.bl_dgemm at small sizes; an independent FP64 GEMM, torch.matmul on float64,
at the full size), and the measure is the relative Frobenius error of the update,
    ||C_got - C_ref||_F / ||C_ref - C0||_F  <=  RTOL_SPLIT = 1e-6,
on inputs drawn like the split-precision workload: A ~ N(0, 1), B = sign * 2^U(-10, 10).
A plain bf16 product of the same inputs is ~1e-3 off; the three-plane split is expected
near 1e-7 (classical) to a few 1e-7 (two Strassen levels, whose sums grow the operands).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import build, runtime as rt  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL_SPLIT = 1e-6
DEV = "cuda"


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    rt.load_library()


_plans = {}


def plan_for(algs, levels):
    key = (tuple(algs), tuple(levels))
    if key not in _plans:
        _plans[key] = rt.Plan.from_levels(algs, levels)
    return _plans[key]


def split_inputs(seed, m, n, k, c0=True):
    rng = np.random.default_rng(seed)
    A = np.asfortranarray(rng.standard_normal((m, k)).astype(np.float32))
    sign = np.where(rng.random((k, n)) < 0.5, -1.0, 1.0)
    B = np.asfortranarray((sign * np.exp2(rng.uniform(-10, 10, (k, n)))).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((m, n)) if c0 else np.zeros((m, n)))
    return A, B, C


def to_dev(x: np.ndarray):
    dt = torch.float32 if x.dtype == np.float32 else torch.float64
    t = rt.colmajor(x.shape[0], x.shape[1], dtype=dt, device=DEV)
    t.copy_(torch.from_numpy(np.ascontiguousarray(x)))
    return t


def run_split(plan, A, B, C):
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.split_gemm(plan, dA, dB, dC)
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    return dC.cpu().numpy()


def oracle_update(oracle_lib, A, B, C):
    want = np.asfortranarray(C.copy())
    oracle_lib.bl_dgemm(A.astype(np.float64), B.astype(np.float64), want)
    return want


def rel_update(got, want, C0):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want - C0), 1e-300))


@pytest.mark.parametrize("shape", [(128, 128, 64), (256, 384, 200), (300, 200, 130), (1, 1, 1), (517, 389, 1000),
                                   (129, 130, 65)])
def test_split_classical_matches_oracle(oracle_lib, shape):
    m, n, k = shape
    A, B, C = split_inputs(sum(shape), m, n, k)
    got = run_split(None, A, B, C)
    want = oracle_update(oracle_lib, A, B, C)
    assert rel_update(got, want, C) <= RTOL_SPLIT


@pytest.mark.parametrize("algs,levels,shape", [
    (["222"], [1], (1024, 1024, 1024)),
    (["222"], [1], (1030, 1001, 777)),     # fringes on every side, peeled like the FP64 path
    (["222"], [2], (2048, 2048, 2048)),
    (["222"], [2], (1100, 900, 1300)),
    (["222", "333"], [1, 1], (1000, 900, 700)),
    (["232"], [1], (517, 389, 263)),
])
def test_split_fmm_matches_oracle(oracle_lib, algs, levels, shape):
    m, n, k = shape
    A, B, C = split_inputs(sum(shape) + len(algs), m, n, k)
    got = run_split(plan_for(algs, levels), A, B, C)
    want = oracle_update(oracle_lib, A, B, C)
    assert rel_update(got, want, C) <= RTOL_SPLIT


def test_split_zero_update_and_empty_dims():
    A, B, C = split_inputs(7, 64, 48, 32)
    got = run_split(plan_for(["222"], [1]), np.zeros_like(A), B, C)
    assert np.array_equal(got, C)  # a zero operand leaves C bit-identical
    dC = to_dev(C)
    for m, n, k in ((0, 48, 32), (64, 0, 32), (64, 48, 0)):
        rt.split_gemm(None, rt.colmajor(m, k, dtype=torch.float32, device=DEV),
                      rt.colmajor(k, n, dtype=torch.float32, device=DEV), rt.colmajor(m, n, device=DEV))
    torch.cuda.synchronize()
    assert np.array_equal(dC.cpu().numpy(), C)


def test_split_is_deterministic_and_additive():
    """Two runs from the same C give bit-identical results (per-tile product order is
    fixed by the tickets); a second call adds the same update again."""
    A, B, C = split_inputs(11, 1000, 900, 700)
    plan = plan_for(["222", "333"], [1, 1])
    dA, dB = to_dev(A), to_dev(B)
    outs = []
    for _ in range(2):
        dC = to_dev(C)
        rt.split_gemm(plan, dA, dB, dC)
        outs.append(dC.clone())
    rt.split_gemm(plan, dA, dB, dC)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
    upd = outs[0] - to_dev(C)
    twice = dC - to_dev(C)
    assert ((twice - 2 * upd).norm() / upd.norm()).item() <= 1e-12


def test_split_views_and_streams():
    """Sub-matrix views (ld > rows) and a side stream."""
    m, n, k = 333, 255, 190
    A, B, C = split_inputs(5, m + 7, n + 3, k + 5)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    vA, vB, vC = dA[3:3 + m, 2:2 + k], dB[1:1 + k, :n], dC[5:5 + m, 1:1 + n]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        rt.split_gemm(plan_for(["222"], [1]), vA, vB, vC, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    want = C.copy()
    want[5:5 + m, 1:1 + n] += A[3:3 + m, 2:2 + k].astype(np.float64) @ B[1:1 + k, :n].astype(np.float64)
    got = dC.cpu().numpy()
    outside = np.ones_like(C, dtype=bool)
    outside[5:5 + m, 1:1 + n] = False
    assert np.array_equal(got[outside], C[outside])
    assert rel_update(got, want, C) <= RTOL_SPLIT


def test_split_full_size_222_2_8192():
    """The split-precision workload at full size: 222 two levels, 8192^3."""
    n = 8192
    g = torch.Generator(device=DEV).manual_seed(3)
    A = rt.colmajor(n, n, dtype=torch.float32, device=DEV).normal_(generator=g)
    e = torch.empty((n, n), device=DEV).uniform_(-10, 10, generator=g)
    s = torch.empty((n, n), device=DEV).uniform_(-1, 1, generator=g).sign()
    B = rt.colmajor(n, n, dtype=torch.float32, device=DEV).copy_(s * torch.exp2(e))
    del e, s
    C = rt.colmajor(n, n, device=DEV).zero_()
    rt.split_gemm(plan_for(["222"], [2]), A, B, C)
    ref = A.double() @ B.double()
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    assert ((C - ref).norm() / ref.norm()).item() <= RTOL_SPLIT


@pytest.mark.parametrize("algs,levels,shape", [
    (["222"], [2], (1000, 900, 1100)),        # 16 blocks per operand, fringes on every side
    (["333"], [1], (700, 650, 610)),           # 9 blocks
    (["222", "333"], [1, 1], (1210, 1190, 1300)),  # 36 blocks: the largest staged tile
    (["222"], [1], (4100, 4097, 4103)),
])
def test_split_operand_forms_are_bit_identical(algs, levels, shape):
    """The operand planes formed from one staged read of each operand (all products per tile,
    the default) and one product per CTA give the same result bit for bit."""
    m, n, k = shape
    lib = rt.load_library()
    p = rt.Plan.from_levels(algs, levels)
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    A = rt.colmajor(m, k, dtype=torch.float32, device="cuda").normal_(generator=g)
    B = rt.colmajor(k, n, dtype=torch.float32, device="cuda").normal_(generator=g)
    C0 = rt.colmajor(m, n, device="cuda").uniform_(-1, 1, generator=g)
    out = []
    try:
        for form in (0, 1):
            assert lib.fmm_debug_set(5, form) == 0
            C = rt.colmajor(m, n, device="cuda").copy_(C0)
            rt.split_gemm(p, A, B, C)
            torch.cuda.synchronize()
            out.append(C)
    finally:
        assert lib.fmm_debug_set(5, 0) == 0
    assert lib.fmm_device_status(1) == 0
    assert torch.equal(out[0], out[1])
