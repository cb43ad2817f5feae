"""GPU parity: the sm_100a path through the C ABI against the oracle and against the
reference's own generated code (golden vectors), plus size-independent properties at
the full benchmark sizes.

Tolerances (written here, used below):
  * vs the reference / oracle at small sizes: relative Frobenius difference
    <= RTOL_SMALL = 1e-13 and max-norm difference <= 2 * algebra.error_bound(...)
    (the GPU accumulates with fused multiply-adds and a full-depth accumulator; the
    reference adds each KC=256 chunk into C, so results agree to rounding, not bits).
  * full sizes: max-norm error against an independent classical FP64 GEMM (cuBLAS via
    torch.matmul) <= error_bound(...) for FMM and for the plain kernel.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import algebra, build, runtime as rt  # noqa: E402
from tests.golden_util import golden_cases, inputs, plain_cases  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL_SMALL = 1e-13
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


def to_dev(x: np.ndarray):
    t = rt.colmajor(x.shape[0], x.shape[1], device=DEV)
    t.copy_(torch.from_numpy(np.ascontiguousarray(x)))
    return t


def rel_fro(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tables(plan):
    dims, nterms, rows, cols, coefs = rt.plan_tables(plan)
    return (dims, plan.rank, nterms, rows, cols, coefs)


CASES = golden_cases()


@pytest.mark.parametrize("case", CASES, ids=[f"{'_'.join(c[0])}-{c[2]}-{c[3]}" for c in CASES])
def test_gpu_matches_reference_golden(case):
    algs, levels, pack, _, (m, n, k), seed, want = case
    A, B, C = inputs(seed, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    p = plan_for(algs, levels)
    rt.fmm_gemm(p, dA, dB, dC, pack)
    got = dC.cpu().numpy()
    assert rel_fro(got, want) <= RTOL_SMALL
    bound = algebra.error_bound(p.algebra, m, n, k, np.abs(A).max(), np.abs(B).max(), np.abs(C).max())
    assert np.abs(got - want).max() <= 2 * bound


@pytest.mark.parametrize("case", plain_cases(), ids=lambda c: str(c[0]))
def test_gpu_plain_matches_reference_golden(case):
    (m, n, k), seed, want = case
    A, B, C = inputs(seed, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.plain_gemm(dA, dB, dC)
    assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL


ORACLE_CASES = [
    (["222"], [1], (517, 389, 263)),
    (["222"], [1], (1024, 1024, 1024)),
    (["222"], [2], (600, 500, 400)),
    (["232"], [1], (403, 301, 299)),
    (["333"], [1], (500, 400, 300)),
    (["222", "333"], [1, 1], (400, 300, 250)),
    (["424"], [1], (300, 256, 200)),
    (["336"], [1], (288, 400, 150)),
    (["222", "232"], [1, 1], (333, 222, 211)),
    # the ABC pack type pre-sums operands in HBM from ms*ns >= 2^17, ks >= 64 (1024^3 above too)
    (["222"], [1], (2056, 2052, 606)),
    (["333"], [1], (3080, 3090, 800)),
    (["424"], [1], (4104, 2060, 1034)),
    # 336 at two levels: 100 operand terms per product side (beyond the sums' staged term table)
    (["336"], [2], (3000, 14420, 910)),
]


@pytest.mark.parametrize("pack", ["abc", "ab", "naive"])
@pytest.mark.parametrize("algs,levels,shape", ORACLE_CASES, ids=lambda x: str(x))
def test_gpu_matches_oracle(oracle_lib, algs, levels, shape, pack):
    m, n, k = shape
    A, B, C = inputs(sum(shape) + 7 * len(algs) + levels[0], m, n, k)
    p = plan_for(algs, levels)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.fmm_gemm(p, dA, dB, dC, pack)
    got = dC.cpu().numpy()
    want = C.copy(order="F")
    oracle_lib.fmm(tables(p.algebra), pack, A, B, want)
    assert rel_fro(got, want) <= RTOL_SMALL


@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 3, 1), (8, 4, 2), (15, 9, 1), (16, 8, 3), (47, 23, 5),
                                   (48, 24, 6), (129, 130, 17), (256, 8, 1000)])
def test_gpu_edge_shapes(oracle_lib, shape):
    """Tiny, fringe-only (md = 0 or kd = 0), single-tile and tall-k shapes."""
    m, n, k = shape
    for algs, levels in ((["222"], [1]), (["222", "333"], [1, 1])):
        p = plan_for(algs, levels)
        A, B, C = inputs(11, m, n, k)
        dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
        rt.fmm_gemm(p, dA, dB, dC, "abc")
        want = C.copy(order="F")
        oracle_lib.fmm(tables(p.algebra), "abc", A, B, want)
        assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL


def test_gpu_zero_sizes_are_noops():
    p = plan_for(["222"], [1])
    for (m, n, k) in ((0, 4, 4), (4, 0, 4), (4, 4, 0)):
        dA = rt.colmajor(m, k, device=DEV).fill_(1)
        dB = rt.colmajor(k, n, device=DEV).fill_(1)
        dC = rt.colmajor(m, n, device=DEV).fill_(3)
        rt.fmm_gemm(p, dA, dB, dC, "abc")
        rt.plain_gemm(dA, dB, dC)
        assert bool((dC == 3).all())


def test_gpu_padded_leading_dimensions_and_views(oracle_lib):
    """ld > m, views into larger buffers, odd k so that B sub-blocks start unaligned."""
    m, n, k = 203, 181, 157
    A, B, C = inputs(21, m, n, k)
    big = lambda r, c: rt.colmajor(r + 13, c + 3, device=DEV).fill_(float("nan"))
    bA, bB, bC = big(m, k), big(k, n), big(m, n)
    dA, dB, dC = bA[5:5 + m, 1:1 + k], bB[3:3 + k, 2:2 + n], bC[7:7 + m, 0:n]
    dA.copy_(torch.from_numpy(A))
    dB.copy_(torch.from_numpy(B))
    dC.copy_(torch.from_numpy(C))
    p = plan_for(["222"], [1])
    rt.fmm_gemm(p, dA, dB, dC, "abc")
    want = C.copy(order="F")
    oracle_lib.fmm(tables(p.algebra), "abc", A, B, want)
    assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL
    # the padding around C is untouched
    assert bool(torch.isnan(bC[:7]).all()) and bool(torch.isnan(bC[7 + m:]).all())


def test_gpu_rejects_bad_operands():
    p = plan_for(["222"], [1])
    A = torch.zeros(8, 8, dtype=torch.float64, device=DEV)  # row-major (stride(0) != 1)
    with pytest.raises(rt.FmmError):
        rt.fmm_gemm(p, A, rt.colmajor(8, 8, device=DEV), rt.colmajor(8, 8, device=DEV))
    with pytest.raises(rt.FmmError):
        rt.fmm_gemm(p, rt.colmajor(8, 4, device=DEV), rt.colmajor(5, 8, device=DEV), rt.colmajor(8, 8, device=DEV))
    with pytest.raises(rt.FmmError):
        rt.fmm_gemm(p, rt.colmajor(8, 8, dtype=torch.float32, device=DEV), rt.colmajor(8, 8, device=DEV),
                    rt.colmajor(8, 8, device=DEV))


def test_gpu_deterministic_and_stream_ordered():
    p = plan_for(["222", "333"], [1, 1])
    m, n, k = 700, 650, 600
    A, B, C = inputs(5, m, n, k)
    s = torch.cuda.Stream()
    outs = []
    for _ in range(2):
        with torch.cuda.stream(s):
            dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
            rt.fmm_gemm(p, dA, dB, dC, "abc")
        s.synchronize()
        outs.append(dC.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_gpu_host_dropin_symbols(oracle_lib):
    """The reference-signature host entry points (bl_dgemm_strassen_*, bl_dgemm)."""
    lib = rt.load_library()
    p = plan_for(["222"], [1])
    p.bind_default()
    m, n, k = 301, 157, 203
    for pack in ("abc", "ab", "naive"):
        A, B, C = inputs(31, m, n, k)
        got = C.copy(order="F")
        fn = getattr(lib, f"bl_dgemm_strassen_{pack}")
        fn(m, n, k, A.ctypes.data, m, B.ctypes.data, k, got.ctypes.data, m)
        assert lib.fmm_last_error() == 0
        want = C.copy(order="F")
        oracle_lib.fmm(tables(p.algebra), pack, A, B, want)
        assert rel_fro(got, want) <= RTOL_SMALL
    A, B, C = inputs(32, m, n, k)
    got = C.copy(order="F")
    lib.bl_dgemm(m, n, k, A.ctypes.data, m, B.ctypes.data, k, got.ctypes.data, m)
    want = C.copy(order="F")
    oracle_lib.bl_dgemm(A, B, want)
    assert rel_fro(got, want) <= RTOL_SMALL
    # host peeling entry point: fringes only
    A, B, C = inputs(33, m, n, k)
    got = C.copy(order="F")
    lib.bl_dynamic_peeling(m, n, k, A.ctypes.data, m, B.ctypes.data, k, got.ctypes.data, m, 16, 2, 8)
    want = C.copy(order="F")
    oracle_lib.load().oracle_dynamic_peeling(m, n, k, A.ctypes.data, m, B.ctypes.data, k, want.ctypes.data, m,
                                             16, 2, 8)
    assert rel_fro(got, want) <= RTOL_SMALL


def test_gpu_host_column_panels():
    """Host calls large enough to run as column panels (copies in and out overlapping the
    compute) match the classical product within rounding, for every pack type and the
    plain kernel; leading dimensions above the row count are honoured and the rows
    between m and ldc are left untouched."""
    p = plan_for(["222"], [1])
    m, n, k = 1030, 4610, 270  # m * n >= 2^22 and n >= 2 * 2048: two panels
    rng = np.random.default_rng(7)
    Abig = np.asfortranarray(rng.uniform(-1, 1, (m + 2, k)))
    Bbig = np.asfortranarray(rng.uniform(-1, 1, (k + 1, n)))
    Cbig = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)))
    A, B = Abig[:m], Bbig[:k]
    want = Cbig[:m] + A @ B
    for pack in ("abc", "ab", "naive", None):
        got = Cbig.copy(order="F")
        if pack is None:
            rt.bl_dgemm_host(A, B, got[:m])
        else:
            rt.fmm_gemm_host(p, A, B, got[:m], pack)
        assert rel_fro(got[:m], want) <= RTOL_SMALL, pack
        assert np.array_equal(got[m:], Cbig[m:]), pack


FULL = [
    (["222"], [1], (2048, 2048, 2048), "abc"),
    (["222", "333"], [1, 1], (14400, 14400, 480), "abc"),
    (["222", "333"], [1, 1], (4000, 16000, 2000), "abc"),
    (["222", "333"], [1, 1], (16384, 16384, 16384), "abc"),
    (["222"], [1], (16384, 16384, 16384), "abc"),
]


@pytest.mark.parametrize("algs,levels,shape,pack", FULL, ids=lambda x: str(x))
def test_gpu_full_size_within_error_bound(algs, levels, shape, pack):
    """Full benchmark sizes: error against an independent classical FP64 GEMM is within
    the FMM bound, and the FMM is linear in C (C0 + A*B with C0 = 0 vs C0 = U(-1,1))."""
    m, n, k = shape
    g = torch.Generator(device=DEV).manual_seed(1234)
    A = rt.colmajor(m, k, device=DEV)
    B = rt.colmajor(k, n, device=DEV)
    A.uniform_(-1, 1, generator=g)
    B.uniform_(-1, 1, generator=g)
    C0 = rt.colmajor(m, n, device=DEV).uniform_(-1, 1, generator=g)
    ref = torch.addmm(C0, A, B)  # cuBLAS DGEMM, the classical FP64 oracle at this size
    p = plan_for(algs, levels)
    C = C0.clone(memory_format=torch.preserve_format)
    C = rt.colmajor(m, n, device=DEV).copy_(C0)
    rt.fmm_gemm(p, A, B, C, pack)
    err = (C - ref).abs().max().item()
    bound = algebra.error_bound(p.algebra, m, n, k, 1.0, 1.0, 1.0)
    assert err <= bound
    relf = ((C - ref).norm() / ref.norm()).item()
    assert relf < 1e-12
    D = rt.colmajor(m, n, device=DEV).copy_(C0)
    rt.plain_gemm(A, B, D)
    assert (D - ref).abs().max().item() <= algebra.error_bound(algebra.classical_plan(), m, n, k, 1, 1, 1)
    del A, B, C, D, ref, C0
    torch.cuda.empty_cache()


def test_gpu_torch_custom_op(oracle_lib):
    """torch.ops.fmm.gemm / fmm.plain_gemm mutate C in place, stream-ordered."""
    from fmm_gen_b200 import ops  # noqa: F401  (registers the ops)

    m, n, k = 300, 260, 220
    A, B, C = inputs(41, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    torch.ops.fmm.gemm(dA, dB, dC, "222-1_232-1", "abc")
    want = C.copy(order="F")
    oracle_lib.fmm(tables(algebra.make_plan(["222", "232"], [1, 1])), "abc", A, B, want)
    assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL
    dC2 = to_dev(C)
    torch.ops.fmm.plain_gemm(dA, dB, dC2)
    want2 = C.copy(order="F")
    oracle_lib.bl_dgemm(A, B, want2)
    assert rel_fro(dC2.cpu().numpy(), want2) <= RTOL_SMALL


@pytest.mark.parametrize("m,n,k", [(300, 200, 1), (129, 257, 5), (640, 384, 13), (1024, 1000, 1001), (77, 4100, 999)])
def test_gpu_plain_k_tail(oracle_lib, m, n, k):
    """The classical kernel with k not a multiple of its 8-deep k step: the last step reads
    the tensor copies' zero fill past the operands' last column / row (direct staging)."""
    A, B, C = inputs(m * 31 + n * 7 + k, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rt.plain_gemm(dA, dB, dC)
    got = dC.cpu().numpy()
    want = C.copy(order="F")
    oracle_lib.bl_dgemm(A, B, want)
    assert rel_fro(got, want) <= RTOL_SMALL


# Launches of few work units split every product's k range (k-split tables): the parts'
# C updates, in order under the same tickets, add up to the product.  These shapes take
# S = 4 (plain 2048^3: 256 tiles on 148 SMs), S = 8 (plain 1024 x 2048 x 4096) and S > 1
# for 222-1 (2048^3: 448 units, pre-summed operands).
KSPLIT_CASES = [
    (None, (2048, 2048, 2048)),
    (None, (1024, 2048, 4096)),
    ((["222"], [1]), (2048, 2048, 2048)),
    ((["222"], [1]), (2048, 1536, 4096)),
]


@pytest.mark.parametrize("algo,shape", KSPLIT_CASES, ids=lambda x: str(x))
def test_gpu_ksplit_matches_oracle(oracle_lib, algo, shape):
    m, n, k = shape
    A, B, C = inputs(m + 2 * n + 5 * k, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    want = C.copy(order="F")
    if algo is None:
        rt.plain_gemm(dA, dB, dC)
        oracle_lib.bl_dgemm(A, B, want)
    else:
        p = plan_for(*algo)
        rt.fmm_gemm(p, dA, dB, dC, "abc")
        oracle_lib.fmm(tables(p.algebra), "abc", A, B, want)
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL


# The last tile row of a block with at most 64 rows runs as a half-height unit in the direct
# variant (a 64-row A box; both rows of consumer warps on those rows, half of the columns each):
# plain 1050 x 700 x 512 (26-row edge), plain 64 x 300 x 256 (one 64-row tile row), 222-1 at
# 2100 x 1800 x 1200 (pre-summed, ms = 1048: 24-row edge), 222-1 x 333-1 at 3312 x 2000 x 960
# (pre-summed, ms = 552: 40-row edge, as at 16384^3).
HALF_CASES = [
    (None, (1050, 700, 512)),
    (None, (64, 300, 256)),
    ((["222"], [1]), (2100, 1800, 1200)),
    ((["222", "333"], [1, 1]), (3312, 2000, 960)),
]


@pytest.mark.parametrize("algo,shape", HALF_CASES, ids=lambda x: str(x))
def test_gpu_half_height_edge_tiles(oracle_lib, algo, shape):
    m, n, k = shape
    A, B, C = inputs(3 * m + n + k, m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    want = C.copy(order="F")
    if algo is None:
        rt.plain_gemm(dA, dB, dC)
        oracle_lib.bl_dgemm(A, B, want)
    else:
        p = plan_for(*algo)
        rt.fmm_gemm(p, dA, dB, dC, "abc")
        oracle_lib.fmm(tables(p.algebra), "abc", A, B, want)
    torch.cuda.synchronize()
    assert rt.load_library().fmm_device_status(1) == 0
    assert rel_fro(dC.cpu().numpy(), want) <= RTOL_SMALL


# A call whose pre-summed workspace would exceed the workspace limit runs its products in
# groups (sums of the next group formed on a second stream while a group runs).  Small
# limits force 2..7 groups here; results match the oracle and the ungrouped call.
@pytest.mark.parametrize("algs,levels,shape,limit", [
    (["222"], [1], (2048, 2048, 1024), 16 << 20),         # one product per group (2 x 8 MB)
    (["222"], [1], (2048, 2048, 1024), 32 << 20),         # groups of 2 (last group smaller)
    (["222", "333"], [1, 1], (2400, 2400, 1000), 40 << 20),  # k per product 166: padded slots
])
def test_gpu_presum_groups_match_oracle(oracle_lib, algs, levels, shape, limit):
    m, n, k = shape
    A, B, C = inputs(m + n + k + limit % 997, m, n, k)
    p = plan_for(algs, levels)
    dA, dB = to_dev(A), to_dev(B)
    whole = to_dev(C)
    rt.fmm_gemm(p, dA, dB, whole, "abc")
    torch.cuda.synchronize()
    full = rt.last_workspace_bytes()
    assert full > limit
    prev = rt.set_workspace_limit(limit)
    try:
        dC = to_dev(C)
        rt.fmm_gemm(p, dA, dB, dC, "abc")
        torch.cuda.synchronize()
        assert 0 < rt.last_workspace_bytes() <= limit
    finally:
        rt.set_workspace_limit(prev)
    assert rt.load_library().fmm_device_status(1) == 0
    want = C.copy(order="F")
    oracle_lib.fmm(tables(p.algebra), "abc", A, B, want)
    got = dC.cpu().numpy()
    assert rel_fro(got, want) <= RTOL_SMALL
    assert rel_fro(got, whole.cpu().numpy()) <= RTOL_SMALL


def test_gpu_host_row_and_column_panels():
    """A host call whose A is large enough for two row panels (C[I, J] += A[I, :] * B[:, J]
    per block, half of A copied before the first kernel) matches the classical product within
    rounding through the FMM and the plain kernel; the rows between m and ldc stay untouched."""
    p = plan_for(["222"], [1])
    m, n, k = 8200, 4610, 8192  # m * k >= 2^26: two row panels; n >= 2 * 2048: two column panels
    rng = np.random.default_rng(8)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    Cbig = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)))
    want = Cbig[:m] + A @ B
    for pack in ("abc", None):
        got = Cbig.copy(order="F")
        if pack is None:
            rt.bl_dgemm_host(A, B, got[:m])
        else:
            rt.fmm_gemm_host(p, A, B, got[:m], pack)
        assert rel_fro(got[:m], want) <= RTOL_SMALL, pack
        assert np.array_equal(got[m:], Cbig[m:]), pack
