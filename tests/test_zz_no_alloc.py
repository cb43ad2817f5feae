"""fmm_dgemm_dev_noalloc: the FMM entry point for callers that cannot allocate device memory
at call time (frameworks that own all device memory through their own allocator, and
latency-critical paths).  Its scratch lives in a static device array; the test checks it
through the C ABI against the regular entry point, fmm_dgemm_dev, on two calls in a row.

Kept in a file of its own that pytest collects last; it does not depend on state left by
other tests (it works alone in a fresh process and after the rest of the suite).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import algebra, build, runtime as rt  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-13  # same tolerance as the other GPU parity tests
FMM_E_TOO_LARGE = -8


@pytest.fixture(scope="module")
def lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    L = rt.load_library()
    f = L.fmm_dgemm_dev_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long,
                  ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_int]
    f.restype = ctypes.c_int
    return L


def _noalloc(L, plan, A, B, C, stream, sync=1):
    m, k = A.shape
    n = B.shape[1]
    return L.fmm_dgemm_dev_noalloc(plan.handle, m, n, k, A.data_ptr(), A.stride(1), B.data_ptr(), B.stride(1),
                                   C.data_ptr(), C.stride(1), ctypes.c_void_p(stream.cuda_stream), sync)


def _rand(m, n, g):
    return rt.colmajor(m, n, device="cuda").uniform_(-1, 1, generator=g)


@pytest.mark.parametrize("algs,levels,shape", [
    (["222"], [1], (1030, 1001, 777)),            # fringes on every side
    (["222", "333"], [1, 1], (1000, 900, 700)),   # tickets ordering product chunks
    (["232"], [1], (517, 389, 263)),
])
def test_noalloc_matches_regular_entry_point_twice(lib, algs, levels, shape):
    m, n, k = shape
    plan = rt.Plan.from_levels(algs, levels)
    g = torch.Generator(device="cuda").manual_seed(sum(shape))
    A, B, C0 = _rand(m, k, g), _rand(k, n, g), _rand(m, n, g)
    stream = torch.cuda.current_stream()
    got = rt.colmajor(m, n, device="cuda").copy_(C0)
    want = rt.colmajor(m, n, device="cuda").copy_(C0)
    for _ in range(2):  # two calls in a row: C += A*B twice, scratch reused
        assert _noalloc(lib, plan, A, B, got, stream) == 0
        rt.fmm_gemm(plan, A, B, want, "abc")
    torch.cuda.synchronize()
    rel = ((got - want).norm() / want.norm()).item()
    assert rel <= RTOL
    bound = algebra.error_bound(plan.algebra, m, n, k, 1.0, 1.0, 1.0)
    assert (got - want).abs().max().item() <= 4 * bound


@pytest.mark.parametrize("algs,levels,shape", [
    (["222"], [1], (15, 9, 300)),                 # fringe only: m below the plan's block multiple (md = 0)
    (["333"], [1], (300, 260, 2)),                # fringe only: k below the plan's k split (kd = 0)
    (None, None, (517, 389, 263)),                # classical 1 x 1 x 1 plan
])
def test_noalloc_fringe_only_and_classical(lib, algs, levels, shape):
    m, n, k = shape
    plan = rt.Plan(algebra.classical_plan()) if algs is None else rt.Plan.from_levels(algs, levels)
    g = torch.Generator(device="cuda").manual_seed(3 * m + n + k)
    A, B, C0 = _rand(m, k, g), _rand(k, n, g), _rand(m, n, g)
    stream = torch.cuda.current_stream()
    got = rt.colmajor(m, n, device="cuda").copy_(C0)
    want = rt.colmajor(m, n, device="cuda").copy_(C0)
    for _ in range(2):
        assert _noalloc(lib, plan, A, B, got, stream) == 0
        rt.fmm_gemm(plan, A, B, want, "abc")
    torch.cuda.synchronize()
    assert ((got - want).norm() / want.norm()).item() <= RTOL


def test_noalloc_back_to_back_without_sync(lib):
    """Two sync = 0 calls on one stream reuse the scratch before the host synchronises; one
    stream synchronisation afterwards, then the status reads clean."""
    m, n, k = 1000, 900, 700
    plan = rt.Plan.from_levels(["222", "333"], [1, 1])
    g = torch.Generator(device="cuda").manual_seed(77)
    A, B, C0 = _rand(m, k, g), _rand(k, n, g), _rand(m, n, g)
    stream = torch.cuda.current_stream()
    got = rt.colmajor(m, n, device="cuda").copy_(C0)
    want = rt.colmajor(m, n, device="cuda").copy_(C0)
    assert _noalloc(lib, plan, A, B, got, stream, sync=0) == 0
    assert _noalloc(lib, plan, A, B, got, stream, sync=0) == 0
    stream.synchronize()
    assert lib.fmm_device_status(1) == 0
    for _ in range(2):
        rt.fmm_gemm(plan, A, B, want, "abc")
    torch.cuda.synchronize()
    assert ((got - want).norm() / want.norm()).item() <= RTOL


def test_noalloc_rejects_sizes_beyond_its_limits(lib):
    plan = rt.Plan.from_levels(["222"], [1])
    m = n = 2 * 16512  # ms = ns = 16512 -> 129 x 129 = 16641 tiles
    fake = 256  # never dereferenced: the size check comes before any device work
    rc = lib.fmm_dgemm_dev_noalloc(plan.handle, m, n, 16, fake, m, fake, 16, fake, m, None, 0)
    assert rc == FMM_E_TOO_LARGE
    assert lib.fmm_error_string(rc)
