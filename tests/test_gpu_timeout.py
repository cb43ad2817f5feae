"""Bounded device-side waits and work-unit claims, through the C ABI.

* The timeout path: every ticket of an FMM launch is started at -1 (fmm_debug_set
  FMM_DEBUG_TICKET_FILL = 0xFF), a value no launch ever releases, with the wait limit
  lowered to 50 ms (FMM_DEBUG_WAIT_LIMIT_NS).  The launch's first ticket waits run out,
  the kernel records the timeout, stops waiting for tickets and finishes; the host reads
  FMM_E_TIMEOUT from fmm_device_status.  Nothing faults or hangs: the wait is bounded,
  and the context stays usable (a normal call afterwards matches the oracle).
* Forward progress without co-residency: work units are claimed in order from a
  launch-wide counter, so an FMM launch whose products wait on each other's tickets
  completes even while another persistent kernel holds SMs on a second stream.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from fmm_gen_b200 import build, runtime as rt  # noqa: E402
from tests.golden_util import inputs  # noqa: E402

pytestmark = pytest.mark.gpu
FMM_E_TIMEOUT = -7
FMM_DEBUG_WAIT_LIMIT_NS = 1
FMM_DEBUG_TICKET_FILL = 2
RTOL = 1e-13


@pytest.fixture(scope="module")
def lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    return rt.load_library()


def to_dev(x):
    t = rt.colmajor(x.shape[0], x.shape[1], device="cuda")
    t.copy_(torch.from_numpy(np.ascontiguousarray(x)))
    return t


def tables(plan):
    dims, nterms, rows, cols, coefs = rt.plan_tables(plan)
    return (dims, plan.rank, nterms, rows, cols, coefs)


@pytest.mark.parametrize("shape", [(1024, 1024, 1024),   # pre-summed operands, per-(tile, C block) tickets
                                   (300, 280, 260)],     # sums folded while staging, per-tile tickets
                         ids=["direct", "folded"])
def test_ticket_wait_times_out_and_the_context_stays_usable(lib, oracle_lib, shape):
    m, n, k = shape
    plan = rt.Plan.from_levels(["222"], [1])
    A, B, C = inputs(sum(shape), m, n, k)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    torch.cuda.synchronize()
    assert lib.fmm_device_status(1) == 0
    try:
        assert lib.fmm_debug_set(FMM_DEBUG_WAIT_LIMIT_NS, 50_000_000) == 0
        assert lib.fmm_debug_set(FMM_DEBUG_TICKET_FILL, 0xFF) == 0
        rt.fmm_gemm(plan, dA, dB, dC, "abc")  # every ticket wait of this launch runs out
        torch.cuda.synchronize()
        assert lib.fmm_device_status(1) == FMM_E_TIMEOUT
    finally:
        assert lib.fmm_debug_set(FMM_DEBUG_TICKET_FILL, 0) == 0
        assert lib.fmm_debug_set(FMM_DEBUG_WAIT_LIMIT_NS, 0) == 0
    assert lib.fmm_device_status(1) == 0  # cleared above
    # the context is intact: a normal call matches the oracle
    dC2 = to_dev(C)
    rt.fmm_gemm(plan, dA, dB, dC2, "abc")
    torch.cuda.synchronize()
    assert lib.fmm_device_status(1) == 0
    want = C.copy(order="F")
    oracle_lib.fmm(tables(plan.algebra), "abc", A, B, want)
    got = dC2.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= RTOL


def test_debug_set_rejects_unknown_settings(lib):
    assert lib.fmm_debug_set(99, 0) != 0
    assert lib.fmm_debug_set(FMM_DEBUG_TICKET_FILL, 256) != 0


def test_fmm_completes_beside_another_persistent_kernel(lib):
    """A split-BF16 launch (persistent, one CTA per SM) on one stream and an FMM launch whose
    products are ordered by tickets on another: both finish, no wait times out, and the FMM
    result is bit-identical to the same call run alone."""
    n = 4096
    g = torch.Generator(device="cuda").manual_seed(5)
    A32 = rt.colmajor(n, n, dtype=torch.float32, device="cuda").normal_(generator=g)
    B32 = rt.colmajor(n, n, dtype=torch.float32, device="cuda").normal_(generator=g)
    Cs = rt.colmajor(n, n, device="cuda").zero_()
    m2 = 3000
    A = rt.colmajor(m2, m2, device="cuda").uniform_(-1, 1, generator=g)
    B = rt.colmajor(m2, m2, device="cuda").uniform_(-1, 1, generator=g)
    C0 = rt.colmajor(m2, m2, device="cuda").uniform_(-1, 1, generator=g)
    plan = rt.Plan.from_levels(["222", "333"], [1, 1])
    p2 = rt.Plan.from_levels(["222"], [2])
    alone = rt.colmajor(m2, m2, device="cuda").copy_(C0)
    rt.fmm_gemm(plan, A, B, alone, "abc")
    torch.cuda.synchronize()
    mixed = rt.colmajor(m2, m2, device="cuda").copy_(C0)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    s1.wait_stream(torch.cuda.current_stream())
    s2.wait_stream(torch.cuda.current_stream())
    for _ in range(3):
        with torch.cuda.stream(s1):
            rt.split_gemm(p2, A32, B32, Cs, stream=s1)
        with torch.cuda.stream(s2):
            mixed.copy_(C0)
            rt.fmm_gemm(plan, A, B, mixed, "abc", stream=s2)
    torch.cuda.synchronize()
    assert lib.fmm_device_status(1) == 0
    assert torch.equal(mixed, alone)
