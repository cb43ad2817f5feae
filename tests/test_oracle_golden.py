"""Pin the oracle: its results are bit-identical to outputs of the reference's own
generated code (tests/golden, made by make_golden.py)."""
import numpy as np
import pytest

from fmm_gen_b200 import algebra, runtime
from tests.golden_util import golden_cases, inputs, plain_cases

CASES = golden_cases()


def _tables(algs, levels):
    plan = algebra.make_plan(algs, levels)
    dims, nterms, rows, cols, coefs = runtime.plan_tables(plan)
    return (dims, plan.rank, nterms, rows, cols, coefs)


@pytest.mark.parametrize("case", CASES, ids=[f"{'_'.join(c[0])}-{c[2]}-{c[3]}" for c in CASES])
def test_oracle_bitwise_equals_reference(oracle_lib, case):
    algs, levels, pack, _, (m, n, k), seed, want = case
    A, B, C = inputs(seed, m, n, k)
    oracle_lib.fmm(_tables(algs, levels), pack, A, B, C)
    assert np.array_equal(C, want)


@pytest.mark.parametrize("case", plain_cases(), ids=lambda c: str(c[0]))
def test_oracle_classical_bitwise(oracle_lib, case):
    (m, n, k), seed, want = case
    A, B, C = inputs(seed, m, n, k)
    oracle_lib.bl_dgemm(A, B, C)
    assert np.array_equal(C, want)


def test_reference_runtime_build_agrees(oracle_lib):
    """The reference's own bl_dgemm compiled into oracle/_ref (when built) reproduces
    the golden vectors too."""
    if oracle_lib.load_ref() is None:
        pytest.skip("oracle/_ref not built here")
    for (m, n, k), seed, want in plain_cases():
        A, B, C = inputs(seed, m, n, k)
        assert oracle_lib.ref_bl_dgemm(A, B, C)
        assert np.array_equal(C, want)


def test_dot2_is_accurate(oracle_lib):
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.uniform(-1, 1, (5, 200)))
    B = np.asfortranarray(rng.uniform(-1, 1, (200, 3)))
    C = np.zeros((5, 3), order="F")
    oracle_lib.dgemm_dot2(A, B, C)
    import math
    for i in range(5):
        for j in range(3):
            exact = math.fsum(A[i, p] * B[p, j] for p in range(200))  # products rounded, sum exact
            assert abs(C[i, j] - exact) <= 1e-13 * max(1.0, abs(exact))


def test_pack_types_agree_bitwise_ab_naive(oracle_lib):
    """AB and NAIVE both form M_r = 0 + sum of KC-chunk products, then scatter, so the
    reference gives them identical bits; ABC differs only by rounding."""
    algs, levels = ["222", "333"], [1, 1]
    t = _tables(algs, levels)
    A, B, C = inputs(77, 100, 53, 40)
    outs = {}
    for pack in ("abc", "ab", "naive"):
        Cp = C.copy(order="F")
        oracle_lib.fmm(t, pack, A, B, Cp)
        outs[pack] = Cp
    assert np.array_equal(outs["ab"], outs["naive"])
    assert np.abs(outs["abc"] - outs["ab"]).max() < 1e-12
