"""Algebra layer vs the reference generator's own composition (golden JSON made by
tests/golden/make_golden.py from meta/common_mix.py:65-92, 184-219, 284-341)."""
import itertools
import os

import numpy as np
import pytest

from fmm_gen_b200 import algebra
from fmm_gen_b200.alg_dic import alg_dic, PURE_PARTITIONS
from tests.golden_util import CONFIGS, load_coeffs


@pytest.mark.parametrize("algs,levels", CONFIGS, ids=lambda x: str(x))
def test_composition_matches_reference(algs, levels):
    gold = load_coeffs(algs, levels)
    plan = algebra.make_plan(algs, levels)
    assert list(plan.dims) == gold["dims"]
    assert plan.rank == gold["rank"]
    assert [list(d) for d in plan.level_dims] == gold["level_dims"]
    for r, (prod, gp) in enumerate(zip(plan.products, gold["products"])):
        for side, mat in (("a", 0), ("b", 1), ("c", 2)):
            mine = getattr(prod, side)
            theirs = gp[side]
            assert [(t.row, t.col, t.coef) for t in mine] == [(g["row"], g["col"], g["coef"]) for g in theirs], (r, side)
            for g in theirs:
                assert algebra.block_name(mat, g["index"], plan.level_dims) == g["name"]
                assert algebra.actual_block_name(mat, g["index"], plan.level_dims) == g["actual"]


def _brent_ok(U, V, W, dims, level_dims=None):
    """sum_r U[a,r] V[b,r] W[c,r] = 1 exactly when the blocks a=(i,p), b=(p,j), c=(i,j)
    line up, with composed indices mapped to global block positions."""
    level_dims = level_dims or [tuple(dims)]
    T = np.einsum("ar,br,cr->abc", U, V, W)
    ga = [algebra._global_rc(a, level_dims, 0, 1) for a in range(U.shape[0])]
    gb = [algebra._global_rc(b, level_dims, 1, 2) for b in range(V.shape[0])]
    gc = [algebra._global_rc(c, level_dims, 0, 2) for c in range(W.shape[0])]
    want = np.zeros_like(T)
    for a, (i, p) in enumerate(ga):
        for b, (p2, j) in enumerate(gb):
            if p2 != p:
                continue
            want[a, b, gc.index((i, j))] = 1.0
    return np.allclose(T, want, atol=1e-12)


MALFORMED = {"grey323_15_89"}  # ignore/ entry: U, V, W have 9, 8, 9 rows; no <m,k,n> fits


@pytest.mark.parametrize("name", sorted(k for k in alg_dic if "approx" not in k and k not in MALFORMED))
def test_every_exact_algorithm_satisfies_brent_equations(name):
    alg = algebra.load_algorithm(name)
    U, V, W = alg.matrices()
    assert _brent_ok(U, V, W, alg.dims), name


@pytest.mark.parametrize("algs,levels", [(["222"], [2]), (["222", "333"], [1, 1]), (["232", "323"], [1, 1])])
def test_composed_plans_are_exact(algs, levels):
    plan = algebra.make_plan(algs, levels)
    assert _brent_ok(plan.U, plan.V, plan.W, plan.dims, plan.level_dims)


def test_malformed_table_entry_is_rejected():
    for name in MALFORMED:
        with pytest.raises(algebra.CoefficientError):
            algebra.load_algorithm(name)


def test_pure_partition_table():
    assert len(PURE_PARTITIONS) == 23
    assert alg_dic["222"][0] == "strassen" and alg_dic["333"][0] == "smirnov333-23-139"
    assert alg_dic["232"][0] == "madan232-11-48"
    for key in PURE_PARTITIONS:
        assert tuple(int(c) for c in key) == alg_dic[key][1]


def test_coefficient_grammar():
    # same C expressions the reference emits (meta/common_util.py:37-82)
    assert algebra.coeff_expr("-x2i") == "-(1.0 / (x * x))"
    assert algebra.coeff_expr("(1+-x3)") == "(1 + -(x * x * x))"
    assert algebra.coeff_expr("2x2") == "2.0 * (x * x)"
    assert algebra.coeff_expr("-.125") == "-.125"
    x = 0.1
    assert algebra.coeff_value("-x2i", x) == pytest.approx(-1.0 / (x * x))
    assert algebra.coeff_value("(x+-x4)", x) == pytest.approx(x - x ** 4)
    assert algebra.coeff_value("-2x3", x) == pytest.approx(-2 * x ** 3)
    with pytest.raises(algebra.CoefficientError):
        algebra.coeff_value("x")  # the parameter must be given
    with pytest.raises(algebra.CoefficientError):
        algebra.coeff_expr("(x")


def test_apa_algorithm_needs_parameter():
    alg = algebra.load_algorithm("bini322_10_52_approx", x=1e-4)
    U, V, W = alg.matrices()
    assert U.shape == (6, 10)
    with pytest.raises(algebra.CoefficientError):
        algebra.load_algorithm("bini322_10_52_approx").matrices()


def test_bad_files(tmp_path):
    p = tmp_path / "bad"
    p.write_text("# only\n1 0\n#\n1 0\n")
    with pytest.raises(algebra.CoefficientError):
        algebra.read_coeffs(str(p))
    q = tmp_path / "ragged"
    q.write_text("#\n1 0\n1\n#\n1 0\n0 1\n#\n1 0\n0 1\n")
    with pytest.raises(algebra.CoefficientError):
        algebra.load_algorithm(str(q), dims=(1, 2, 1))


def test_partition_matches_reference_formula():
    p = algebra.partition(16384, 16384, 16384, (6, 6, 6))
    assert (p.mr, p.kr, p.nr) == (16, 4, 16)
    assert (p.ms, p.ks, p.ns) == (2728, 2730, 2728)
    p = algebra.partition(4000, 16000, 2000, (6, 6, 6))
    assert (p.mr, p.kr, p.nr, p.ms, p.ks, p.ns) == (16, 2, 16, 664, 333, 2664)
    p = algebra.partition(14400, 14400, 480, (6, 6, 6))
    assert (p.mr, p.kr, p.nr, p.ms, p.ks, p.ns) == (0, 0, 0, 2400, 80, 2400)
    p = algebra.partition(2048, 2048, 2048, (2, 2, 2))
    assert (p.ms, p.ks, p.ns, p.mr, p.kr, p.nr) == (1024, 1024, 1024, 0, 0, 0)
    p = algebra.partition(7, 3, 1, (2, 2, 2))
    assert (p.md, p.kd, p.nd) == (0, 0, 0)


def test_plan_statistics():
    s = algebra.make_plan(["222"], [1])
    assert s.rank == 7 and s.nnz == (12, 12, 12) and s.max_terms == (2, 2, 2)
    assert algebra.e_max(s) == 12.0
    h = algebra.make_plan(["222", "333"], [1, 1])
    assert h.rank == 161 and h.nnz == (588, 540, 540) and h.max_terms == (8, 8, 8)
    assert algebra.e_max(h) == pytest.approx(12.0 * algebra.e_max(algebra.make_plan(["333"], [1])))
    assert h.job_levels == "222-1_333-1"
    assert algebra.make_plan(["222"], [2]).job_levels == "222-2"
    c = algebra.classical_plan(2, 2, 2)
    assert c.rank == 8 and _brent_ok(c.U, c.V, c.W, c.dims)


def test_error_bound_dominates_observed_error(oracle_lib):
    from fmm_gen_b200 import runtime

    plan = algebra.make_plan(["222"], [2])
    rng = np.random.default_rng(3)
    m, n, k = 64, 48, 56
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    C = np.zeros((m, n), order="F")
    dims, nterms, rows, cols, coefs = runtime.plan_tables(plan)
    oracle_lib.fmm((dims, plan.rank, nterms, rows, cols, coefs), "abc", A, B, C)
    E = np.zeros((m, n), order="F")
    oracle_lib.dgemm_dot2(A, B, E)
    err = np.abs(C - E).max()
    assert 0 < err <= algebra.error_bound(plan, m, n, k, 1.0, 1.0)
