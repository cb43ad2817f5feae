"""The reference's own generated multithreaded FMM libraries (oracle/build_ref_fmm.py) against
the oracle, bit for bit, on the CPU.

These libraries are the timed CPU arm of bench.py; the oracle is the parity checker of the
CUDA path.  Both follow the reference's arithmetic, so they must agree exactly:
  * the whole 222-1 x 333-1 and 222-1 abc jobs on shapes with every fringe (the reference's
    bl_dynamic_peeling included), four OpenMP threads;
  * every 8-product sample library against the oracle restricted to the same products, on a
    shape without fringes (the sampled 16384^3 core is one).
Skipped where the libraries were not built (they need an fmm-gen checkout: FMM_REF).
"""
import os

import numpy as np
import pytest

from oracle import build_ref_fmm, cpu

PATHS = build_ref_fmm.library_paths()
pytestmark = pytest.mark.skipif(not all(os.path.exists(p) for p in [PATHS["full"], PATHS["strassen"]] + PATHS["groups"]),
                                reason="reference FMM libraries not built (FMM_REF=<checkout> python oracle/build_ref_fmm.py)")


def _tables(algs, levels):
    from fmm_gen_b200 import algebra, runtime

    plan = algebra.make_plan(algs, levels)
    dims, nterms, rows, cols, coefs = runtime.plan_tables(plan)
    return (dims, plan.rank, nterms, rows, cols, coefs)


def _inputs(seed, m, n, k):
    rng = np.random.default_rng(seed)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    C = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    return A, B, C


def _ref_and_oracle(lib, tables, shape, seed):
    m, n, k = shape
    A, B, C = _inputs(seed, m, n, k)
    got = cpu.aligned_colmajor(m, n)
    got[:] = C
    lib(A, B, got)
    want = C.copy(order="F")
    cpu.fmm(tables, "abc", A, B, want)
    return got, want


@pytest.fixture(scope="module", autouse=True)
def _threads():
    cpu.set_ref_threads(4)
    # The product library exports the reference's drop-in names and is loaded RTLD_GLOBAL;
    # the reference's libraries must keep calling their own (its fringe peeling among them).
    from fmm_gen_b200 import runtime

    if os.path.exists(runtime.LIB_PATH):
        runtime.load_library()


# shapes in non-increasing n per library: each library sizes its packing pool on its first call
@pytest.mark.parametrize("job,shapes", [
    ("full", [(101, 77, 53), (96, 48, 36), (50, 31, 13)]),
    ("strassen", [(64, 48, 40), (101, 77, 53), (17, 9, 300)]),
])
def test_whole_job_matches_oracle_bit_for_bit(job, shapes):
    lib = cpu.RefFMMLib(PATHS[job])
    tables = _tables(["222", "333"], [1, 1]) if job == "full" else _tables(["222"], [1])
    for i, shape in enumerate(shapes):
        got, want = _ref_and_oracle(lib, tables, shape, 40 + i)
        assert np.array_equal(got, want), (job, shape, float(np.abs(got - want).max()))


def test_sample_libraries_match_the_oracle_on_their_products():
    tables = _tables(["222", "333"], [1, 1])
    groups = build_ref_fmm.sample_groups(tables[1])
    assert len(groups) == len(PATHS["groups"])
    covered = set()
    for g, (grp, path) in enumerate(zip(groups, PATHS["groups"])):
        lib = cpu.RefFMMLib(path)
        got, want = _ref_and_oracle(lib, cpu.product_subset(tables, grp), (96, 48, 36), 70 + g)
        assert np.array_equal(got, want), (g, float(np.abs(got - want).max()))
        covered.update(grp)
    assert covered == set(range(tables[1]))


def test_aligned_layout_is_checked():
    lib = cpu.RefFMMLib(PATHS["strassen"])
    A, B, _ = _inputs(1, 16, 8, 8)
    C = cpu.aligned_colmajor(17, 8)[1:, :]  # base 8 bytes past a 32-byte boundary
    with pytest.raises(ValueError):
        lib(A, B, C)
