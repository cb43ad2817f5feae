"""Every pure partition of the algorithm table (the reference's alg_dic, 23 entries) and a
few two-level plans through the GPU path, with fringes on every side, against the oracle:
FP64 ABC within relative Frobenius 1e-13 (the same tolerance as the other FP64 parity
tests), and the split-BF16 path within 1e-6 (FP32 inputs against the FP64 oracle)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import importlib  # noqa: E402

from fmm_gen_b200 import build, runtime as rt  # noqa: E402

pytestmark = pytest.mark.gpu
# the package re-exports the name table as `alg_dic`; the module holds the partition list
PURE = importlib.import_module("fmm_gen_b200.alg_dic").PURE_PARTITIONS
RTOL_FP64 = 1e-13
RTOL_SPLIT = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    rt.load_library()


def shape_for(dims):
    mt, kt, nt = dims
    return (8 * mt * 5 + 3, 4 * nt * 7 + 2, kt * 19 + 1)


def run_case(oracle_lib, algs, levels, split):
    p = rt.Plan.from_levels(algs, levels)
    m, n, k = shape_for(p.algebra.dims)
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    dt = np.float32 if split else np.float64
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)).astype(dt))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)).astype(dt))
    C = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    tdt = torch.float32 if split else torch.float64
    dA = rt.colmajor(m, k, dtype=tdt, device="cuda").copy_(torch.from_numpy(A))
    dB = rt.colmajor(k, n, dtype=tdt, device="cuda").copy_(torch.from_numpy(B))
    dC = rt.colmajor(m, n, device="cuda").copy_(torch.from_numpy(C))
    want = C.copy(order="F")
    if split:
        rt.split_gemm(p, dA, dB, dC)
        oracle_lib.bl_dgemm(np.asfortranarray(A.astype(np.float64)), np.asfortranarray(B.astype(np.float64)), want)
        return float(np.linalg.norm(dC.cpu().numpy() - want) / np.linalg.norm(want - C))
    rt.fmm_gemm(p, dA, dB, dC, "abc")
    dims, nterms, rows, cols, coefs = rt.plan_tables(p.algebra)
    oracle_lib.fmm((dims, p.rank, nterms, rows, cols, coefs), "abc", A, B, want)
    return float(np.linalg.norm(dC.cpu().numpy() - want) / np.linalg.norm(want))


@pytest.mark.parametrize("name", PURE)
def test_every_partition_fp64_abc(oracle_lib, name):
    assert run_case(oracle_lib, [name], [1], split=False) <= RTOL_FP64


@pytest.mark.parametrize("name", PURE)
def test_every_partition_split_bf16(oracle_lib, name):
    assert run_case(oracle_lib, [name], [1], split=True) <= RTOL_SPLIT


@pytest.mark.parametrize("algs,levels", [(["232"], [2]), (["333"], [2]), (["222", "424"], [1, 1]),
                                         (["322", "232"], [1, 1])])
def test_two_level_plans(oracle_lib, algs, levels):
    assert run_case(oracle_lib, algs, levels, split=False) <= RTOL_FP64
    assert run_case(oracle_lib, algs, levels, split=True) <= RTOL_SPLIT


# Approximate (APA) algorithms: the coefficient files use a parameter x (the reference keeps it
# symbolic in its generated C, meta/common_util.py:56-60); Plan.from_levels takes its value.
@pytest.mark.parametrize("name", ["bini322_10_52_approx", "smirnov323_14_108_approx"])
def test_gpu_approximate_algorithm_matches_oracle(oracle_lib, name):
    p = rt.Plan.from_levels([name], [1], x=0.5)
    m, n, k = shape_for(p.algebra.dims)
    rng = np.random.default_rng(len(name) + m)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    C = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    dA = rt.colmajor(m, k, device="cuda").copy_(torch.from_numpy(A))
    dB = rt.colmajor(k, n, device="cuda").copy_(torch.from_numpy(B))
    dC = rt.colmajor(m, n, device="cuda").copy_(torch.from_numpy(C))
    rt.fmm_gemm(p, dA, dB, dC, "abc")
    want = C.copy(order="F")
    dims, nterms, rows, cols, coefs = rt.plan_tables(p.algebra)
    oracle_lib.fmm((dims, p.rank, nterms, rows, cols, coefs), "abc", A, B, want)
    assert float(np.linalg.norm(dC.cpu().numpy() - want) / np.linalg.norm(want)) <= RTOL_FP64
