"""ORACLE — test infrastructure only.  ctypes wrapper of liboracle.so (fmm_oracle.c),
the bit-exact CPU restatement of fmm-gen's arithmetic, of the reference's own classical
runtime when it was compiled into _ref/ (Makefile target `ref`), and of the reference's
own generated FMM libraries when build_ref_fmm.py compiled them into _ref/fmm/.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libblislab_ref.so")
PACKS = {"abc": 0, "ab": 1, "naive": 2}

_lib = None
_ref = None
# The reference's libraries resolve their own symbols first: the product library is loaded
# RTLD_GLOBAL and exports the same drop-in names (bl_dgemm, bl_dynamic_peeling, ...), which
# would otherwise take the reference's internal calls (its fringe peeling among them).
_REF_MODE = ctypes.RTLD_LOCAL | getattr(os, "RTLD_DEEPBIND", 0)


def build(ref: bool = False) -> None:
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.oracle_bl_dgemm.argtypes = [ci, ci, ci, vp, ci, vp, ci, vp, ci]
        L.oracle_fmm.argtypes = [ci, vp, ci, vp, vp, vp, vp, ci, ci, ci, vp, ci, vp, ci, vp, ci]
        L.oracle_dgemm_dot2.argtypes = [ci, ci, ci, vp, ci, vp, ci, vp, ci]
        L.oracle_dynamic_peeling.argtypes = [ci, ci, ci, vp, ci, vp, ci, vp, ci, ci, ci, ci]
        L.oracle_num_threads.argtypes = []
        _lib = L
    return _lib


def load_ref():
    """The reference's classical runtime (bl_dgemm), or None when it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        L = ctypes.CDLL(REF_LIB, mode=_REF_MODE)
        L.bl_dgemm.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int] * 3
        L.bl_dgemm.restype = None
        _ref = L
    return _ref


def _cm(x: np.ndarray) -> np.ndarray:
    if x.dtype != np.float64 or not x.flags.f_contiguous:
        raise ValueError("oracle arrays must be float64 Fortran-ordered")
    return x


def _p(x):
    return x.ctypes.data_as(ctypes.c_void_p)


def bl_dgemm(A, B, C) -> None:
    """C += A @ B with the reference's per-element arithmetic (in place, Fortran arrays)."""
    m, k = A.shape
    n = B.shape[1]
    load().oracle_bl_dgemm(m, n, k, _p(_cm(A)), max(m, 1), _p(_cm(B)), max(k, 1), _p(_cm(C)), max(m, 1))


def _ld(x: np.ndarray) -> int:
    """Leading dimension of a float64 column-major array or of a column-major view of one
    (unit row stride), e.g. A[:md, :kd] of a Fortran array."""
    if x.dtype != np.float64 or x.ndim != 2 or (x.shape[0] > 1 and x.strides[0] != 8) or x.strides[1] % 8:
        raise ValueError("oracle arrays must be float64, column-major (unit row stride)")
    return max(x.strides[1] // 8, x.shape[0], 1)


def fmm(tables, pack: str, A, B, C) -> None:
    """FMM C += A @ B; `tables` = (dims, R, nterms, rows, cols, coefs) as int32/float64 arrays.
    A, B, C are Fortran arrays or column-major views of them (their leading dimensions are
    passed on)."""
    dims, R, nterms, rows, cols, coefs = tables
    m, k = A.shape
    n = B.shape[1]
    rc = load().oracle_fmm(PACKS[pack], _p(dims), int(R), _p(nterms), _p(rows), _p(cols), _p(coefs), m, n, k,
                           _p(A), _ld(A), _p(B), _ld(B), _p(C), _ld(C))
    if rc:
        raise RuntimeError(f"oracle_fmm failed: {rc}")


def dynamic_peeling(A, B, C, d1: int, d2: int, d3: int) -> None:
    """The fringe strips of an FMM call (the reference's bl_dynamic_peeling), in place."""
    m, k = A.shape
    n = B.shape[1]
    load().oracle_dynamic_peeling(m, n, k, _p(A), _ld(A), _p(B), _ld(B), _p(C), _ld(C), d1, d2, d3)


def product_subset(tables, prods):
    """Plan tables restricted to the products `prods` (in that order): used to time a sample
    of a large call's products."""
    dims, R, nterms, rows, cols, coefs = tables
    nt = np.asarray(nterms, dtype=np.int32).reshape(R, 3)
    starts = np.concatenate([[0], np.cumsum(nt.sum(axis=1))])
    sel = np.concatenate([np.arange(starts[r], starts[r + 1]) for r in prods])
    return (dims, len(prods), np.ascontiguousarray(nt[list(prods)].reshape(-1)),
            np.ascontiguousarray(rows[sel], dtype=np.int32), np.ascontiguousarray(cols[sel], dtype=np.int32),
            np.ascontiguousarray(coefs[sel], dtype=np.float64))


def dgemm_dot2(A, B, C) -> None:
    """C += A @ B with compensated (Dot2) dot products: the accuracy reference."""
    m, k = A.shape
    n = B.shape[1]
    load().oracle_dgemm_dot2(m, n, k, _p(_cm(A)), max(m, 1), _p(_cm(B)), max(k, 1), _p(_cm(C)), max(m, 1))


def ref_bl_dgemm(A, B, C) -> bool:
    """The reference's own bl_dgemm (needs a padded, 32 B aligned C; done here).  False if absent."""
    L = load_ref()
    if L is None:
        return False
    m, k = A.shape
    n = B.shape[1]
    ldc = ((m - 1) // 8 + 1) * 8
    buf = np.zeros(ldc * (n + 4) + 8)
    off = (-buf.ctypes.data % 32) // 8
    flat = buf[off:off + ldc * (n + 4)]
    Cv = flat[: ldc * n].reshape(n, ldc).T
    Cv[:m, :] = C
    L.bl_dgemm(m, n, k, _p(_cm(A)), m, _p(_cm(B)), k, flat.ctypes.data_as(ctypes.c_void_p), ldc)
    C[:, :] = Cv[:m, :n]
    return True


def num_threads() -> int:
    return int(load().oracle_num_threads())


# ---------------------------------------------------------------------------------------
# The reference's generated multithreaded FMM libraries (built by build_ref_fmm.py)
# ---------------------------------------------------------------------------------------
_ref_threads = None


def aligned_colmajor(m: int, n: int, ld_multiple: int = 8) -> np.ndarray:
    """A zeroed m x n column-major view laid out as the reference's driver allocates C
    (meta/misc_gen.py test driver: ldc = ceil(m/8)*8, n+4 columns, 32-byte aligned base);
    the generated micro-kernels store C with aligned AVX moves."""
    ld = max(((m - 1) // ld_multiple + 1) * ld_multiple, ld_multiple)
    buf = np.zeros(ld * (n + 4) + 8)
    off = (-buf.ctypes.data % 32) // 8
    flat = buf[off:off + ld * (n + 4)]
    return flat[: ld * n].reshape(n, ld).T[:m, :]


def set_ref_threads(nt: int) -> None:
    """Threads of the reference libraries (their BLISLAB_IC_NT).  Fixed once per process:
    each library sizes its packing pool on its first call (bl_malloc_packing_pool,
    common/dgemm/bl_dgemm_util.c:375-394)."""
    global _ref_threads
    if _ref_threads is not None and _ref_threads != nt:
        raise RuntimeError("the reference libraries' thread count is fixed once per process")
    _ref_threads = nt
    os.environ["BLISLAB_IC_NT"] = str(nt)


class RefFMMLib:
    """One generated reference library: bl_dgemm_strassen_abc(m, n, k, A, lda, B, ldb, C, ldc),
    C += A*B with the reference's packing, AVX micro-kernels and fringe peeling."""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = ctypes.CDLL(path, mode=_REF_MODE)
        f = self.lib.bl_dgemm_strassen_abc
        f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int] * 3
        f.restype = None
        self.fn = f

    def __call__(self, A, B, C) -> None:
        if _ref_threads is None:
            raise RuntimeError("call set_ref_threads() first")
        m, k = A.shape
        n = B.shape[1]
        if C.shape != (m, n) or B.shape[0] != k:
            raise ValueError("shape mismatch")
        ldc = _ld(C)
        if C.ctypes.data % 32 or ldc % 8:
            raise ValueError("C must be 32-byte aligned with a leading dimension that is a multiple of 8 "
                             "(aligned_colmajor)")
        if m == 0 or n == 0 or k == 0:
            return
        self.fn(m, n, k, _p(A), _ld(A), _p(B), _ld(B), _p(C), ldc)


def ref_fmm_dir() -> str:
    return os.path.join(HERE, "_ref", "fmm")
