"""ctypes binding of the fmm_b200 C ABI (include/fmm_b200.h).

The compiled library is built in-tree (fmm_gen_b200/lib/libfmm_b200.so) by
`python -m fmm_gen_b200.build` or `__graft_entry__.build()`.  There is no CPU
fallback: every entry point here raises FmmError when the library is missing.

Matrices are column-major, as in the reference (common/include/bl_dgemm.h:54-56):
a torch tensor of shape (m, k) with stride (1, lda), or a numpy array in Fortran
order.  `colmajor(m, n)` makes one.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional

import numpy as np

from . import algebra

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.environ.get("FMM_B200_LIB") or os.path.join(LIB_DIR, "libfmm_b200.so")

PACK_TYPES = {"abc": 0, "ab": 1, "naive": 2}

FMM_OK = 0
_ERRORS = {
    -1: "invalid argument",
    -2: "no plan bound",
    -3: "CUDA runtime error",
    -4: "out of memory",
    -5: "malformed plan",
    -6: "unsupported",
    -7: "device-side wait timed out",
}


class FmmError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: fmm error {code} ({_ERRORS.get(code, 'unknown')})")


_lib = None
_lib_lock = threading.Lock()


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Load libfmm_b200.so (once).  Raises FmmError if it is not built."""
    global _lib
    with _lib_lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise FmmError(-6, f"{p} is not built (run fmm_gen_b200.build)")
        lib = ctypes.CDLL(p, mode=ctypes.RTLD_GLOBAL)
        _declare(lib)
        if path is None:
            _lib = lib
        return lib


def _declare(lib: ctypes.CDLL) -> None:
    c_int, c_long, c_void_p, c_double_p = ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    c_int_p = ctypes.POINTER(ctypes.c_int)
    lib.fmm_plan_create.argtypes = [c_int_p, c_int, c_int_p, c_int_p, c_int_p, c_double_p, ctypes.POINTER(c_void_p)]
    lib.fmm_plan_create.restype = c_int
    lib.fmm_plan_destroy.argtypes = [c_void_p]
    lib.fmm_plan_destroy.restype = c_int
    lib.fmm_plan_rank.argtypes = [c_void_p]
    lib.fmm_plan_rank.restype = c_int
    lib.fmm_plan_combine_info.argtypes = [c_void_p, c_int_p, c_int_p, c_int_p]
    lib.fmm_plan_combine_info.restype = c_int
    lib.fmm_bind_default_plan.argtypes = [c_void_p]
    lib.fmm_bind_default_plan.restype = c_int
    lib.fmm_default_plan.argtypes = []
    lib.fmm_default_plan.restype = c_void_p
    lib.fmm_dgemm_dev.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_long, c_void_p, c_long,
                                  c_void_p, c_long, c_void_p]
    lib.fmm_dgemm_dev.restype = c_int
    lib.fmm_plain_dgemm_dev.argtypes = [c_int, c_int, c_int, c_void_p, c_long, c_void_p, c_long, c_void_p, c_long,
                                        c_void_p]
    lib.fmm_plain_dgemm_dev.restype = c_int
    lib.fmm_dgemm_host.argtypes = [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int,
                                   c_void_p, c_int]
    lib.fmm_dgemm_host.restype = c_int
    lib.fmm_split_gemm_dev.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p, c_long, c_void_p, c_long, c_void_p,
                                       c_long, c_void_p]
    lib.fmm_split_gemm_dev.restype = c_int
    lib.fmm_batch_create.argtypes = [c_int, ctypes.POINTER(c_void_p), c_int_p, c_int_p, c_int_p, ctypes.POINTER(c_void_p)]
    lib.fmm_batch_create.restype = c_int
    lib.fmm_batch_create_tiled.argtypes = [c_int, ctypes.POINTER(c_void_p), c_int_p, c_int_p, c_int_p, c_int_p,
                                           ctypes.POINTER(c_void_p)]
    lib.fmm_batch_create_tiled.restype = c_int
    lib.fmm_batch_dgemm.argtypes = [c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_long), ctypes.POINTER(c_void_p),
                                    ctypes.POINTER(c_long), ctypes.POINTER(c_void_p), ctypes.POINTER(c_long), c_void_p]
    lib.fmm_batch_dgemm.restype = c_int
    lib.fmm_batch_units.argtypes = [c_void_p, c_int]
    lib.fmm_batch_units.restype = c_int
    lib.fmm_batch_destroy.argtypes = [c_void_p]
    lib.fmm_batch_destroy.restype = c_int
    lib.fmm_batch_submit.argtypes = [c_int, ctypes.POINTER(c_void_p), c_int_p, c_int_p, c_int_p, ctypes.POINTER(c_void_p),
                                     ctypes.POINTER(c_long), ctypes.POINTER(c_void_p), ctypes.POINTER(c_long),
                                     ctypes.POINTER(c_void_p), ctypes.POINTER(c_long), c_void_p]
    lib.fmm_batch_submit.restype = c_int
    for name in ("bl_dgemm", "bl_dgemm_strassen_abc", "bl_dgemm_strassen_ab", "bl_dgemm_strassen_naive"):
        f = getattr(lib, name)
        f.argtypes = [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int]
        f.restype = None
    lib.bl_dynamic_peeling.argtypes = [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
                                       c_int, c_int, c_int]
    lib.bl_dynamic_peeling.restype = None
    lib.fmm_last_error.argtypes = []
    lib.fmm_last_error.restype = c_int
    lib.fmm_error_string.argtypes = [c_int]
    lib.fmm_error_string.restype = ctypes.c_char_p
    lib.fmm_kernel_launch_count.argtypes = []
    lib.fmm_kernel_launch_count.restype = ctypes.c_longlong
    lib.fmm_profile_begin.argtypes = []
    lib.fmm_profile_begin.restype = c_int
    lib.fmm_profile_end.argtypes = [c_double_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.fmm_profile_end.restype = c_int
    lib.fmm_profile_num_kinds.argtypes = []
    lib.fmm_profile_num_kinds.restype = c_int
    lib.fmm_profile_kind_name.argtypes = [c_int]
    lib.fmm_profile_kind_name.restype = ctypes.c_char_p
    lib.fmm_device_status.argtypes = [c_int]
    lib.fmm_device_status.restype = c_int
    lib.fmm_debug_set.argtypes = [c_int, ctypes.c_longlong]
    lib.fmm_debug_set.restype = c_int
    lib.fmm_set_workspace_limit.argtypes = [ctypes.c_longlong]
    lib.fmm_set_workspace_limit.restype = ctypes.c_longlong
    lib.fmm_last_workspace_bytes.argtypes = []
    lib.fmm_last_workspace_bytes.restype = ctypes.c_longlong


def _check(rc: int, what: str) -> None:
    if rc != FMM_OK:
        raise FmmError(rc, what)


def plan_tables(plan: algebra.FMMPlan):
    """Flatten a composed plan into the C ABI's term arrays."""
    nterms, rows, cols, coefs = [], [], [], []
    for p in plan.products:
        nterms.extend([len(p.a), len(p.b), len(p.c)])
        for side in (p.a, p.b, p.c):
            for t in side:
                rows.append(t.row)
                cols.append(t.col)
                coefs.append(t.coef)
    return (np.asarray(plan.dims, dtype=np.int32), np.asarray(nterms, dtype=np.int32),
            np.asarray(rows, dtype=np.int32), np.asarray(cols, dtype=np.int32), np.asarray(coefs, dtype=np.float64))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Plan:
    """Device-side FMM plan (owns a fmm_plan*)."""

    def __init__(self, plan: algebra.FMMPlan):
        self.algebra = plan
        self._lib = load_library()
        dims, nterms, rows, cols, coefs = plan_tables(plan)
        self._keep = (dims, nterms, rows, cols, coefs)
        h = ctypes.c_void_p()
        rc = self._lib.fmm_plan_create(_iptr(dims), plan.rank, _iptr(nterms), _iptr(rows), _iptr(cols),
                                       coefs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(h))
        _check(rc, "fmm_plan_create")
        self.handle = h

    @classmethod
    def from_levels(cls, algs, levels, x: Optional[float] = None) -> "Plan":
        """The composed plan of e.g. (['222', '333'], [1, 1]); `x` is the value of the
        approximate algorithms' parameter (alg_dic's *_approx entries)."""
        return cls(algebra.make_plan(algs, levels, x=x))

    @property
    def rank(self) -> int:
        """Number of products R."""
        return self.algebra.rank

    def bind_default(self) -> None:
        _check(self._lib.fmm_bind_default_plan(self.handle), "fmm_bind_default_plan")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.fmm_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------------
# torch (device) entry points
# --------------------------------------------------------------------------------
def colmajor(m: int, n: int, *, dtype=None, device=None):
    """Column-major (m, n) torch tensor with ld = m."""
    import torch

    return torch.empty((n, m), dtype=dtype or torch.float64, device=device).t()


def _ld(t, rows: int) -> int:
    if t.dim() != 2:
        raise FmmError(-1, "expected a 2-D tensor")
    if t.shape[1] > 1 and t.stride(0) != 1:
        raise FmmError(-1, "matrices must be column-major (stride(0) == 1)")
    return max(t.stride(1), rows, 1) if t.shape[1] > 1 else max(rows, 1)


def _check_operands(A, B, C, ab_dtype=None):
    import torch

    for name, t in (("A", A), ("B", B), ("C", C)):
        want = torch.float64 if (name == "C" or ab_dtype is None) else ab_dtype
        if t.dtype != want:
            raise FmmError(-1, f"{name} must be {str(want).replace('torch.', '')}")
        if not t.is_cuda:
            raise FmmError(-1, f"{name} must be a CUDA tensor")
    m, k = A.shape
    k2, n = B.shape
    if k2 != k or tuple(C.shape) != (m, n):
        raise FmmError(-1, f"shape mismatch A{tuple(A.shape)} B{tuple(B.shape)} C{tuple(C.shape)}")
    return m, n, k


def fmm_gemm(plan: Plan, A, B, C, pack: str = "abc", stream=None) -> None:
    """C += A @ B with the FMM plan, stream-ordered on the current CUDA stream."""
    import torch

    m, n, k = _check_operands(A, B, C)
    lib = load_library()
    s = stream if stream is not None else torch.cuda.current_stream(C.device)
    rc = lib.fmm_dgemm_dev(plan.handle, PACK_TYPES[pack], m, n, k, A.data_ptr(), _ld(A, m), B.data_ptr(),
                           _ld(B, k), C.data_ptr(), _ld(C, m), ctypes.c_void_p(s.cuda_stream))
    _check(rc, "fmm_dgemm_dev")


def plain_gemm(A, B, C, stream=None) -> None:
    """Classical C += A @ B (the comparator), stream-ordered."""
    import torch

    m, n, k = _check_operands(A, B, C)
    lib = load_library()
    s = stream if stream is not None else torch.cuda.current_stream(C.device)
    rc = lib.fmm_plain_dgemm_dev(m, n, k, A.data_ptr(), _ld(A, m), B.data_ptr(), _ld(B, k), C.data_ptr(),
                                 _ld(C, m), ctypes.c_void_p(s.cuda_stream))
    _check(rc, "fmm_plain_dgemm_dev")


def split_gemm(plan, A, B, C, stream=None) -> None:
    """C += A @ B on the tensor cores at FP32-level accuracy: float32 A and B, float64 C.

    plan=None runs the classical product; otherwise the FMM plan's products, each as six
    bf16 plane products with FP64 accumulation across 128-deep k chunks."""
    import torch

    m, n, k = _check_operands(A, B, C, ab_dtype=torch.float32)
    lib = load_library()
    s = stream if stream is not None else torch.cuda.current_stream(C.device)
    rc = lib.fmm_split_gemm_dev(plan.handle if plan is not None else None, m, n, k, A.data_ptr(), _ld(A, m),
                                B.data_ptr(), _ld(B, k), C.data_ptr(), _ld(C, m), ctypes.c_void_p(s.cuda_stream))
    _check(rc, "fmm_split_gemm_dev")


class Batch:
    """Many independent FP64 problems C_i += A_i @ B_i in one persistent launch.

    `shapes` is a list of (m, n, k); `plans[i]` is a Plan or None (classical).  Creating a
    batch fixes the shapes and plans, splits every problem into its FMM core and fringe
    strips (the same partition as fmm_gemm), orders the work units longest first and
    allocates the job tables, tickets and pre-summed operand workspaces once.  `run`
    then takes this call's operands (column-major float64 CUDA tensors) and enqueues
    the launch on the current stream; it can be captured in a CUDA graph (the graph
    replays with the operand pointers of the captured call).  `tiles[i]` is problem i's
    tile height, 128 (default) or 64 rows (fmm_batch_create_tiled)."""

    def __init__(self, shapes, plans=None, tiles=None):
        self._lib = load_library()
        shapes = [tuple(int(v) for v in s) for s in shapes]
        if not shapes:
            raise FmmError(-1, "empty batch")
        count = len(shapes)
        plans = list(plans) if plans is not None else [None] * count
        if len(plans) != count:
            raise FmmError(-1, "plans and shapes differ in length")
        self.shapes, self.plans = shapes, plans
        self.tiles = [int(t) for t in tiles] if tiles is not None else None
        if self.tiles is not None and len(self.tiles) != count:
            raise FmmError(-1, "tiles and shapes differ in length")
        ci = ctypes.c_int * count
        handles = (ctypes.c_void_p * count)(*[p.handle if p is not None else None for p in plans])
        h = ctypes.c_void_p()
        dims = (ci(*[s[0] for s in shapes]), ci(*[s[1] for s in shapes]), ci(*[s[2] for s in shapes]))
        if self.tiles is None:
            _check(self._lib.fmm_batch_create(count, handles, *dims, ctypes.byref(h)), "fmm_batch_create")
        else:
            _check(self._lib.fmm_batch_create_tiled(count, handles, *dims, ci(*self.tiles), ctypes.byref(h)),
                   "fmm_batch_create_tiled")
        self.handle = h

    def units(self, phase: int = 0) -> int:
        return int(self._lib.fmm_batch_units(self.handle, phase))

    def run(self, As, Bs, Cs, stream=None) -> None:
        import torch

        count = len(self.shapes)
        if not (len(As) == len(Bs) == len(Cs) == count):
            raise FmmError(-1, "operand lists must match the batch size")
        vp, cl = ctypes.c_void_p * count, ctypes.c_long * count
        pa, pb, pc, la, lb, lc = [], [], [], [], [], []
        for (m, n, k), A, B, C in zip(self.shapes, As, Bs, Cs):
            if (tuple(A.shape), tuple(B.shape), tuple(C.shape)) != ((m, k), (k, n), (m, n)):
                raise FmmError(-1, f"operands do not match the batch shape {(m, n, k)}")
            _check_operands(A, B, C)
            pa.append(A.data_ptr()); la.append(_ld(A, m))
            pb.append(B.data_ptr()); lb.append(_ld(B, k))
            pc.append(C.data_ptr()); lc.append(_ld(C, m))
        s = stream if stream is not None else torch.cuda.current_stream()
        rc = self._lib.fmm_batch_dgemm(self.handle, vp(*pa), cl(*la), vp(*pb), cl(*lb), vp(*pc), cl(*lc),
                                       ctypes.c_void_p(s.cuda_stream))
        _check(rc, "fmm_batch_dgemm")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.fmm_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_submit(plans, As, Bs, Cs, stream=None) -> None:
    """One batch formed, run and released in a single stream-ordered call (no cudaMalloc /
    cudaFree, so it does not synchronise the device): C_i += A_i @ B_i for every i, with
    plans[i] a Plan or None (classical).  For request loops; results equal Batch.run's."""
    import torch

    count = len(As)
    if not (len(Bs) == len(Cs) == len(plans) == count) or count == 0:
        raise FmmError(-1, "plans and operand lists must have the same non-zero length")
    lib = load_library()
    ci, vp, cl = ctypes.c_int * count, ctypes.c_void_p * count, ctypes.c_long * count
    ms, ns, ks, pa, pb, pc, la, lb, lc = [], [], [], [], [], [], [], [], []
    for A, B, C in zip(As, Bs, Cs):
        m, n, k = _check_operands(A, B, C)
        ms.append(m); ns.append(n); ks.append(k)
        pa.append(A.data_ptr()); la.append(_ld(A, m))
        pb.append(B.data_ptr()); lb.append(_ld(B, k))
        pc.append(C.data_ptr()); lc.append(_ld(C, m))
    handles = vp(*[p.handle if p is not None else None for p in plans])
    s = stream if stream is not None else torch.cuda.current_stream()
    rc = lib.fmm_batch_submit(count, handles, ci(*ms), ci(*ns), ci(*ks), vp(*pa), cl(*la), vp(*pb), cl(*lb),
                              vp(*pc), cl(*lc), ctypes.c_void_p(s.cuda_stream))
    _check(rc, "fmm_batch_submit")


# --------------------------------------------------------------------------------
# host (numpy) entry points: the reference-shaped synchronous API
# --------------------------------------------------------------------------------
def _np_ld(x: np.ndarray) -> int:
    if x.dtype != np.float64:
        raise FmmError(-1, "arrays must be float64")
    if x.ndim != 2:
        raise FmmError(-1, "expected a 2-D array")
    if x.shape[1] > 1 and x.strides[0] != 8:
        raise FmmError(-1, "arrays must be column-major (Fortran order)")
    return max(x.strides[1] // 8 if x.shape[1] > 1 else x.shape[0], 1)


def fmm_gemm_host(plan: Plan, A: np.ndarray, B: np.ndarray, C: np.ndarray, pack: str = "abc") -> None:
    lib = load_library()
    m, k = A.shape
    n = B.shape[1]
    rc = lib.fmm_dgemm_host(plan.handle, PACK_TYPES[pack], m, n, k, A.ctypes.data, _np_ld(A), B.ctypes.data,
                            _np_ld(B), C.ctypes.data, _np_ld(C))
    _check(rc, "fmm_dgemm_host")


def bl_dgemm_host(A: np.ndarray, B: np.ndarray, C: np.ndarray) -> None:
    lib = load_library()
    m, k = A.shape
    n = B.shape[1]
    lib.bl_dgemm(m, n, k, A.ctypes.data, _np_ld(A), B.ctypes.data, _np_ld(B), C.ctypes.data, _np_ld(C))
    _check(lib.fmm_last_error(), "bl_dgemm")


def set_workspace_limit(nbytes: int) -> int:
    """Cap one call's pre-summed operand workspace (bytes <= 0: the default, 8 GiB); returns
    the previous cap.  Calls that would need more run their products in groups."""
    return int(load_library().fmm_set_workspace_limit(int(nbytes)))


def last_workspace_bytes() -> int:
    """Pre-summed workspace bytes of this thread's last FMM call."""
    return int(load_library().fmm_last_workspace_bytes())


def kernel_launch_count() -> int:
    return int(load_library().fmm_kernel_launch_count())


class KernelTimer:
    """Per-kernel CUDA-event timing of every library launch inside the `with` block.

    After exit, `.ms[name]` and `.count[name]` hold the summed device time and the
    number of launches per kernel kind."""

    def __enter__(self):
        self._lib = load_library()
        _check(self._lib.fmm_profile_begin(), "fmm_profile_begin")
        return self

    def __exit__(self, *exc):
        n = self._lib.fmm_profile_num_kinds()
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_longlong * n)()
        _check(self._lib.fmm_profile_end(ms, cnt), "fmm_profile_end")
        names = [self._lib.fmm_profile_kind_name(i).decode() for i in range(n)]
        self.ms = {names[i]: ms[i] for i in range(n)}
        self.count = {names[i]: int(cnt[i]) for i in range(n)}
        return False
