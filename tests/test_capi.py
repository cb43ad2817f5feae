"""The C-ABI library loads and exports every symbol include/fmm_b200.h declares; plan
tables are validated on the host.  No GPU needed (no compute calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from fmm_gen_b200 import algebra, build, runtime

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fmm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return runtime.load_library()


def test_header_declares_the_reference_symbols():
    names = declared_functions()
    for ref in ("bl_dgemm", "bl_dgemm_strassen_abc", "bl_dgemm_strassen_ab", "bl_dgemm_strassen_naive",
                "bl_dynamic_peeling"):
        assert ref in names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", runtime.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)  # resolvable through ctypes


def test_plan_roundtrip_and_validation(lib):
    plan = algebra.make_plan(["222", "333"], [1, 1])
    p = runtime.Plan(plan)
    assert lib.fmm_plan_rank(p.handle) == 161 == p.rank
    p.bind_default()
    assert lib.fmm_default_plan() == p.handle.value
    p.close()
    assert lib.fmm_default_plan() is None
    dims, nterms, rows, cols, coefs = runtime.plan_tables(algebra.make_plan(["222"], [1]))
    bad = rows.copy()
    bad[0] = 5  # outside the 2x2 block grid
    h = ctypes.c_void_p()
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    rc = lib.fmm_plan_create(ip(dims), 7, ip(nterms), ip(bad), ip(cols),
                             coefs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(h))
    assert rc == -5
    zero = nterms.copy()
    zero[1] = 0
    rc = lib.fmm_plan_create(ip(dims), 7, ip(zero), ip(rows), ip(cols),
                             coefs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(h))
    assert rc == -5


def test_error_strings_and_argument_checks(lib):
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert lib.fmm_error_string(code)
    # invalid leading dimension is rejected before any device work
    rc = lib.fmm_plain_dgemm_dev(4, 4, 4, 1, 2, 1, 4, 1, 4, None)
    assert rc == -1
    rc = lib.fmm_dgemm_dev(None, 0, 4, 4, 4, 1, 4, 1, 4, 1, 4, None)
    assert rc == -2
    # zero-size problems are a no-op (no device work)
    assert lib.fmm_plain_dgemm_dev(0, 4, 4, None, 1, None, 1, None, 1, None) == 0
    lib.bl_dgemm(2, 2, 2, None, 1, None, 2, None, 2)  # lda < m
    assert lib.fmm_last_error() == -1
    lib.bl_dgemm_strassen_abc(0, 3, 3, None, 1, None, 1, None, 1)  # zero-size early return
    assert lib.fmm_last_error() == 0


def test_python_layer_fails_loudly_without_library(tmp_path, monkeypatch):
    monkeypatch.setattr(runtime, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(runtime, "_lib", None)
    with pytest.raises(runtime.FmmError):
        runtime.load_library()


@pytest.mark.parametrize("algs,levels,groups,entries", [
    (["222", "333"], [1, 1], 5, 299),  # greedy grouping of the 36 C blocks (nnz(W) = 540)
    (["222"], [2], 2, 81),              # 16 blocks, nnz(W) = 144
    (["222"], [1], 1, 7),
])
def test_combine_tables_group_blocks_that_share_products(lib, algs, levels, groups, entries):
    """The combine pass's grouped tables pass their own checks (else the scatter would run)
    and merge each group's products: fewer M loads per position than nnz(W)."""
    p = runtime.Plan(algebra.make_plan(algs, levels))
    g, e, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.fmm_plan_combine_info(p.handle, ctypes.byref(g), ctypes.byref(e), ctypes.byref(c)) == 0
    assert (g.value, e.value) == (groups, entries)
    assert c.value >= (entries + 7) // 8 and c.value <= entries // 8 + groups
    p.close()
