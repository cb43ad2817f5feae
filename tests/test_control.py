"""Generator CLI contract (meta/control.py:42-141): argument parsing, job naming, the
emitted job library and test driver."""
import json
import os
import subprocess

import pytest

from fmm_gen_b200 import algebra, build, control


def test_parse_argv_like_reference():
    assert control.parse_argv(["1", "222", "1"]) == (["222"], [1], "abc", "../")
    assert control.parse_argv(["2", "222", "1", "333", "1", "ab", "/x"]) == (["222", "333"], [1, 1], "ab", "/x")
    assert control.parse_argv(["1", "222", "2", "naive"])[2] == "naive"
    with pytest.raises(SystemExit):
        control.parse_argv(["2", "222", "1"])
    with pytest.raises(SystemExit):
        control.parse_argv(["1", "222", "1", "abcd"])
    with pytest.raises(SystemExit):
        control.parse_argv(["1", "nope", "1"])


def test_job_names():
    assert control.job_name(["222"], [1], "abc") == "222-1_abc"
    assert control.job_name(["222", "333"], [1, 1], "abc") == "222-1_333-1_abc"
    assert control.job_name(["222"], [2], "naive") == "222-2_naive"


@pytest.mark.parametrize("pack", ["abc", "ab", "naive"])
def test_generate_job(tmp_path, pack):
    build.build()
    d = control.generate_code(["222", "333"], [1, 1], pack, str(tmp_path))
    job = f"222-1_333-1_{pack}"
    assert os.path.basename(d) == job
    plan = json.load(open(os.path.join(d, "plan.json")))
    ref = algebra.make_plan(["222", "333"], [1, 1])
    assert plan["rank"] == ref.rank == 161
    assert plan["products"][5]["a"] == [[t.row, t.col, t.coef] for t in ref.products[5].a]
    lib = os.path.join(d, "lib", f"lib{job}.so")
    syms = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    assert f"bl_dgemm_strassen_{pack}" in syms
    assert os.path.exists(os.path.join(d, "test", f"test_{job}_mt.x"))
    assert os.path.islink(os.path.join(d, "test", f"test_{job}_st.x"))


def test_job_library_binds_its_plan_on_load(tmp_path):
    """Loading the job library creates its plan and binds it as the default (host only)."""
    import ctypes

    from fmm_gen_b200 import runtime

    build.build()
    d = control.generate_code(["232"], [1], "abc", str(tmp_path))
    L = runtime.load_library()
    job = ctypes.CDLL(os.path.join(d, "lib", "lib232-1_abc.so"))
    job.fmm_job_status.restype = ctypes.c_int
    assert job.fmm_job_status() == 0
    h = L.fmm_default_plan()
    assert h and L.fmm_plan_rank(h) == 11


def test_generator_accepts_the_approximate_parameter(tmp_path):
    """An approximate algorithm's job needs a value for x (--x on the CLI); the job's
    plan.json then holds the evaluated coefficients."""
    import json

    from fmm_gen_b200 import algebra, control

    d = control.generate_code(["bini322_10_52_approx"], [1], "abc", str(tmp_path), compile_code=False, x=0.25)
    with open(os.path.join(d, "plan.json")) as fh:
        plan = json.load(fh)
    want = algebra.make_plan(["bini322_10_52_approx"], [1], x=0.25)
    assert plan["rank"] == want.rank == 10
    coefs = [abs(c[2]) for p in plan["products"] for side in ("a", "b", "c") for c in p[side]]
    assert max(coefs) == 4.0 == float(abs(want.W).max())  # 1 / x
