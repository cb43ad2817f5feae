"""ORACLE build recipe (test infrastructure only): the reference's own generated FMM library.

fmm-gen's FMM entry points are generated code: its Python generator (meta/abc_gen_mix.py,
gen_abc_fmm) writes the C for one algorithm, and the job's makefile (meta/misc_gen.py:78-145)
compiles it with the reference runtime (common/dgemm, common/kernels) and `-D_PARALLEL_` into a
multithreaded library whose `bl_dgemm_strassen_abc` runs each product's OpenMP m-range split
(bl_get_range, common/dgemm/bl_dgemm_util.c:189-280) on BLISLAB_IC_NT threads.

This recipe does the same for the timed CPU arm, from an fmm-gen checkout named by FMM_REF:
the generator is loaded in memory through the Python 3 shim of tests/golden/make_golden.py
(which also repairs the multi-destination asm operand commas), its C is emitted into a
temporary directory and compiled with the reference's gcc flags plus -D_PARALLEL_.  Outputs go
only to oracle/_ref/fmm/ (git-ignored):

  lib222-1_333-1_abc.so        the whole 161-product job
  lib222-1_333-1_abc_g<g>.so   the same job's code for products GROUP*g .. GROUP*g+GROUP-1
                               (mod 161), one library per group: the sample of a 16384^3
                               call that one CPU step times
  lib222-1_abc.so              the one-level Strassen job

Usage:  FMM_REF=<fmm-gen checkout> python oracle/build_ref_fmm.py [--jobs N]
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref", "fmm")
GROUP = 8          # products per sample library
HYBRID = (["222", "333"], [1, 1])
STRASSEN = (["222"], [1])


def _golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden",
                                                                              "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def sample_groups(rank: int, group: int = GROUP):
    """Product groups of `group` consecutive products (wrapping), covering all `rank`."""
    n = (rank + group - 1) // group
    return [[(g * group + i) % rank for i in range(group)] for g in range(n)]


def library_paths(rank: int = 161):
    """{"full": path, "strassen": path, "groups": [path per group]} of the built libraries."""
    return {"full": os.path.join(OUT, "lib222-1_333-1_abc.so"),
            "strassen": os.path.join(OUT, "lib222-1_abc.so"),
            "groups": [os.path.join(OUT, f"lib222-1_333-1_abc_g{g}.so") for g in range(len(sample_groups(rank)))]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    args = ap.parse_args()
    mg = _golden()
    if not mg.REF or not os.path.isdir(mg.META):
        sys.exit("set FMM_REF to an fmm-gen checkout (the directory that holds meta/ and common/)")
    mods = mg.load_reference()
    os.makedirs(OUT, exist_ok=True)
    paths = library_paths()
    work = tempfile.mkdtemp(prefix="fmm_ref_")
    par = ["-D_PARALLEL_"]
    jobs = [(HYBRID, None, paths["full"]), (STRASSEN, None, paths["strassen"])]
    jobs += [(HYBRID, grp, out) for grp, out in zip(sample_groups(161), paths["groups"])]
    # the generator runs serially (it swaps a module global for subsets); gcc runs in parallel
    cmds = [mg.build_job(mods, algs, levels, "abc", work, products=grp, extra_cflags=par, out=out,
                         compile_now=False) for (algs, levels), grp, out in jobs]
    with ThreadPoolExecutor(args.jobs) as ex:
        for _ in ex.map(lambda c: subprocess.run(c, check=True), cmds):
            pass
    shutil.rmtree(work, ignore_errors=True)
    print(f"{len(cmds)} reference libraries in {OUT}")


if __name__ == "__main__":
    main()
