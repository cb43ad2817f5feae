"""Generator CLI with the reference's contract (meta/control.py:42-141):

    python -m fmm_gen_b200.control N alg1 L1 ... algN LN [pack_type] [gen_path]

e.g. `python -m fmm_gen_b200.control 2 222 1 333 1 abc ./jobs`.  It composes the
levels (Kronecker product, outer level first), names the job
`<alg1>-<L1>_..._<pack_type>` (control.py:47) and writes `<gen_path>/<job>/`:

    plan.json                 the composed plan: per product the A, B, C terms
    dgemm/my_dgemm_<job>.c    the job library's C source: the plan as static tables,
                              bound at load time, and the entry point
                              bl_dgemm_strassen_<pack_type>(m,n,k,A,lda,B,ldb,C,ldc)
    lib/lib<job>.so           the job library (links libfmm_b200.so)
    test/test_<job>.c, test/test_<job>_{st,mt}.x
                              the test driver: `test_<job>_mt.x m n k` prints
                              `m n k GFLOPS_fmm GFLOPS_gemm` (meta/misc_gen.py:147-261)

Where the reference emits specialised C + AVX per configuration, the GPU kernels here
are generic over the plan tables; what is generated per job is the table and the thin
library that binds it.  A process that links one job library gets that job's FMM from
the reference's symbol names, as with the reference (one configuration per library).
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
from typing import List, Optional, Sequence

from . import algebra
from .alg_dic import alg_dic
from .runtime import LIB_DIR, PACK_TYPES, plan_tables

PKG = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(os.path.dirname(PKG), "include")
USAGE = "USAGE: python -m fmm_gen_b200.control N alg1 L1 ... algN LN [pack_type] [gen_path]"


def job_name(algs: Sequence[str], levels: Sequence[int], pack_type: str) -> str:
    return "_".join(f"{a}-{int(l)}" for a, l in zip(algs, levels)) + "_" + pack_type


def parse_argv(argv: List[str]):
    """Parse `N alg1 L1 ... [pack_type] [gen_path]` exactly as meta/control.py:120-141."""
    try:
        num = int(argv[0])
        algs, levels = [], []
        for i in range(num):
            algs.append(argv[1 + 2 * i])
            levels.append(int(argv[2 + 2 * i]))
        pack_type = "abc"
        gen_path = "../"
        if len(argv) > 1 + 2 * num:
            pack_type = argv[1 + 2 * num]
        if len(argv) > 2 + 2 * num:
            gen_path = argv[2 + 2 * num]
    except (IndexError, ValueError):
        raise SystemExit(USAGE)
    if num < 1:
        raise SystemExit(USAGE)
    if pack_type not in PACK_TYPES:
        raise SystemExit(f"pack_type not supported: {pack_type} (abc, ab, naive)")
    for a in algs:
        if a not in alg_dic:
            raise SystemExit(f"unknown algorithm {a!r}; see fmm_gen_b200.alg_dic")
    return algs, levels, pack_type, gen_path


def _c_array(ctype: str, name: str, vals) -> str:
    body = ", ".join(repr(float(v)) if ctype == "double" else str(int(v)) for v in vals)
    return f"static const {ctype} {name}[{max(len(vals), 1)}] = {{{body}}};\n"


def job_library_source(plan: algebra.FMMPlan, job: str, pack_type: str) -> str:
    dims, nterms, rows, cols, coefs = plan_tables(plan)
    pk = {"abc": "FMM_PACK_ABC", "ab": "FMM_PACK_AB", "naive": "FMM_PACK_NAIVE"}[pack_type]
    out = [f"/* job library {job}: generated by fmm_gen_b200.control; plan of {plan.rank} products */\n",
           '#include "fmm_b200.h"\n\n',
           _c_array("int", "kDims", dims), f"static const int kRank = {plan.rank};\n",
           _c_array("int", "kNterms", nterms), _c_array("int", "kRows", rows), _c_array("int", "kCols", cols),
           _c_array("double", "kCoefs", coefs),
           "static fmm_plan *g_plan = 0;\n"
           "static int g_status = 0;\n\n"
           "__attribute__((constructor)) static void job_init(void) {\n"
           "  g_status = fmm_plan_create(kDims, kRank, kNterms, kRows, kCols, kCoefs, &g_plan);\n"
           "  if (g_status == FMM_OK) fmm_bind_default_plan(g_plan);\n"
           "}\n\n"
           "__attribute__((destructor)) static void job_fini(void) {\n"
           "  if (g_plan) fmm_plan_destroy(g_plan);\n"
           "  g_plan = 0;\n"
           "}\n\n"
           f"void bl_dgemm_strassen_{pack_type}(int m, int n, int k, double *A, int lda, double *B, int ldb,\n"
           f"                                  double *C, int ldc) {{\n"
           f"  g_status = g_plan ? fmm_dgemm_host(g_plan, {pk}, m, n, k, A, lda, B, ldb, C, ldc) : FMM_E_NOPLAN;\n"
           "}\n\n"
           "int fmm_job_status(void) { return g_status; }\n"]
    return "".join(out)


def test_driver_source(pack_type: str) -> str:
    """Driver with the reference driver's inputs and output line (meta/misc_gen.py:147-261),
    seeded instead of time-seeded, comparing with a relative tolerance."""
    return f"""/* test driver generated by fmm_gen_b200.control */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include "fmm_b200.h"

void bl_dgemm_strassen_{pack_type}(int m, int n, int k, double *A, int lda, double *B, int ldb, double *C, int ldc);

static double now(void) {{
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}}

int main(int argc, char *argv[]) {{
  int m, n, k, i, r;
  if (argc != 4) {{
    printf("Error: require 3 arguments, but only %d provided.\\n", argc - 1);
    return 0;
  }}
  m = atoi(argv[1]);
  n = atoi(argv[2]);
  k = atoi(argv[3]);
  double *A = malloc(sizeof(double) * (size_t)m * k), *B = malloc(sizeof(double) * (size_t)k * n);
  double *C = calloc((size_t)m * n, sizeof(double)), *Cr = calloc((size_t)m * n, sizeof(double));
  if (!A || !B || !C || !Cr) return 1;
  srand48(1);
  for (i = 0; i < m * k; ++i) A[i] = drand48();
  for (i = 0; i < k * n; ++i) B[i] = drand48();
  double t_fmm = 1e30, t_ref = 1e30;
  for (r = 0; r < 3; ++r) {{
    double t0 = now();
    bl_dgemm_strassen_{pack_type}(m, n, k, A, m, B, k, C, m);
    double t = now() - t0;
    if (t < t_fmm) t_fmm = t;
  }}
  for (r = 0; r < 3; ++r) {{
    double t0 = now();
    bl_dgemm(m, n, k, A, m, B, k, Cr, m);
    double t = now() - t0;
    if (t < t_ref) t_ref = t;
  }}
  double num = 0, den = 0;
  for (i = 0; i < m * n; ++i) {{
    num += (C[i] - Cr[i]) * (C[i] - Cr[i]);
    den += Cr[i] * Cr[i];
  }}
  double flops = ((double)m * n / (1000.0 * 1000.0 * 1000.0)) * (2.0 * k);
  printf("%5d\\t %5d\\t %5d\\t %5.2lf\\t %5.2lf\\n", m, n, k, flops / t_fmm, flops / t_ref);
  if (den > 0 && sqrt(num / den) > 1e-12) printf("C != C_ref: relative Frobenius difference %E\\n", sqrt(num / den));
  free(A);
  free(B);
  free(C);
  free(Cr);
  return 0;
}}
"""


def _cc() -> str:
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def generate_code(algs: Sequence[str], levels: Sequence[int], pack_type: str = "abc", path_prefix: str = "../",
                  compile_code: bool = True, x: Optional[float] = None) -> str:
    """Write (and by default compile) the job directory; returns its path.  `x` is the value
    of the approximate algorithms' parameter (the reference leaves it symbolic in its generated
    C, meta/common_util.py:56-60); it must be given when a level uses one."""
    job = job_name(algs, levels, pack_type)
    d = os.path.join(os.path.abspath(path_prefix), job)
    for sub in ("dgemm", "lib", "test", "include"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    plan = algebra.make_plan(list(algs), list(levels), x=x)
    with open(os.path.join(d, "plan.json"), "w") as fh:
        json.dump({"job": job, "levels": [[a, int(l)] for a, l in zip(algs, levels)], "dims": list(plan.dims),
                   "rank": plan.rank, "pack_type": pack_type,
                   "products": [{"a": [[t.row, t.col, t.coef] for t in p.a],
                                 "b": [[t.row, t.col, t.coef] for t in p.b],
                                 "c": [[t.row, t.col, t.coef] for t in p.c]} for p in plan.products]}, fh)
    src = os.path.join(d, "dgemm", f"my_dgemm_{job}.c")
    with open(src, "w") as fh:
        fh.write(job_library_source(plan, job, pack_type))
    shutil.copy(os.path.join(INCLUDE, "fmm_b200.h"), os.path.join(d, "include", "fmm_b200.h"))
    tsrc = os.path.join(d, "test", f"test_{job}.c")
    with open(tsrc, "w") as fh:
        fh.write(test_driver_source(pack_type))
    if compile_code:
        lib = os.path.join(d, "lib", f"lib{job}.so")
        inc = ["-I", os.path.join(d, "include")]
        subprocess.run([_cc(), "-O2", "-fPIC", "-shared"] + inc + ["-o", lib, src, "-L", LIB_DIR,
                        "-Wl,--no-as-needed", "-lfmm_b200", f"-Wl,-rpath,{LIB_DIR}"], check=True)
        exe = os.path.join(d, "test", f"test_{job}_mt.x")
        subprocess.run([_cc(), "-O2"] + inc + ["-o", exe, tsrc, "-L", os.path.join(d, "lib"), f"-l{job}",
                        "-L", LIB_DIR, "-lfmm_b200", "-lm",
                        f"-Wl,-rpath,{os.path.join(d, 'lib')}:{LIB_DIR}"], check=True)
        st = os.path.join(d, "test", f"test_{job}_st.x")
        if os.path.lexists(st):
            os.unlink(st)
        os.symlink(os.path.basename(exe), st)
    return d


def main(argv=None) -> None:
    argv = list(sys.argv[1:] if argv is None else argv)
    x = None
    if "--x" in argv:  # value of the approximate algorithms' parameter (an addition to the CLI)
        i = argv.index("--x")
        try:
            x = float(argv[i + 1])
        except (IndexError, ValueError):
            raise SystemExit("--x needs a number")
        del argv[i:i + 2]
    algs, levels, pack_type, gen_path = parse_argv(argv)
    from .build import build

    build()
    d = generate_code(algs, levels, pack_type, gen_path, x=x)
    print(d)


if __name__ == "__main__":
    main()
