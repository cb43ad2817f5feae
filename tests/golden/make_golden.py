"""Generate the golden fixtures that pin the oracle and the algebra layer to fmm-gen.

Run where an fmm-gen checkout exists, named by the environment variable FMM_REF (no
default); the fixtures it writes next to this file are committed, so the tests never
read the checkout.

What it does:
  1. Loads the reference's Python 2 generator modules (meta/*.py) into memory with a
     minimal source-level Python 3 shim (print statements, xrange, integer division
     in the block-name helpers, len(filter(...))).  Nothing under the checkout is
     written.
  2. For each algorithm configuration, records the composed [U,V,W] exactly as the
     reference composes them (meta/common_mix.py:324-341) and every product's block
     names (meta/common_mix.py:184-219, 284-310)  ->  coeffs_<job>.json
  3. Emits the reference's C for configurations x pack types with its own generator
     functions (gen_abc_fmm / gen_ab_fmm / gen_naive_fmm, meta/*_gen_mix.py) into a
     temporary directory, compiles it with gcc together with the reference runtime
     (common/dgemm, common/kernels) using the reference's gcc flags, and runs the
     generated bl_dgemm_strassen_<pack> and bl_dgemm on seeded inputs with fringe
     shapes  ->  out_<job>.npz
     One reference defect is repaired in the emitted text, not in the generator: the
     multi-destination micro-kernel's asm input operands are emitted without commas
     (meta/abc_micro_kernel_gen.py:1104-1108), so it does not compile when a product
     updates two or more C blocks; the missing commas are inserted.

Usage:  FMM_REF=<fmm-gen checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import json
import os
import re
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("FMM_REF", "")
META = os.path.join(REF, "meta")
ALGS = os.path.join(META, "algorithms")

# (algorithms, levels) -> tag.  Pure partitions map through the reference table.
CONFIGS = [
    (["222"], [1]),
    (["222"], [2]),
    (["232"], [1]),
    (["333"], [1]),
    (["222", "333"], [1, 1]),
    (["222", "232"], [1, 1]),
    (["424"], [1]),   # +-0.5 coefficients
    (["336"], [1]),   # +-0.125 coefficients, W columns with many nonzeros
    (["323"], [1]),
    (["classical222_8_24"], [1]),
]

# Generated-code runs: (config index, pack types, shapes (m, n, k)) -- shapes include
# every fringe (mr, kr, nr > 0) and one that is an exact multiple.
RUNS = [
    (0, ["abc", "ab", "naive"], [(64, 48, 40), (101, 77, 53)]),
    (1, ["abc"], [(128, 96, 72), (141, 103, 67)]),
    (2, ["abc"], [(80, 64, 60), (97, 70, 61)]),
    (3, ["abc"], [(96, 72, 54), (103, 77, 58)]),
    (4, ["abc", "ab", "naive"], [(96, 48, 36), (100, 53, 40)]),
    (6, ["abc"], [(128, 64, 40), (133, 70, 43)]),
    (7, ["abc"], [(96, 96, 45), (101, 99, 47)]),
]
PLAIN_SHAPES = [(1, 1, 1), (9, 5, 3), (37, 29, 300), (130, 67, 517)]


def job_name(algs, levels):
    return "_".join(f"{a}-{l}" for a, l in zip(algs, levels))


# ---------------------------------------------------------------------------------
# Python 3 shim for the reference generator
# ---------------------------------------------------------------------------------
def _py3(src: str) -> str:
    out = []
    for line in src.split("\n"):
        m = re.match(r"^(\s*)print\s+(?!\()(.*)$", line)
        if m:
            line = f"{m.group(1)}print({m.group(2)})"
        m = re.match(r"^(\s*)print\s*(\(.*)$", line)
        if m and not line.rstrip().endswith(")"):
            pass
        out.append(line)
    s = "\n".join(out)
    s = re.sub(r"\bxrange\b", "range", s)
    s = re.sub(r"len\(filter\(([^()]*)\)\)", r"len(list(filter(\1)))", s)
    s = s.replace("ii = remainder / dims[nn]", "ii = remainder // dims[nn]")
    s = s.replace("dividend = dividend / ( dims[mm] * dims[nn] )", "dividend = dividend // ( dims[mm] * dims[nn] )")
    return s


def load_reference():
    mods = {}
    order = ["common_util", "common_mix", "abc_micro_kernel_gen", "abc_gen_mix", "ab_gen_mix", "naive_gen_mix",
             "alg_dic"]
    for name in order:
        path = os.path.join(META, name + ".py")
        with open(path) as fh:
            src = _py3(fh.read())
        mod = types.ModuleType(name)
        mod.__file__ = path
        sys.modules[name] = mod
        exec(compile(src, path, "exec"), mod.__dict__)
        mods[name] = mod
    return mods


def resolve(mods, algs, levels):
    dic = mods["alg_dic"].alg_dic
    files, dims = [], []
    for a in algs:
        rel, d = dic[a]
        files.append(os.path.join(ALGS, os.path.basename(rel)) if "ignore" not in rel
                     else os.path.join(ALGS, "ignore", os.path.basename(rel)))
        dims.append(tuple(d))
    return files, dims


def coeff_fixture(mods, algs, levels):
    cu, cm = mods["common_util"], mods["common_mix"]
    files, dims = resolve(mods, algs, levels)
    coeffs_mix, dims_mix = [], []
    for f, d, lv in zip(files, dims, levels):
        c = cu.read_coeffs(f)
        for _ in range(lv):
            coeffs_mix.append(c)
            dims_mix.append(d)
    comp = cm.generateCoeffs(coeffs_mix)
    R = len(comp[0][0])
    prods = []
    for r in range(R):
        entry = {}
        for mat, key in ((0, "a"), (1, "b"), (2, "c")):
            col = [row[r] for row in comp[mat]]
            terms = []
            for i, v in enumerate(col):
                if cu.is_nonzero(v):
                    actual = cm.getActualBlockName(mat, i, dims_mix)
                    rr, cc = re.match(r"[ABC]\((\d+),(\d+)\)", actual).groups()
                    terms.append({"index": i, "row": int(rr), "col": int(cc), "coef": float(v), "text": str(v),
                                  "name": cm.getBlockName(mat, i, dims_mix), "actual": actual})
            entry[key] = terms
        prods.append(entry)
    tot = [1, 1, 1]
    for d in dims_mix:
        tot = [tot[0] * d[0], tot[1] * d[1], tot[2] * d[2]]
    return {"algs": algs, "levels": levels, "level_dims": [list(d) for d in dims_mix], "dims": tot, "rank": R,
            "products": prods}


# ---------------------------------------------------------------------------------
# Build and run the generated C
# ---------------------------------------------------------------------------------
CFLAGS = ["-O3", "-mavx", "-fopenmp", "-ffp-contract=off", "-fgnu89-inline", "-fPIC", "-shared", "-w"]
GCC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _fix_asm_operands(path):
    """Insert the commas missing between consecutive asm input operands."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    opnd = re.compile(r'^(\s*"m" \((?:c\d+|alpha_list)\))(\s*//.*)?$')
    for i in range(len(lines) - 1):
        m = opnd.match(lines[i])
        if m and opnd.match(lines[i + 1]):
            lines[i] = m.group(1) + "," + (m.group(2) or "")
    with open(path, "w") as fh:
        fh.write("\n".join(lines))


def _product_subset(gen_mod, products):
    """Restrict the generator's composed [U,V,W] to the product columns `products` (in that
    order) while a subset library is emitted: every kept product's code is the one the full
    generator writes for it, the products are renumbered 0..len-1."""
    full = gen_mod.generateCoeffs

    def subset(coeffs_mix):
        return [[[row[r] for r in products] for row in mat] for mat in full(coeffs_mix)]

    gen_mod.generateCoeffs = subset
    return full


def build_job(mods, algs, levels, pack, work, products=None, extra_cflags=(), out=None, compile_now=True):
    """Emit the reference's C for one job with its own generator and compile it (with the
    reference runtime) into a shared library; `products` keeps only those products of the
    composed algorithm (abc only), `out` names the library (default: under `work`); with
    compile_now=False the gcc command is returned instead of run."""
    if products is not None and pack != "abc":
        raise ValueError("product subsets are emitted for the abc pack type only")
    job = job_name(algs, levels) + "_" + pack
    if products is not None:
        job += "_p" + "-".join(str(r) for r in products[:1]) + f"x{len(products)}"
    d = os.path.join(work, job)
    for sub in ("dgemm", "kernels", "include"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    files, dims = resolve(mods, algs, levels)
    out_c = os.path.join(d, "dgemm", f"my_dgemm_{job}.c")
    srcs = [out_c]
    cwd = os.getcwd()
    os.chdir(d)
    try:
        if pack == "abc":
            mk = f"./kernels/bl_kernel_{job}.c"
            hd = f"./include/bl_kernel_{job}.h"
            gen = mods["abc_gen_mix"]
            full = _product_subset(gen, products) if products is not None else None
            try:
                gen.gen_abc_fmm(files, dims, levels, out_c, mk, hd)
            finally:
                if full is not None:
                    gen.generateCoeffs = full
            srcs.append(os.path.join(d, mk))
        elif pack == "ab":
            mods["ab_gen_mix"].gen_ab_fmm(files, dims, levels, out_c)
        else:
            mods["naive_gen_mix"].gen_naive_fmm(files, dims, levels, out_c)
    finally:
        os.chdir(cwd)
    for s in srcs:
        _fix_asm_operands(s)
    common = os.path.join(REF, "common")
    lib = out or os.path.join(d, f"lib{job}.so")
    cmd = [GCC] + CFLAGS + list(extra_cflags) + ["-I", os.path.join(d, "include"), "-I", os.path.join(common, "include"), "-o", lib] + srcs + [
        os.path.join(common, "dgemm", "my_dgemm.c"), os.path.join(common, "dgemm", "bl_dgemm_util.c"),
        os.path.join(common, "kernels", "bl_dgemm_asm_8x4.c"),
        os.path.join(common, "kernels", "bl_dgemm_asm_8x4_mulstrassen.c"),
        os.path.join(os.path.dirname(HERE), "..", "oracle", "ref_blas_stub.c")]
    if not compile_now:
        return cmd
    subprocess.run(cmd, check=True)
    return lib


def padded(m, n):
    """C as the reference's driver allocates it: ldc = ceil(m/8)*8, n+4 columns, 32 B aligned."""
    ldc = ((m - 1) // 8 + 1) * 8
    buf = np.zeros(ldc * (n + 4) + 8)
    off = (-buf.ctypes.data % 32) // 8
    flat = buf[off:off + ldc * (n + 4)]
    return flat, ldc


def run_lib(lib, fn, cases):
    """Run `fn` from `lib` in a fresh process per library (the reference's packing pool
    is sized by the first call, so shapes run in non-increasing n)."""
    L = ctypes.CDLL(lib)
    f = getattr(L, fn)
    f.restype = None
    outs = []
    for (m, n, k, A, B, C0) in cases:
        flat, ldc = padded(m, n)
        Cv = flat[: ldc * n].reshape(n, ldc).T
        Cv[:m, :] = C0
        Af = np.asfortranarray(A)
        Bf = np.asfortranarray(B)
        f(ctypes.c_int(m), ctypes.c_int(n), ctypes.c_int(k), Af.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(m),
          Bf.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(k), flat.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(ldc))
        outs.append(np.array(Cv[:m, :n]))
    return outs


def inputs(seed, m, n, k):
    rng = np.random.Generator(np.random.PCG64(seed))
    A = rng.uniform(-1.0, 1.0, size=(m, k))
    B = rng.uniform(-1.0, 1.0, size=(k, n))
    C = rng.uniform(-1.0, 1.0, size=(m, n))
    return A, B, C


def _child(lib, fn, shapes, seed0, out):
    cases = []
    for i, (m, n, k) in enumerate(shapes):
        A, B, C = inputs(seed0 + i, m, n, k)
        cases.append((m, n, k, A, B, C))
    order = sorted(range(len(cases)), key=lambda i: -cases[i][1])
    res = run_lib(lib, fn, [cases[i] for i in order])
    outs = [None] * len(cases)
    for j, i in enumerate(order):
        outs[i] = res[j]
    np.savez(out, *outs)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--child":
        _, _, lib, fn, shapes, seed0, out = sys.argv
        _child(lib, fn, json.loads(shapes), int(seed0), out)
        return
    if not REF or not os.path.isdir(META):
        sys.exit("set FMM_REF to an fmm-gen checkout (the directory that holds meta/ and common/)")
    os.environ["BLISLAB_IC_NT"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    mods = load_reference()
    for algs, levels in CONFIGS:
        fx = coeff_fixture(mods, algs, levels)
        with open(os.path.join(HERE, f"coeffs_{job_name(algs, levels)}.json"), "w") as fh:
            json.dump(fx, fh, indent=0, separators=(",", ":"))
    work = tempfile.mkdtemp(prefix="fmm_golden_")
    seed = 1000
    for ci, packs, shapes in RUNS:
        algs, levels = CONFIGS[ci]
        job = job_name(algs, levels)
        record = {}
        for pack in packs:
            lib = build_job(mods, algs, levels, pack, work)
            tmp = os.path.join(work, f"{job}_{pack}.npz")
            subprocess.run([sys.executable, __file__, "--child", lib, f"bl_dgemm_strassen_{pack}",
                            json.dumps(shapes), str(seed), tmp], check=True)
            got = np.load(tmp)
            for i, (m, n, k) in enumerate(shapes):
                record[f"{pack}_{i}"] = got[f"arr_{i}"]
        meta = {"shapes": shapes, "seed0": seed, "packs": packs}
        np.savez_compressed(os.path.join(HERE, f"out_{job}.npz"), meta=json.dumps(meta), **record)
        seed += 100
    # the reference's classical bl_dgemm
    lib = build_job(mods, ["222"], [1], "ab", work)  # any job library also exports bl_dgemm
    tmp = os.path.join(work, "plain.npz")
    subprocess.run([sys.executable, __file__, "--child", lib, "bl_dgemm", json.dumps(PLAIN_SHAPES), "5000", tmp],
                   check=True)
    got = np.load(tmp)
    np.savez_compressed(os.path.join(HERE, "out_plain.npz"),
                        meta=json.dumps({"shapes": PLAIN_SHAPES, "seed0": 5000}),
                        **{f"plain_{i}": got[f"arr_{i}"] for i in range(len(PLAIN_SHAPES))})
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
