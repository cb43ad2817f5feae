"""Algorithm algebra for generated fast matrix multiplication (FMM).

An FMM algorithm for a <mt,kt,nt> partition is a triple [U, V, W] of coefficient
matrices: product r is

    M_r = (sum_i U[i, r] * A_i) * (sum_j V[j, r] * B_j),   C_l += W[l, r] * M_r

where A_i, B_j, C_l are the sub-blocks of A (mt x kt grid), B (kt x nt grid) and
C (mt x nt grid), numbered row-major within the grid.  Several levels (or a hybrid
of different partitions) compose by the Kronecker product, outer level major.

Reference behaviour restated here (fmm-gen, paths relative to the project root):
  * coefficient grammar          meta/common_util.py:37-82   (parse_coeff)
  * coefficient file format      meta/common_util.py:84-104  (read_coeffs)
  * Kronecker composition        meta/common_mix.py:65-92, 324-341
  * level expansion (alg, L)     meta/abc_gen_mix.py:409-424
  * fringe split / sub-blocks    meta/common_mix.py:124-171, common/dgemm/bl_dgemm_util.c:284-298
  * block names                  meta/common_mix.py:184-219 (global (row, col)), 284-310 (a_i_j)
  * products execute in order r = 0..R-1 (meta/abc_gen_mix.py:259-263)
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# Register-tile granularity that decides the FMM/fringe split.  The split is part of
# the drop-in contract: rows m % (prod_mt * MR) and columns n % (prod_nt * NR) go to
# the classical fringe GEMMs (common/include/bl_config.h:16-17).
DGEMM_MR = 8
DGEMM_NR = 4

ALGORITHM_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "algorithms")


class CoefficientError(ValueError):
    pass


# ----------------------------------------------------------------------------------
# Coefficient grammar (meta/common_util.py:37-82):
#   e := number | letter | '(' e '+' e ... ')' | '-' e | e 'i' (inverse) |
#        digit e (multiplier) | e digit (power)
# A letter is the single algorithm parameter x of the approximate (APA) algorithms.
# ----------------------------------------------------------------------------------
def _is_number(tok: str) -> bool:
    try:
        float(tok)
        return True
    except ValueError:
        return False


def coeff_expr(tok: str) -> str:
    """Canonical C expression for a coefficient token (same grammar as the reference)."""
    tok = tok.strip()
    if _is_number(tok):
        return tok
    if len(tok) == 1:
        return "x"
    if tok[0] == "(":
        if tok[-1] != ")":
            raise CoefficientError(f"unbalanced coefficient: {tok}")
        return "(" + " + ".join(coeff_expr(t) for t in tok[1:-1].split("+")) + ")"
    if tok[0] == "-":
        return "-(%s)" % coeff_expr(tok[1:])
    if tok[-1] == "i":
        return "1.0 / (%s)" % coeff_expr(tok[:-1])
    if tok[0].isdigit():
        return "%s * (%s)" % (float(tok[0]), coeff_expr(tok[1:]))
    if tok[-1].isdigit():
        return " * ".join(coeff_expr(tok[:-1]) for _ in range(int(tok[-1])))
    raise CoefficientError(f"Cannot parse coefficient: {tok}")


def coeff_value(tok: str, x: Optional[float] = None) -> float:
    """Numeric value of a coefficient token; `x` is the APA parameter when one is used."""
    tok = tok.strip()
    if _is_number(tok):
        return float(tok)
    if len(tok) == 1:
        if x is None:
            raise CoefficientError(f"coefficient '{tok}' needs the algorithm parameter x")
        return float(x)
    if tok[0] == "(":
        if tok[-1] != ")":
            raise CoefficientError(f"unbalanced coefficient: {tok}")
        return sum(coeff_value(t, x) for t in tok[1:-1].split("+"))
    if tok[0] == "-":
        return -coeff_value(tok[1:], x)
    if tok[-1] == "i":
        return 1.0 / coeff_value(tok[:-1], x)
    if tok[0].isdigit():
        return float(tok[0]) * coeff_value(tok[1:], x)
    if tok[-1].isdigit():
        base = coeff_value(tok[:-1], x)
        out = 1.0
        for _ in range(int(tok[-1])):
            out *= base
        return out
    raise CoefficientError(f"Cannot parse coefficient: {tok}")


@dataclass
class Algorithm:
    """One coefficient file: U (mt*kt x R), V (kt*nt x R), W (mt*nt x R)."""

    name: str
    dims: Tuple[int, int, int]  # (mt, kt, nt)
    tokens: Tuple[List[List[str]], List[List[str]], List[List[str]]]
    x: Optional[float] = None

    @property
    def rank(self) -> int:
        return len(self.tokens[0][0])

    def matrices(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        return tuple(
            np.array([[coeff_value(t, self.x) for t in row] for row in grp], dtype=np.float64)
            for grp in self.tokens
        )

    def validate(self) -> None:
        mt, kt, nt = self.dims
        U, V, W = self.tokens
        want = (mt * kt, kt * nt, mt * nt)
        for name, grp, rows in zip("UVW", (U, V, W), want):
            if len(grp) != rows:
                raise CoefficientError(
                    f"{self.name}: {name} has {len(grp)} rows, expected {rows} for dims {self.dims}")
            if any(len(r) != self.rank for r in grp):
                raise CoefficientError(f"{self.name}: ragged {name} rows")


def read_coeffs(path: str) -> Tuple[List[List[str]], List[List[str]], List[List[str]]]:
    """Read a coefficient file: three '#'-separated groups (U, V, W).

    Lines starting with '#' end the current group (meta/common_util.py:84-104); other
    lines are whitespace-separated coefficient tokens, one row per sub-block.
    """
    groups: List[List[List[str]]] = []
    cur: List[List[str]] = []
    with open(path, "r") as fh:
        for line in fh:
            if line.startswith("#"):
                if cur:
                    groups.append(cur)
                    cur = []
                continue
            toks = line.split()
            if toks:
                cur.append(toks)
    groups.append(cur)
    groups = [g for g in groups if g]
    if len(groups) < 3:
        raise CoefficientError("Expected three sets of coefficients!")
    for g in groups[:3]:
        for row in g:
            for t in row:
                coeff_expr(t)  # grammar check
    return groups[0], groups[1], groups[2]


def load_algorithm(name_or_path: str, dims: Optional[Sequence[int]] = None,
                   x: Optional[float] = None) -> Algorithm:
    """Load an algorithm by table name (see alg_dic) or by coefficient-file path."""
    from .alg_dic import alg_dic

    if name_or_path in alg_dic:
        fname, tdims = alg_dic[name_or_path]
        path = os.path.join(ALGORITHM_DIR, fname)
        dims = tuple(tdims) if dims is None else tuple(dims)
        name = name_or_path
    else:
        path = name_or_path
        if dims is None:
            raise CoefficientError("dims are required when loading a coefficient file by path")
        name = os.path.basename(path)
    alg = Algorithm(name=name, dims=tuple(int(d) for d in dims), tokens=read_coeffs(path), x=x)
    alg.validate()
    return alg


# ----------------------------------------------------------------------------------
# Composition
# ----------------------------------------------------------------------------------
@dataclass
class Term:
    row: int      # global block row in the composed grid
    col: int      # global block column
    coef: float


@dataclass
class Product:
    a: List[Term]
    b: List[Term]
    c: List[Term]


@dataclass
class FMMPlan:
    """A composed multi-level FMM: the per-level algorithms and the product list."""

    level_names: List[str]
    level_dims: List[Tuple[int, int, int]]
    U: np.ndarray
    V: np.ndarray
    W: np.ndarray
    products: List[Product] = field(default_factory=list)

    @property
    def dims(self) -> Tuple[int, int, int]:
        m = k = n = 1
        for d in self.level_dims:
            m *= d[0]
            k *= d[1]
            n *= d[2]
        return (m, k, n)

    @property
    def rank(self) -> int:
        return self.U.shape[1]

    @property
    def nnz(self) -> Tuple[int, int, int]:
        return tuple(int(np.count_nonzero(X)) for X in (self.U, self.V, self.W))

    @property
    def max_terms(self) -> Tuple[int, int, int]:
        return tuple(int(np.count_nonzero(X, axis=0).max()) for X in (self.U, self.V, self.W))

    @property
    def job_levels(self) -> str:
        """'222-1_333-1'-style level string (control.py:47)."""
        out: List[str] = []
        prev = None
        for name in self.level_names:
            if out and name == prev:
                alg, lv = out[-1].rsplit("-", 1)
                out[-1] = f"{alg}-{int(lv) + 1}"
            else:
                out.append(f"{name}-1")
            prev = name
        return "_".join(out)

    def executed_flop_fraction(self) -> float:
        m, k, n = self.dims
        return self.rank / float(m * k * n)


def _global_rc(index: int, level_dims: Sequence[Tuple[int, int, int]], mm: int, nn: int) -> Tuple[int, int]:
    """Composed sub-block index -> global (row, col); outer level major
    (meta/common_mix.py:184-219)."""
    row = col = 0
    mbase = nbase = 1
    rem = index
    for d in reversed(level_dims):
        sz = d[mm] * d[nn]
        local = rem % sz
        ii, jj = divmod(local, d[nn])
        row += ii * mbase
        col += jj * nbase
        rem //= sz
        mbase *= d[mm]
        nbase *= d[nn]
    return row, col


def block_name(matrix: int, index: int, level_dims: Sequence[Tuple[int, int, int]]) -> str:
    """Per-level block name 'a_i_j...' (meta/common_mix.py:284-310)."""
    mm, nn = ((0, 1), (1, 2), (0, 2))[matrix]
    parts = []
    rem = index
    for d in reversed(level_dims):
        sz = d[mm] * d[nn]
        parts.append(str(rem % sz))
        rem //= sz
    return "abc"[matrix] + "".join("_" + p for p in reversed(parts))


def actual_block_name(matrix: int, index: int, level_dims: Sequence[Tuple[int, int, int]]) -> str:
    """Global block name 'A(row,col)' (meta/common_mix.py:184-219)."""
    mm, nn = ((0, 1), (1, 2), (0, 2))[matrix]
    r, c = _global_rc(index, level_dims, mm, nn)
    return "ABC"[matrix] + f"({r},{c})"


def compose(levels: Sequence[Algorithm]) -> FMMPlan:
    """Kronecker-compose per-level algorithms (outer level first)."""
    if not levels:
        raise CoefficientError("at least one level is required")
    U, V, W = levels[0].matrices()
    for alg in levels[1:]:
        u, v, w = alg.matrices()
        U, V, W = np.kron(U, u), np.kron(V, v), np.kron(W, w)
    level_dims = [alg.dims for alg in levels]
    plan = FMMPlan([alg.name for alg in levels], level_dims, U, V, W)
    for r in range(U.shape[1]):
        terms = []
        for mat, (X, (mm, nn)) in enumerate(zip((U, V, W), ((0, 1), (1, 2), (0, 2)))):
            col = X[:, r]
            ts = []
            for i in np.nonzero(col)[0]:
                br, bc = _global_rc(int(i), level_dims, mm, nn)
                ts.append(Term(br, bc, float(col[i])))
            terms.append(ts)
        plan.products.append(Product(*terms))
    return plan


def expand_levels(algs: Sequence[str], levels: Sequence[int], x: Optional[float] = None) -> List[Algorithm]:
    """(alg, L) pairs -> one Algorithm per level (meta/abc_gen_mix.py:409-424)."""
    if len(algs) != len(levels):
        raise CoefficientError("each algorithm needs a level count")
    out: List[Algorithm] = []
    for name, lv in zip(algs, levels):
        if int(lv) < 1:
            raise CoefficientError(f"level count must be >= 1 (got {lv} for {name})")
        alg = load_algorithm(name, x=x)
        out.extend([alg] * int(lv))
    return out


def make_plan(algs: Sequence[str], levels: Sequence[int], x: Optional[float] = None) -> FMMPlan:
    """Compose the plan for e.g. (['222', '333'], [1, 1])."""
    plan = compose(expand_levels(algs, levels, x=x))
    plan.level_names = []
    for name, lv in zip(algs, levels):
        plan.level_names.extend([name] * int(lv))
    return plan


def classical_plan(mt: int = 1, kt: int = 1, nt: int = 1) -> FMMPlan:
    """The classical algorithm as a plan (every product is one block product)."""
    R = mt * kt * nt
    U = np.zeros((mt * kt, R))
    V = np.zeros((kt * nt, R))
    W = np.zeros((mt * nt, R))
    r = 0
    for i in range(mt):
        for j in range(nt):
            for p in range(kt):
                U[i * kt + p, r] = 1
                V[p * nt + j, r] = 1
                W[i * nt + j, r] = 1
                r += 1
    tokens = tuple([[("1" if v else "0") for v in row] for row in X] for X in (U, V, W))
    alg = Algorithm(f"classical{mt}{kt}{nt}", (mt, kt, nt), tokens)
    plan = compose([alg])
    return plan


# ----------------------------------------------------------------------------------
# Fringe split (meta/common_mix.py:124-171; common/dgemm/bl_dgemm_util.c:316-353)
# ----------------------------------------------------------------------------------
@dataclass(frozen=True)
class Partition:
    m: int
    n: int
    k: int
    ms: int
    ks: int
    ns: int
    md: int
    kd: int
    nd: int
    mr: int
    kr: int
    nr: int


def partition(m: int, n: int, k: int, dims: Tuple[int, int, int]) -> Partition:
    mt, kt, nt = dims
    mr = m % (mt * DGEMM_MR)
    kr = k % kt
    nr = n % (nt * DGEMM_NR)
    md, kd, nd = m - mr, k - kr, n - nr
    return Partition(m, n, k, md // mt, kd // kt, nd // nt, md, kd, nd, mr, kr, nr)


def effective_flops(m: int, n: int, k: int) -> float:
    """The reference's effective flop count 2mnk (meta/misc_gen.py:227)."""
    return 2.0 * m * n * k


def executed_flops(plan: FMMPlan, m: int, n: int, k: int) -> float:
    """Flops the FMM actually executes: R sub-GEMMs plus the classical fringes."""
    p = partition(m, n, k, plan.dims)
    core = plan.rank * 2.0 * p.ms * p.ns * p.ks
    fringe = 2.0 * (p.md * p.nd * p.kr + m * p.nr * k + p.mr * p.nd * k)
    return core + fringe


def e_max(plan: FMMPlan) -> float:
    """Largest coefficient-weighted product count feeding one C block:

        e_max = max_l sum_r |W[l,r]| * ||U[:,r]||_1 * ||V[:,r]||_1

    (12 for Strassen).  It is multiplicative under the Kronecker composition, so the
    composed plan's value equals the product of the levels' values.  This quantity
    appears in the stability analysis of fast matrix multiplication by Ballard,
    Benson, Druinsky, Lipshitz and Schwartz (SIMAX 37(4), 2016).
    """
    a = np.abs(plan.U).sum(axis=0)
    b = np.abs(plan.V).sum(axis=0)
    return float((np.abs(plan.W) * (a * b)[None, :]).sum(axis=1).max())


def error_bound(plan: FMMPlan, m: int, n: int, k: int, amax: float, bmax: float, cmax: float = 0.0,
                unit_roundoff: float = 2.0 ** -53) -> float:
    """First-order max-norm forward error bound of one FMM call C += A*B.

    Derivation (elementwise, standard rounding-error analysis): an operand sum with
    at most `a` terms is off by <= a*u*sum|u_i||A_i|; a product of depth K_s adds
    K_s*u*|S||T|; accumulating the products into a C block with at most `c` terms adds
    c*u*(|C| + sum_r |w||M_r|).  With |S_r| <= ||U[:,r]||_1 ||A||_max and likewise for
    T_r this gives

        |C_hat - C|_max <= (a + b + c + K_s) u K_s e_max ||A||_max ||B||_max + (c+1) u ||C0||_max

    and the classical fringe GEMMs satisfy the same form with e_max = 1, depth k.
    The bound holds for any summation order, so it covers both the reference's
    KC-chunked CPU arithmetic and the GPU's fused multiply-adds.
    """
    p = partition(m, n, k, plan.dims)
    ta, tb, tc = plan.max_terms
    ks = max(p.ks, 1)
    core = (ta + tb + tc + ks) * ks * e_max(plan)
    fringe = (k + 2) * k
    if p.kr > 0:
        core += (p.kr + 2) * p.kr
    return unit_roundoff * (max(core, fringe) * amax * bmax + (tc + 2) * cmax)
