/*
 * ORACLE — test infrastructure only.  Not part of the product: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only as
 * the checker or the timed CPU reference arm.
 *
 * A plain-C restatement of the reference's CPU arithmetic (fmm-gen), written so that
 * every element is computed with the same operations in the same order as the
 * reference's generated code.  Compiled with -ffp-contract=off (no fused multiply-
 * add, like the reference's AVX1 vmulpd+vaddpd), its results are bit-identical to
 * the reference's; tests/golden pins that against outputs of the reference itself.
 *
 * Followed reference code (paths relative to the fmm-gen project root):
 *   classical GEMM, per element C += sum over each KC=256 chunk, mul then add
 *       common/dgemm/my_dgemm.c:115-210, common/kernels/bl_dgemm_asm_8x4.c:3-375
 *   ABC:   for r: for each KC chunk: pack sums (left-to-right expression),
 *          rank-KC product, C_l = C_l (+|-) acc or C_l + (w*acc)
 *       meta/abc_gen_mix.py:171-251 (packing expression), :302-391 (loop order),
 *       meta/abc_micro_kernel_gen.py:147-244 (C update)
 *   AB:    M_r = 0; M_r += each chunk's product; C_l += w-expression of M_r
 *       meta/ab_gen_mix.py:219-303, :341-372
 *   NAIVE: S_r, T_r temporaries (only if the column has more than one entry that is
 *          not 1, zeros included), M_r = bl_dgemm(S_r, T_r), C_l += ...
 *       meta/naive_gen_mix.py:60-137, :205-212, :244-361
 *   fringe split and peeling
 *       meta/common_mix.py:124-171, common/dgemm/bl_dgemm_util.c:316-353
 *
 * Also: a compensated (Dot2, Ogita-Rump-Oishi 2005) classical GEMM used as the
 * accuracy oracle for relative Frobenius errors.
 */
#include <math.h>
#ifdef __AVX__
#include <immintrin.h>
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KC 256
#define MR 8
#define NR 4

/* expression value of one packed element: t0 op t1 op ... (meta/abc_gen_mix.py:229-251) */
static inline double lin_expr(int nt, const double *const *src, const double *coef, long off) {
  double v;
  const double c0 = coef[0];
  if (c0 == 1.0)
    v = src[0][off];
  else if (c0 == -1.0)
    v = -src[0][off];
  else
    v = c0 * src[0][off];
  for (int t = 1; t < nt; ++t) {
    const double c = coef[t];
    const double x = src[t][off];
    if (c == 1.0)
      v = v + x;
    else if (c == -1.0)
      v = v - x;
    else
      v = v + c * x;
  }
  return v;
}

/* C update of one destination (meta/abc_micro_kernel_gen.py:147-244; M_Add: ab_gen_mix.py:341-372) */
static inline double upd(double c, double w, double acc) {
  if (w == 1.0) return c + acc;
  if (w == -1.0) return c - acc;
  return c + w * acc;
}

#define MAX_TERMS 1024 /* operand / C terms of one product (three-level plans reach 1000) */
typedef struct {
  int nt;
  const double *src[MAX_TERMS];
  double coef[MAX_TERMS];
  long ld;
} opnd_t;

/* Pack rows [0, m) x k-chunk [pc, pc+pb) of an operand sum into MR-row panels;
 * rows past m are zero. layout: panel ip, column p, row ii -> out[(ip*pb+p)*MR+ii] */
static void pack_rows(const opnd_t *A, int m, int pc, int pb, double *out) {
  const int np = (m + MR - 1) / MR;
#pragma omp parallel for schedule(static)
  for (int ip = 0; ip < np; ++ip) {
    for (int p = 0; p < pb; ++p) {
      double *dst = out + ((long)ip * pb + p) * MR;
      for (int ii = 0; ii < MR; ++ii) {
        const int i = ip * MR + ii;
        dst[ii] = (i < m) ? lin_expr(A->nt, A->src, A->coef, i + (long)(pc + p) * A->ld) : 0.0;
      }
    }
  }
}

/* Pack k-chunk x columns [0, n) of an operand sum into NR-column panels. */
static void pack_cols(const opnd_t *B, int n, int pc, int pb, double *out) {
  const int np = (n + NR - 1) / NR;
#pragma omp parallel for schedule(static)
  for (int jp = 0; jp < np; ++jp) {
    for (int p = 0; p < pb; ++p) {
      double *dst = out + ((long)jp * pb + p) * NR;
      for (int jj = 0; jj < NR; ++jj) {
        const int j = jp * NR + jj;
        dst[jj] = (j < n) ? lin_expr(B->nt, B->src, B->coef, (pc + p) + (long)j * B->ld) : 0.0;
      }
    }
  }
}

/* The 8x4 register tile of one KC chunk: acc(ii,jj) = sum_p a(ii,p)*b(p,jj), each step
 * a multiply then an add (both rounded), p in order from 0 -- the operation sequence of
 * the reference's AVX micro-kernel (common/kernels/bl_dgemm_asm_8x4.c:59-300). */
static inline void micro_8x4(int pb, const double *a, const double *b, double acc[NR][MR]) {
#ifdef __AVX__
  __m256d c[NR][2];
  for (int jj = 0; jj < NR; ++jj) c[jj][0] = c[jj][1] = _mm256_setzero_pd();
  for (int p = 0; p < pb; ++p) {
    const __m256d a0 = _mm256_loadu_pd(a + p * MR), a1 = _mm256_loadu_pd(a + p * MR + 4);
    for (int jj = 0; jj < NR; ++jj) {
      const __m256d bv = _mm256_broadcast_sd(b + p * NR + jj);
      c[jj][0] = _mm256_add_pd(c[jj][0], _mm256_mul_pd(a0, bv));
      c[jj][1] = _mm256_add_pd(c[jj][1], _mm256_mul_pd(a1, bv));
    }
  }
  for (int jj = 0; jj < NR; ++jj) {
    _mm256_storeu_pd(acc[jj], c[jj][0]);
    _mm256_storeu_pd(acc[jj] + 4, c[jj][1]);
  }
#else
  for (int jj = 0; jj < NR; ++jj)
    for (int ii = 0; ii < MR; ++ii) acc[jj][ii] = 0.0;
  for (int p = 0; p < pb; ++p)
    for (int jj = 0; jj < NR; ++jj) {
      const double bv = b[p * NR + jj];
      for (int ii = 0; ii < MR; ++ii) acc[jj][ii] = acc[jj][ii] + a[p * MR + ii] * bv;
    }
#endif
}

/* One KC chunk: for every element acc = sum_p a*b (in p order, from 0), then each
 * destination d: D_d(i,j) = upd(D_d(i,j), w_d, acc).  Threads own blocks of MC rows
 * (the reference's ic loop, my_dgemm.c:168-198) so a packed A block stays in cache. */
#define MC_PANELS 12 /* 96 rows, DGEMM_MC (common/include/bl_config.h:13) */
static void chunk_update(int m, int n, int pb, const double *Ap, const double *Bp, int nd, double *const *dst,
                         const double *w, long ldd) {
  const int npi = (m + MR - 1) / MR, npj = (n + NR - 1) / NR;
  const int nblk = (npi + MC_PANELS - 1) / MC_PANELS;
#pragma omp parallel for schedule(dynamic, 1)
  for (int ib = 0; ib < nblk; ++ib) {
    const int ip0 = ib * MC_PANELS, ip1 = (ip0 + MC_PANELS < npi) ? ip0 + MC_PANELS : npi;
    for (int jp = 0; jp < npj; ++jp) {
      const double *b = Bp + (long)jp * pb * NR;
      for (int ip = ip0; ip < ip1; ++ip) {
        double acc[NR][MR];
        micro_8x4(pb, Ap + (long)ip * pb * MR, b, acc);
        for (int jj = 0; jj < NR; ++jj) {
          const int j = jp * NR + jj;
          if (j >= n) break;
          for (int ii = 0; ii < MR; ++ii) {
            const int i = ip * MR + ii;
            if (i >= m) break;
            for (int d = 0; d < nd; ++d) {
              double *c = dst[d] + i + (long)j * ldd;
              *c = upd(*c, w[d], acc[jj][ii]);
            }
          }
        }
      }
    }
  }
}

/* C(m x n) += opA(m x k) * opB(k x n), chunked by KC, into nd destinations. */
static int product_into(const opnd_t *A, const opnd_t *B, int m, int n, int k, int nd, double *const *dst,
                        const double *w, long ldd) {
  if (m <= 0 || n <= 0 || k <= 0) return 0;
  const int npi = (m + MR - 1) / MR, npj = (n + NR - 1) / NR;
  double *Ap = (double *)malloc(sizeof(double) * (size_t)npi * MR * KC);
  double *Bp = (double *)malloc(sizeof(double) * (size_t)npj * NR * KC);
  if (!Ap || !Bp) {
    free(Ap);
    free(Bp);
    return -4;
  }
  for (int pc = 0; pc < k; pc += KC) {
    const int pb = (k - pc) < KC ? (k - pc) : KC;
    pack_rows(A, m, pc, pb, Ap);
    pack_cols(B, n, pc, pb, Bp);
    chunk_update(m, n, pb, Ap, Bp, nd, dst, w, ldd);
  }
  free(Ap);
  free(Bp);
  return 0;
}

/* Classical C += A*B with the reference's per-element arithmetic. */
int oracle_bl_dgemm(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc) {
  opnd_t a = {1, {A}, {1.0}, lda};
  opnd_t b = {1, {B}, {1.0}, ldb};
  double *d[1] = {C};
  const double w[1] = {1.0};
  return product_into(&a, &b, m, n, k, 1, d, w, ldc);
}

static int peel(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc, int d1,
                int d2, int d3) {
  const int mr = m % d1, kr = k % d2, nr = n % d3;
  const int ms = m - mr, ns = n - nr, ks = k - kr;
  int rc = 0;
  if (kr > 0 && ms > 0 && ns > 0) rc |= oracle_bl_dgemm(ms, ns, kr, A + (long)ks * lda, lda, B + ks, ldb, C, ldc);
  if (nr > 0) rc |= oracle_bl_dgemm(m, nr, k, A, lda, B + (long)ns * ldb, ldb, C + (long)ns * ldc, ldc);
  if (mr > 0 && ns > 0) rc |= oracle_bl_dgemm(mr, ns, k, A + ms, lda, B, ldb, C + ms, ldc);
  return rc;
}

int oracle_dynamic_peeling(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C,
                           int ldc, int d1, int d2, int d3) {
  return peel(m, n, k, A, lda, B, ldb, C, ldc, d1, d2, d3);
}

/*
 * FMM C += A*B.  pack: 0 abc, 1 ab, 2 naive.  Plan tables as in fmm_plan_create():
 * dims = (prod mt, prod kt, prod nt), R products, nterms[3R] (#A, #B, #C terms per
 * product), then rows/cols/coefs of the terms product-major (A, B, C).
 */
int oracle_fmm(int pack, const int *dims, int R, const int *nterms, const int *rows, const int *cols,
               const double *coefs, int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C,
               int ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return 0;
  const int d1 = dims[0] * MR, d2 = dims[1], d3 = dims[2] * NR;
  const int md = m - m % d1, kd = k - k % d2, nd = n - n % d3;
  const int ms = md / dims[0], ks = kd / dims[1], ns = nd / dims[2];
  int rc = 0;
  if (ms > 0 && ns > 0 && ks > 0) {
    double *M = NULL;
    if (pack != 0) {
      M = (double *)malloc(sizeof(double) * (size_t)ms * ns);
      if (!M) return -4;
    }
    int pos = 0;
    for (int r = 0; r < R && rc == 0; ++r) {
      const int na = nterms[3 * r], nb = nterms[3 * r + 1], nc = nterms[3 * r + 2];
      if (na > MAX_TERMS || nb > MAX_TERMS || nc > MAX_TERMS) {
        rc = -6;
        break;
      }
      opnd_t a, b;
      a.nt = na;
      a.ld = lda;
      for (int t = 0; t < na; ++t, ++pos) {
        a.src[t] = A + (long)rows[pos] * ms + (long)cols[pos] * ks * lda;
        a.coef[t] = coefs[pos];
      }
      b.nt = nb;
      b.ld = ldb;
      for (int t = 0; t < nb; ++t, ++pos) {
        b.src[t] = B + (long)rows[pos] * ks + (long)cols[pos] * ns * ldb;
        b.coef[t] = coefs[pos];
      }
      double *cd[MAX_TERMS];
      double w[MAX_TERMS];
      for (int t = 0; t < nc; ++t, ++pos) {
        cd[t] = C + (long)rows[pos] * ms + (long)cols[pos] * ns * ldc;
        w[t] = coefs[pos];
      }
      if (pack == 2) {
        /* need_tmp_mat: more than one entry of the full column is not 1 (zeros count) */
        const int nnon_a = dims[0] * dims[1] - na + (int)0;
        int na_nonone = nnon_a, nb_nonone = dims[1] * dims[2] - nb;
        for (int t = 0; t < na; ++t) na_nonone += (a.coef[t] != 1.0);
        for (int t = 0; t < nb; ++t) nb_nonone += (b.coef[t] != 1.0);
        if (na_nonone <= 1) {
          a.nt = 1;
          a.coef[0] = 1.0;
        }
        if (nb_nonone <= 1) {
          b.nt = 1;
          b.coef[0] = 1.0;
        }
      }
      if (pack == 0) {
        rc = product_into(&a, &b, ms, ns, ks, nc, cd, w, ldc);
      } else {
        memset(M, 0, sizeof(double) * (size_t)ms * ns);
        double *md_[1] = {M};
        const double one[1] = {1.0};
        rc = product_into(&a, &b, ms, ns, ks, 1, md_, one, ms);
        if (rc) break;
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ns; ++j)
          for (int i = 0; i < ms; ++i) {
            const double mv = M[i + (long)j * ms];
            for (int t = 0; t < nc; ++t) {
              double *c = cd[t] + i + (long)j * ldc;
              *c = upd(*c, w[t], mv);
            }
          }
      }
    }
    free(M);
    if (rc) return rc;
  }
  return peel(m, n, k, A, lda, B, ldb, C, ldc, d1, d2, d3);
}

/* Dot2 (Ogita, Rump, Oishi, "Accurate sum and dot product", SISC 2005): error-free
 * TwoProduct by Dekker/Veltkamp splitting, TwoSum by Knuth; result as if computed in
 * twice the working precision, then rounded.  C += A*B, used only to measure errors. */
static inline void two_sum(double a, double b, double *s, double *e) {
  const double x = a + b;
  const double z = x - a;
  *e = (a - (x - z)) + (b - z);
  *s = x;
}
static inline void split(double a, double *hi, double *lo) {
  const double f = 134217729.0; /* 2^27 + 1 */
  const double c = f * a;
  const double h = c - (c - a);
  *hi = h;
  *lo = a - h;
}
static inline void two_prod(double a, double b, double *p, double *e) {
  const double x = a * b;
  double ah, al, bh, bl;
  split(a, &ah, &al);
  split(b, &bh, &bl);
  *e = al * bl - (((x - ah * bh) - al * bh) - ah * bl);
  *p = x;
}

int oracle_dgemm_dot2(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < m; ++i) {
      double s, c;
      two_sum(C[i + (long)j * ldc], 0.0, &s, &c);
      for (int p = 0; p < k; ++p) {
        double h, r, q;
        two_prod(A[i + (long)p * lda], B[p + (long)j * ldb], &h, &r);
        two_sum(s, h, &s, &q);
        c = c + (q + r);
      }
      C[i + (long)j * ldc] = s + c;
    }
  }
  return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
