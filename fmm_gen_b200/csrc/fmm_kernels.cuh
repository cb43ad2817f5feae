// fmm_b200 device code: FP64 DMMA GEMM mainloop with fused operand linear combinations
// and a multi-destination epilogue, plus the elementwise helpers of the AB / NAIVE
// pack types.  sm_100a only.
//
// Mapping of the reference's CPU design (fmm-gen):
//   * BLIS packing with fused sums (meta/abc_gen_mix.py:171-251, packA/B_add_stra_abc<r>)
//     -> cp.async staging of every U/V term tile into thread-private shared-memory
//        slots, summed once per CTA tile into the operand buffer.
//   * AVX 8x4 micro-kernel (common/kernels/bl_dgemm_asm_8x4.c)
//     -> 128x128x16 CTA tile of mma.sync.m16n8k4 FP64 (DMMA) fragments.
//   * multi-destination C update (meta/abc_micro_kernel_gen.py:147-244)
//     -> epilogue C_l += W[l,r] * M_r for every nonzero W of product r, done by the
//        CTA that owns the tile position in all C blocks, so no two CTAs ever touch
//        the same C element (no atomics, deterministic).
//   * M_Add / S_Add / T_Add (meta/ab_gen_mix.py:341-372, meta/naive_gen_mix.py:60-137)
//     -> fmm_scatter_kernel / fmm_lincomb_kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fmm {

constexpr int BM = 128;   // CTA tile rows (m)
constexpr int BN = 128;   // CTA tile columns (n)
constexpr int BK = 16;    // k depth of one staged tile
constexpr int NTHREADS = 256;
constexpr int LDA_S = BM + 4;  // opA[k][m], padded: conflict-free fragment loads
constexpr int LDB_S = BK + 4;  // opB[n][k]
constexpr int NRAW = 4;        // thread-private raw term slots in flight
constexpr int EA = BM * BK / NTHREADS;  // A elements a thread stages per term (8)
constexpr int EB = BN * BK / NTHREADS;  // B elements a thread stages per term (8)
constexpr int OPA_SZ = BK * LDA_S;
constexpr int OPB_SZ = BN * LDB_S;
constexpr int RAW_SZ = (EA + EB) * NTHREADS;
constexpr size_t SMEM_BYTES = (size_t)(2 * OPA_SZ + 2 * OPB_SZ + NRAW * RAW_SZ) * sizeof(double);
constexpr int GROUP_M = 8;     // tile raster: groups of 8 tile rows for L2 reuse

struct Term {
  int row;      // global block row in the composed grid
  int col;      // global block column
  double coef;  // coefficient
};

struct Prod {
  int a0, na;   // A terms: terms[a0 .. a0+na)
  int b0, nb;   // B terms
  int c0, nc;   // C terms
};

enum Mode : int { MODE_ACCUM_C = 0, MODE_STORE_M = 1 };

struct GemmArgs {
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  double* C;      // MODE_ACCUM_C: C blocks receive C_l += w * M_r
  long long ldc;
  double* M;      // MODE_STORE_M: product r stored at M + r * m_stride (ld = ldm)
  long long ldm;
  long long m_stride;
  int ms, ns, ks;   // sub-block sizes
  const Prod* prods;
  const Term* terms;
  int r_begin, r_end;   // products handled (MODE_ACCUM_C: every CTA loops over all of them)
  int tiles_m, tiles_n;
  int mode;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async8(unsigned dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], const double (&a)[2], double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(b));
}

// Position of one load unit = (product, k step, term) in the flattened stream.
struct UnitIter {
  int r, s, t;
  int T;        // max(na, nb) of product r
};

__device__ __forceinline__ int prod_T(const Prod& p) { return p.na > p.nb ? p.na : p.nb; }

// Issue the cp.async copies of one unit: term t of product r at k step s.
__device__ __forceinline__ void issue_unit(const GemmArgs& a, const Prod& p, int s, int t, double* raw_slot,
                                           int m0, int n0, int tid) {
  const unsigned sbase = smem_u32(raw_slot);
  if (t < p.na) {
    const Term tm = a.terms[p.a0 + t];
    const double* base = a.A + (long long)tm.row * a.ms + (long long)tm.col * a.ks * a.lda;
#pragma unroll
    for (int e = 0; e < EA; ++e) {
      const int idx = e * NTHREADS + tid;
      const int mm = idx % BM, kk = idx / BM;
      const int gm = m0 + mm, gk = s * BK + kk;
      const bool v = (gm < a.ms) && (gk < a.ks);
      const double* src = v ? base + gm + (long long)gk * a.lda : a.A;
      cp_async8(sbase + (unsigned)(idx * sizeof(double)), src, v ? 8 : 0);
    }
  }
  if (t < p.nb) {
    const Term tm = a.terms[p.b0 + t];
    const double* base = a.B + (long long)tm.row * a.ks + (long long)tm.col * a.ns * a.ldb;
#pragma unroll
    for (int e = 0; e < EB; ++e) {
      const int idx = e * NTHREADS + tid;
      const int kk = idx % BK, nn = idx / BK;
      const int gk = s * BK + kk, gn = n0 + nn;
      const bool v = (gk < a.ks) && (gn < a.ns);
      const double* src = v ? base + gk + (long long)gn * a.ldb : a.B;
      cp_async8(sbase + (unsigned)((EA * NTHREADS + idx) * sizeof(double)), src, v ? 8 : 0);
    }
  }
}

// Fold one staged term into the operand buffers.  A thread reads back only the
// elements it copied itself, so no barrier is needed between arrival and use.
__device__ __forceinline__ void consume_unit(const GemmArgs& a, const Prod& p, int t, const double* raw_slot,
                                             double* opA, double* opB, int tid) {
  if (t < p.na) {
    const double c = a.terms[p.a0 + t].coef;
#pragma unroll
    for (int e = 0; e < EA; ++e) {
      const int idx = e * NTHREADS + tid;
      const int mm = idx % BM, kk = idx / BM;
      const double v = raw_slot[idx];
      double* dst = opA + kk * LDA_S + mm;
      *dst = (t == 0) ? c * v : fma(c, v, *dst);
    }
  }
  if (t < p.nb) {
    const double c = a.terms[p.b0 + t].coef;
#pragma unroll
    for (int e = 0; e < EB; ++e) {
      const int idx = e * NTHREADS + tid;
      const int kk = idx % BK, nn = idx / BK;
      const double v = raw_slot[EA * NTHREADS + idx];
      double* dst = opB + nn * LDB_S + kk;
      *dst = (t == 0) ? c * v : fma(c, v, *dst);
    }
  }
}

__device__ __forceinline__ void mma_tile(const double* opA, const double* opB, double (&acc)[4][4][4], int wm,
                                         int wn, int g, int t4) {
#pragma unroll
  for (int kq = 0; kq < BK / 4; ++kq) {
    double af[4][2], bf[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = wm * 64 + i * 16 + g;
      af[i][0] = opA[(kq * 4 + t4) * LDA_S + row];
      af[i][1] = opA[(kq * 4 + t4) * LDA_S + row + 8];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = wn * 32 + j * 8 + g;
      bf[j] = opB[col * LDB_S + kq * 4 + t4];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[i][j], af[i], bf[j]);
  }
}

__device__ __forceinline__ void epilogue(const GemmArgs& a, const Prod& p, int r, const double (&acc)[4][4][4],
                                         int m0, int n0, int wm, int wn, int g, int t4) {
  if (a.mode == MODE_STORE_M) {
    double* Mr = a.M + (long long)r * a.m_stride;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int rr = m0 + wm * 64 + i * 16 + g + 8 * h;
            const int cc = n0 + wn * 32 + j * 8 + t4 * 2 + q;
            if (rr < a.ms && cc < a.ns) Mr[rr + (long long)cc * a.ldm] = acc[i][j][2 * h + q];
          }
    return;
  }
  for (int c = 0; c < p.nc; ++c) {
    const Term tm = a.terms[p.c0 + c];
    const double w = tm.coef;
    double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int rr = m0 + wm * 64 + i * 16 + g + 8 * h;
            const int cc = n0 + wn * 32 + j * 8 + t4 * 2 + q;
            if (rr < a.ms && cc < a.ns) {
              double* ptr = Cb + rr + (long long)cc * a.ldc;
              *ptr = fma(w, acc[i][j][2 * h + q], *ptr);
            }
          }
  }
}

// One CTA computes one BMxBN tile position for products [r_begin, r_end) in order
// (MODE_ACCUM_C), or for the single product blockIdx.y + r_begin (MODE_STORE_M).
__global__ void __launch_bounds__(NTHREADS, 1) fmm_gemm_kernel(const GemmArgs a) {
  extern __shared__ __align__(16) double smem[];
  double* opA = smem;                    // [2][OPA_SZ]
  double* opB = smem + 2 * OPA_SZ;       // [2][OPB_SZ]
  double* raw = opB + 2 * OPB_SZ;        // [NRAW][RAW_SZ]

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;

  // Grouped raster over tile positions.
  const int bid = blockIdx.x;
  const int group_rows = GROUP_M;
  const int per_group = group_rows * a.tiles_n;
  const int grp = bid / per_group;
  const int first_m = grp * group_rows;
  const int rows_here = min(a.tiles_m - first_m, group_rows);
  const int in_grp = bid % per_group;
  const int tile_m = first_m + in_grp % rows_here;
  const int tile_n = in_grp / rows_here;
  const int m0 = tile_m * BM, n0 = tile_n * BN;

  int rb = a.r_begin, re = a.r_end;
  if (a.mode == MODE_STORE_M) {
    rb = a.r_begin + blockIdx.y;
    re = rb + 1;
  }
  const int nks = (a.ks + BK - 1) / BK;

  // Issue iterator.
  int ir = rb, is = 0, it = 0;
  Prod ip = a.prods[ir];
  int iT = prod_T(ip);
  bool issuing = true;
  auto advance_issue = [&]() {
    if (++it < iT) return;
    it = 0;
    if (++is < nks) return;
    is = 0;
    if (++ir < re) {
      ip = a.prods[ir];
      iT = prod_T(ip);
    } else {
      issuing = false;
    }
  };

  int unit = 0;
#pragma unroll 1
  for (int i = 0; i < NRAW - 1; ++i) {
    if (issuing) {
      issue_unit(a, ip, is, it, raw + (size_t)((unit + i) % NRAW) * RAW_SZ, m0, n0, tid);
      advance_issue();
    }
    cp_async_commit();
  }

  int kcount = 0;
  double acc[4][4][4];
#pragma unroll 1
  for (int r = rb; r < re; ++r) {
    const Prod p = a.prods[r];
    const int T = prod_T(p);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

#pragma unroll 1
    for (int s = 0; s < nks; ++s) {
      const int buf = kcount & 1;
      double* oa = opA + buf * OPA_SZ;
      double* ob = opB + buf * OPB_SZ;
#pragma unroll 1
      for (int t = 0; t < T; ++t) {
        cp_async_wait<NRAW - 2>();
        consume_unit(a, p, t, raw + (size_t)(unit % NRAW) * RAW_SZ, oa, ob, tid);
        if (issuing) {
          issue_unit(a, ip, is, it, raw + (size_t)((unit + NRAW - 1) % NRAW) * RAW_SZ, m0, n0, tid);
          advance_issue();
        }
        cp_async_commit();
        ++unit;
      }
      __syncthreads();
      mma_tile(oa, ob, acc, wm, wn, g, t4);
      ++kcount;
    }
    epilogue(a, p, r, acc, m0, n0, wm, wn, g, t4);
  }
  cp_async_wait<0>();
}

// S_r / T_r temporaries of the NAIVE pack type: out_r = sum_t coef_t * X_{blk_t}.
// side 0 uses the A terms of each product, side 1 the B terms.
struct LincombArgs {
  const double* X;
  long long ldx;
  int rows, cols;          // sub-block size
  int blk_row_stride;      // rows per block row (ms for A, ks for B)
  int blk_col_stride;      // cols per block column (ks for A, ns for B)
  double* out;
  long long ldo;
  long long out_stride;    // per product
  const Prod* prods;
  const Term* terms;
  int side;
  int r_begin;
};

__global__ void fmm_lincomb_kernel(const LincombArgs a) {
  const int r = a.r_begin + blockIdx.y;
  const Prod p = a.prods[r];
  const int t0 = a.side == 0 ? p.a0 : p.b0;
  const int nt = a.side == 0 ? p.na : p.nb;
  double* out = a.out + (long long)blockIdx.y * a.out_stride;
  const long long total = (long long)a.rows * a.cols;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % a.rows);
    const long long j = e / a.rows;
    double v = 0.0;
    for (int t = 0; t < nt; ++t) {
      const Term tm = a.terms[t0 + t];
      const double x = a.X[(long long)tm.row * a.blk_row_stride + i +
                           ((long long)tm.col * a.blk_col_stride + j) * a.ldx];
      v = (t == 0) ? tm.coef * x : fma(tm.coef, x, v);
    }
    out[i + j * a.ldo] = v;
  }
}

// M_Add: C_l += sum_r W[l, r] * M_r for every C block l, products applied in order r.
struct ScatterArgs {
  double* C;
  long long ldc;
  int ms, ns;
  const double* M;
  long long ldm;
  long long m_stride;
  const int* cblk;          // per C block: row, col, first entry, #entries (4 ints)
  const int* ent_r;         // entries: product index
  const double* ent_w;      // entries: coefficient
};

__global__ void fmm_scatter_kernel(const ScatterArgs a) {
  const int l = blockIdx.y;
  const int row = a.cblk[4 * l + 0], col = a.cblk[4 * l + 1];
  const int e0 = a.cblk[4 * l + 2], ne = a.cblk[4 * l + 3];
  double* Cb = a.C + (long long)row * a.ms + (long long)col * a.ns * a.ldc;
  const long long total = (long long)a.ms * a.ns;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % a.ms);
    const long long j = e / a.ms;
    double c = Cb[i + j * a.ldc];
    for (int q = 0; q < ne; ++q) {
      const double mv = a.M[(long long)a.ent_r[e0 + q] * a.m_stride + i + j * a.ldm];
      c = fma(a.ent_w[e0 + q], mv, c);
    }
    Cb[i + j * a.ldc] = c;
  }
}

}  // namespace fmm
