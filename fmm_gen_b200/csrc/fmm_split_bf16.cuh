// Split-BF16 FMM on sm_100a tensor cores (tcgen05): FP32 inputs, FP64 C, products at
// FP32-level accuracy.  The reference is FP64 only; this path keeps its algebra (products r
// in order, C_l += W[l,r] * M_r, fringes peeled the same way) and changes the arithmetic:
//
//   1. fmm_split_operands_kernel: for every product r the operand sum
//      S_r = sum_i U[i,r] A_i is formed in FP64 from the FP32 inputs and split exactly into
//      three bf16 planes, S = hi + mid + lo (hi = bf16(S), mid = bf16(S - hi),
//      lo = bf16(S - hi - mid)), stored K-major (k contiguous, row pitch kpad, a multiple
//      of 64, zero padded).  Likewise T_r = sum_j V[j,r] B_j.
//   2. fmm_split_gemm_kernel: M_r = S_r T_r as six plane products
//      hi*hi + hi*mid + mid*hi + mid*mid + hi*lo + lo*hi (the dropped ones are ~2^-24
//      relative), tcgen05.mma kind::f16 into FP32 accumulators in tensor memory: hi*hi
//      into one, the five smaller products into another, so that the accumulators' own
//      rounding never drops the small terms against the large ones.  Every 256-deep k
//      chunk is drained with tcgen05.ld (the two accumulators added once in FP32) and
//      added into FP64 registers, so FP32 rounding only acts within a chunk.  With several
//      products the epilogue stores M_r (FP64) to a workspace and fmm_combine_kernel adds
//      W[l,r] * M_r into C afterwards; a single product is added into C directly.
//
// Work unit = (128 x 128 tile position, product r), claimed in order from a launch-wide
// counter (fmm::UnitClaimer); a unit owns its tile position in every C block, and per-tile
// tickets order the products' C updates (no atomics on C, the result does not depend on
// scheduling).  Warp roles (384 threads, one CTA per SM, persistent):
// warp 0 lane 0 issues TMA (128-byte swizzle, each CTA loads its own tiles), warp 1 owns tensor memory and
// its lane 0 issues the MMAs, warps 4..11 drain the accumulator and run the epilogue.
// Every wait is bounded; tensor memory is freed on every path.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fmm_kernels.cuh"

namespace fmms {

using fmm::Prod;
using fmm::Term;

constexpr int BM = 128;        // tile rows (m) = tensor-memory lanes
constexpr int BN = 128;        // tile columns (n) = accumulator columns
constexpr int BK = 64;         // k per stage: 64 bf16 = one 128-byte swizzle row
constexpr int UK = 16;         // k per tcgen05.mma (kind::f16)
constexpr int NPLANE = 3;
constexpr int NPAIR = 6;
constexpr int NSTG = 2;
constexpr int TILE_BYTES = BM * BK * 2;                  // 16 KB: one plane tile
constexpr int STAGE_BYTES = 2 * NPLANE * TILE_BYTES;     // 96 KB: three A planes, three B planes
constexpr int NACC = 2;                                  // chunk buffers in tensor memory: the MMAs run
                                                         // up to NACC chunks ahead of the drain
constexpr int ACC_COLS = 2 * BN;                         // a chunk buffer: hi*hi accumulator, then the
                                                         // accumulator of the five smaller plane products
constexpr int TMEM_COLS = NACC * ACC_COLS;               // 512 columns (all of tensor memory)
constexpr int NTHREADS = 384;
constexpr int NEPI = 256;                                // epilogue threads (warps 4..11)
constexpr int KPAD = 64;                                 // plane row pitch multiple
constexpr int NBARS = 2 * NSTG + 2 * NACC + 1;
constexpr size_t SMEM_BYTES =
    (size_t)NSTG * STAGE_BYTES + 1024 /*alignment slack*/ + 8 * NBARS + 16 /*tensor-memory address*/ + fmm::RING_BYTES;
constexpr int GROUP_M = 8;
constexpr int DRAIN_STAGES = 4;                          // stages (of BK) accumulated in FP32 before each FP64 drain
constexpr int C_PREFETCH_CHUNKS = 4;                     // C tiles go to L2 this many drains before a unit ends
constexpr int C_BATCH = 16;                              // C elements in flight per thread in the epilogue
constexpr int LAUNCH_REGS = 65536 / NTHREADS / 8 * 8;    // 168 with one CTA per SM
constexpr int CTL_REGS = 56;
constexpr int EPI_REGS = 224;
static_assert(128 * CTL_REGS + NEPI * EPI_REGS <= NTHREADS * LAUNCH_REGS, "register split exceeds the launch budget");
static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");

struct SplitGemmArgs {
  CUtensorMap tmA;   // A planes: row (3 r + p) ms + i, column k (pitch kpad); bf16, box 64 x 128, 128-byte swizzle
  CUtensorMap tmB;   // B planes: row (3 r + p) ns + j
  double* C;
  long long ldc;
  int ms, ns, kpad;
  const Prod* prods;  // C terms of product r: terms[c0 .. c0+nc)
  const Term* terms;
  int nprod;
  int tiles_m, tiles_n;
  int* tickets;      // per tile: products whose C updates are done (zeroed before launch)
  double* M;         // when set: product r's tile is stored to M + r * m_stride (ld ldm) instead
  long long ldm;     // of being added into C; a combine pass applies W afterwards
  long long m_stride;
  unsigned* status;
  int* counter;      // work units claimed so far (zeroed before launch)
};

// Where the split kernel's work units come from (for fmm::UnitClaimer).
struct SplitSrc {
  const SplitGemmArgs& a;
  __device__ __forceinline__ int total() const { return a.tiles_m * a.tiles_n * a.nprod; }
  __device__ __forceinline__ unsigned* status() const { return a.status; }
  __device__ __forceinline__ int* counter() const { return a.counter; }
};

// UMMA shared-memory descriptor of a K-major operand tile stored with the 128-byte
// swizzle (rows of 128 bytes, 8-row atoms of 1024 bytes): start address >> 4, leading
// byte offset 16 (unused by this layout), stride byte offset 1024, descriptor version 1,
// layout type 2 (SWIZZLE_128B).  The k offset inside the 128-byte row is added to the
// start address; the hardware applies the swizzle to the full address.
__device__ __forceinline__ uint64_t smem_desc_sw128(unsigned saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)(16 >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// kind::f16 instruction descriptor: D format F32 (bits 4-5 = 1), A and B BF16 (bits 7-9
// and 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t instr_desc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          int accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// The barrier receives one arrive when every tcgen05 operation this thread issued so far
// has completed.
__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's lane (32x32b shape, 16 repeats);
// the caller waits (tmem_wait_ld) before using the values.
__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

using fmm::mbar_wait_drain;  // time-limited wait for copies and MMAs still in flight at the end

// The unit's C tiles (every C block of product p) into L2: 128-byte lines of 16 rows of
// one column, spread over the epilogue threads.
__device__ __forceinline__ void prefetch_c_tiles(const SplitGemmArgs& a, const Prod& p, int m0, int n0, int et) {
  for (int c = 0; c < p.nc; ++c) {
    const Term tm = a.terms[p.c0 + c];
    const double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc;
#pragma unroll
    for (int e = 0; e < (BM / 16) * BN / NEPI; ++e) {
      const int l = et + e * NEPI;
      const int rr = m0 + (l % (BM / 16)) * 16, cc = n0 + l / (BM / 16);
      if (rr < a.ms && cc < a.ns) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(Cb + rr + (long long)cc * a.ldc));
    }
  }
}

struct SUnit {
  int m0, n0, tile, r;
};

// Units in product-major order; tiles rastered in groups of GROUP_M tile rows so that
// concurrent units share operand panels in L2.
__device__ __forceinline__ SUnit s_decode(const SplitGemmArgs& a, int u) {
  const int ntiles = a.tiles_m * a.tiles_n;
  SUnit w;
  w.r = u / ntiles;
  const int bid = u % ntiles;
  const int per_group = GROUP_M * a.tiles_n;
  const int first_m = (bid / per_group) * GROUP_M;
  const int rows_here = min(a.tiles_m - first_m, GROUP_M);
  const int in_grp = bid % per_group;
  w.m0 = (first_m + in_grp % rows_here) * BM;
  w.n0 = (in_grp / rows_here) * BN;
  w.tile = bid;
  return w;
}

__global__ void __launch_bounds__(NTHREADS, 1) fmm_split_gemm_kernel(const __grid_constant__ SplitGemmArgs a) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte alignment for the 128-byte swizzle atoms
  unsigned char* smem = smem_raw + ((1024 - (fmm::smem_u32(smem_raw) & 1023)) & 1023);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + (size_t)NSTG * STAGE_BYTES);
  const unsigned full0 = fmm::smem_u32(bars);                    // [NSTG] stage bytes landed
  const unsigned empty0 = fmm::smem_u32(bars + NSTG);            // [NSTG] MMAs done reading the stage
  const unsigned accf0 = fmm::smem_u32(bars + 2 * NSTG);         // [NACC] chunk accumulated
  const unsigned acce0 = fmm::smem_u32(bars + 2 * NSTG + NACC);  // [NACC] chunk drained
  const unsigned done_bar = fmm::smem_u32(bars + 2 * NSTG + 2 * NACC);  // every MMA complete
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + NBARS);
  const fmm::UnitRing q{fmm::smem_u32(bars + NBARS + 2)};
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nks = a.kpad / BK;

  if (tid == 0) {
    for (int s = 0; s < NSTG; ++s) {
      fmm::mbar_init(full0 + 8 * s, 1);
      fmm::mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < NACC; ++b) {
      fmm::mbar_init(accf0 + 8 * b, 1);
      fmm::mbar_init(acce0 + 8 * b, NEPI / 32);
    }
    fmm::mbar_init(done_bar, 1);
    fmm::unit_ring_init(q, 1 + NEPI / 32);  // ring readers: the MMA thread and the epilogue warps
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(fmm::smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *reinterpret_cast<volatile unsigned*>(tmem_slot);

  if (warp == 0) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(CTL_REGS));
    if (lane == 0) {  // ---- TMA producer; claims the work units ----
      const SplitSrc src{a};
      fmm::UnitClaimer<SplitSrc> nx{src, q};
      long long kc = 0;
      for (int u = nx.next(); u >= 0; u = nx.next()) {
        const SUnit w = s_decode(a, u);
        const int ya = 3 * w.r * a.ms + w.m0, yb = 3 * w.r * a.ns + w.n0;
        for (int s = 0; s < nks; ++s, ++kc) {
          const int stg = (int)(kc % NSTG);
          fmm::mbar_wait(empty0 + 8 * stg, (unsigned)(((kc / NSTG) & 1) ^ 1), a.status);
          const unsigned fb = full0 + 8 * stg;
          fmm::mbar_arrive_expect_tx(fb, (unsigned)STAGE_BYTES);
          const unsigned base = fmm::smem_u32(smem + (size_t)stg * STAGE_BYTES);
#pragma unroll
          for (int pl = 0; pl < NPLANE; ++pl) {
            fmm::tma_load_2d(base + pl * TILE_BYTES, &a.tmA, s * BK, ya + pl * a.ms, fb);
            fmm::tma_load_2d(base + (NPLANE + pl) * TILE_BYTES, &a.tmB, s * BK, yb + pl * a.ns, fb);
          }
        }
      }
      // copies still in flight (only on an error path) land before the CTA exits
      for (long long q = kc - NSTG; q < kc; ++q)
        if (q >= 0) mbar_wait_drain(full0 + 8 * (int)(q % NSTG), (unsigned)((q / NSTG) & 1));
    }
  } else if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(CTL_REGS));
    if (warp == 1 && lane == 0) {  // ---- MMA issuer ----
      constexpr uint32_t idesc = instr_desc_bf16_f32(BM, BN);
      // plane pairs (A plane, B plane); the last, hi*hi, has an accumulator of its own
      constexpr int pa[NPAIR] = {2, 0, 1, 1, 0, 0};
      constexpr int pb[NPAIR] = {0, 2, 1, 0, 1, 0};
      fmm::UnitReader nx{q, a.status, true, 0, true};
      long long kc = 0, ch = 0;
      for (int u = nx.next(); u >= 0; u = nx.next()) {
        for (int s = 0; s < nks; ++s, ++kc) {
          const int stg = (int)(kc % NSTG);
          const int b = (int)(ch % NACC);
          const bool first = s % DRAIN_STAGES == 0, last = s % DRAIN_STAGES == DRAIN_STAGES - 1 || s == nks - 1;
          fmm::mbar_wait(full0 + 8 * stg, (unsigned)((kc / NSTG) & 1), a.status);
          if (first) fmm::mbar_wait(acce0 + 8 * b, (unsigned)(((ch / NACC) & 1) ^ 1), a.status);
          tc_fence_after();
          const unsigned base = fmm::smem_u32(smem + (size_t)stg * STAGE_BYTES);
          const uint64_t dbase = smem_desc_sw128(base);
          const unsigned dt = tmem + (unsigned)(b * ACC_COLS);
#pragma unroll
          for (int q = 0; q < NPAIR; ++q) {
#pragma unroll
            for (int kk = 0; kk < BK / UK; ++kk) {
              const uint64_t ad = dbase + (uint64_t)((pa[q] * TILE_BYTES + kk * UK * 2) >> 4);
              const uint64_t bd = dbase + (uint64_t)(((NPLANE + pb[q]) * TILE_BYTES + kk * UK * 2) >> 4);
              if (q == NPAIR - 1)
                umma_bf16(dt, ad, bd, idesc, !first || kk != 0);
              else
                umma_bf16(dt + BN, ad, bd, idesc, !first || (kk | q) != 0);
            }
          }
          umma_commit(empty0 + 8 * stg);  // stage reusable once these MMAs have read it
          if (last) {
            umma_commit(accf0 + 8 * b);  // chunk ready for the drain
            ++ch;
          }
        }
      }
      umma_commit(done_bar);
      mbar_wait_drain(done_bar, 0u);
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(EPI_REGS));
    // ---- drain + epilogue: lane quarter = warp % 4 (tensor-memory lanes), column half ----
    const int et = tid - 128;
    const int quarter = warp & 3, half = (warp - 4) >> 2;
    const int row = quarter * 32 + lane;
    const bool ordered = a.nprod > 1 && a.M == nullptr;
    fmm::UnitReader nx{q, a.status, true};
    long long ch = 0;
    for (int u = nx.next(); u >= 0; u = nx.next()) {
      const SUnit w = s_decode(a, u);
      double acc[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.0;
      const Prod p = a.prods[w.r];
      const int nch = (nks + DRAIN_STAGES - 1) / DRAIN_STAGES;
      for (int c = 0; c < nch; ++c, ++ch) {
        if (!a.M && c == (nch > C_PREFETCH_CHUNKS ? nch - C_PREFETCH_CHUNKS : 0)) prefetch_c_tiles(a, p, w.m0, w.n0, et);
        const int b = (int)(ch % NACC);
        fmm::mbar_wait(accf0 + 8 * b, (unsigned)((ch / NACC) & 1), a.status);
        tc_fence_after();
        const unsigned taddr = tmem + ((unsigned)(quarter * 32) << 16) + (unsigned)(b * ACC_COLS + half * 64);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          unsigned v[16], e[16];
          tmem_ld16(taddr + 16 * h, v);
          tmem_ld16(taddr + BN + 16 * h, e);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[16 * h + i] += (double)(__uint_as_float(v[i]) + __uint_as_float(e[i]));
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) fmm::mbar_arrive(acce0 + 8 * b);
      }
      if (a.M) {  // store-only epilogue: no loads, so it does not hold up the next drains
        const int rr = w.m0 + row;
        if (rr < a.ms) {
          double* Mr = a.M + (long long)w.r * a.m_stride + rr;
#pragma unroll
          for (int j = 0; j < 64; ++j) {
            const int cc = w.n0 + half * 64 + j;
            if (cc < a.ns) Mr[(long long)cc * a.ldm] = acc[j];
          }
        }
        continue;
      }
      // this tile position's updates from products < r are complete
      if (ordered && w.r > 0) {
        if (et == 0) fmm::ticket_spin(a.tickets + w.tile, w.r, a.status, 256);
        fmm::named_bar_sync(1, NEPI);
      }
      // C_l += W[l, r] * M_r in FP64; a warp's lanes cover 32 consecutive rows of a column
      const int rr = w.m0 + row;
      if (rr < a.ms) {
        for (int c = 0; c < p.nc; ++c) {
          const Term tm = a.terms[p.c0 + c];
          double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc + rr;
#pragma unroll
          for (int j0 = 0; j0 < 64; j0 += C_BATCH) {
            double cv[C_BATCH];
#pragma unroll
            for (int j = 0; j < C_BATCH; ++j) {
              const int cc = w.n0 + half * 64 + j0 + j;
              cv[j] = cc < a.ns ? Cb[(long long)cc * a.ldc] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < C_BATCH; ++j) {
              const int cc = w.n0 + half * 64 + j0 + j;
              if (cc < a.ns) Cb[(long long)cc * a.ldc] = fma(tm.coef, acc[j0 + j], cv[j]);
            }
          }
        }
      }
      if (ordered) {
        __threadfence();
        fmm::named_bar_sync(1, NEPI);
        if (et == 0) fmm::st_release(a.tickets + w.tile, w.r + 1);
      }
    }
  }
  // every role is done with tensor memory before it is freed
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// S_r (side 0) or T_r (side 1) of product r = blockIdx.x, summed in FP64 from FP32 inputs
// and split into three bf16 planes, K-major: plane p of product r holds rows
// (3 r + p) * rows .. + rows, row pitch kpad; columns k in [ks, kpad) are zeros.  A CTA
// makes a 32-row x 64-k tile; products vary fastest in the grid, so the CTAs resident at
// one time read the same input tiles and every input element comes from HBM about once.
//   side 0: X = A (column-major, m x k), plane row i = row of A; the tile is transposed
//           through shared memory so that both the reads and the writes coalesce.
//   side 1: X = B (column-major, k x n), plane row j = column of B (k already contiguous).
struct SplitArgs {
  const float* X;
  long long ldx;
  int rows, ks, kpad;
  int blk_row_stride;       // A: ms (rows per block row), B: ks
  int blk_col_stride;       // A: ks (columns per block column), B: ns
  __nv_bfloat16* out;
  const Prod* prods;
  const Term* terms;
  int side;
};

constexpr int SPLIT_ROWS = 32, SPLIT_K = 64;

__device__ __forceinline__ void split3(double x, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo) {
  hi = __double2bfloat16(x);
  const double r1 = x - (double)__bfloat162float(hi);  // exact: hi is within 2^-9 |x| of x
  mid = __double2bfloat16(r1);
  const double r2 = r1 - (double)__bfloat162float(mid);
  lo = __double2bfloat16(r2);
}

// Planes of two k-adjacent values, stored as bf16 pairs.
__device__ __forceinline__ void store_split_pair(const SplitArgs& a, int r, int row, int kk, double x0, double x1) {
  __nv_bfloat16 h0, m0, l0, h1, m1, l1;
  split3(x0, h0, m0, l0);
  split3(x1, h1, m1, l1);
  const size_t plane = (size_t)a.rows * a.kpad;
  __nv_bfloat162* P = reinterpret_cast<__nv_bfloat162*>(a.out + (size_t)(3 * r) * plane + (size_t)row * a.kpad + kk);
  const size_t step = plane / 2;  // plane size in bf16 pairs (kpad is even)
  P[0] = __halves2bfloat162(h0, h1);
  P[step] = __halves2bfloat162(m0, m1);
  P[2 * step] = __halves2bfloat162(l0, l1);
}

__global__ void __launch_bounds__(256) fmm_split_operands_kernel(const SplitArgs a) {
  const int r = blockIdx.x;
  const Prod p = a.prods[r];
  const int t0 = a.side == 0 ? p.a0 : p.b0;
  const int nt = a.side == 0 ? p.na : p.nb;
  const int k0 = blockIdx.y * SPLIT_K, row0 = blockIdx.z * SPLIT_ROWS;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  if (a.side == 0) {
    __shared__ double tile[SPLIT_K][SPLIT_ROWS + 1];
    const int i = row0 + tx;
    for (int j = ty; j < SPLIT_K; j += 8) {  // a warp reads 32 consecutive rows of one column
      const int kk = k0 + j;
      double v = 0.0;
      if (i < a.rows && kk < a.ks) {
        for (int t = 0; t < nt; ++t) {
          const Term tm = a.terms[t0 + t];
          const float x =
              a.X[(long long)tm.row * a.blk_row_stride + i + ((long long)tm.col * a.blk_col_stride + kk) * a.ldx];
          v = fma(tm.coef, (double)x, v);
        }
      }
      tile[j][tx] = v;
    }
    __syncthreads();
    for (int j = ty; j < SPLIT_ROWS; j += 8) {  // a warp writes 64 consecutive k of one plane row
      if (row0 + j < a.rows) store_split_pair(a, r, row0 + j, k0 + 2 * tx, tile[2 * tx][j], tile[2 * tx + 1][j]);
    }
  } else {
    for (int jj = ty; jj < SPLIT_ROWS; jj += 8) {
      const int j = row0 + jj, kk = k0 + 2 * tx;
      if (j >= a.rows) continue;
      double v0 = 0.0, v1 = 0.0;
      for (int t = 0; t < nt; ++t) {
        const Term tm = a.terms[t0 + t];
        const float* col = a.X + (long long)tm.row * a.blk_row_stride + ((long long)tm.col * a.blk_col_stride + j) * a.ldx;
        if (kk < a.ks) v0 = fma(tm.coef, (double)col[kk], v0);
        if (kk + 1 < a.ks) v1 = fma(tm.coef, (double)col[kk + 1], v1);
      }
      store_split_pair(a, r, j, kk, v0, v1);
    }
  }
}

// Every product's operand sum from one read of the operand: a CTA stages one tile position of
// all the operand's blocks (side 0: 16 rows x 32 k of each A block, side 1: 8 columns x 64 k
// of each B block) in shared memory in the output orientation (row, k), then makes all R
// products' sums of that tile in FP64 in term order (the same arithmetic as
// fmm_split_operands_kernel, so the planes are bit-identical) and stores their three bf16
// planes.  Each input element is read from HBM once and no CTA waits on a global load per
// term: the per-product kernel read each block once per product that uses it.
//   tables (shared memory): per product its first term and term count; per term its block
//   (row * block_cols + col of the operand's block grid) and coefficient.
template <int SIDE>
struct SplitAllShape;
template <>
struct SplitAllShape<0> {  // A: 16 rows x 32 k, loads coalesced along rows
  static constexpr int TR = 16, TK = 32;
};
template <>
struct SplitAllShape<1> {  // B: 8 columns x 64 k, loads coalesced along k
  static constexpr int TR = 8, TK = 64;
};

struct SplitAllArgs {
  SplitArgs s;
  int nblk, block_cols;  // the operand's block grid: nblk blocks, block_cols per block row
  int nprod;
  int nterm;             // sum of the products' term counts on this side
};

__host__ __device__ constexpr size_t split_all_smem_bytes(int side, int nblk, int nprod, int nterm) {
  return sizeof(float) * (size_t)nblk * (side == 0 ? 16 * 33 : 8 * 65) + sizeof(int) * (2 * (size_t)nprod + nterm) +
         sizeof(double) * (size_t)nterm + 16;
}

template <int SIDE>
__global__ void __launch_bounds__(256) fmm_split_all_kernel(const SplitAllArgs g) {
  constexpr int TR = SplitAllShape<SIDE>::TR, TK = SplitAllShape<SIDE>::TK, LD = TK + 1;
  const SplitArgs& a = g.s;
  extern __shared__ __align__(16) double sall[];
  double* tcoef = sall;                                      // [nterm]
  int* tblk = reinterpret_cast<int*>(tcoef + g.nterm);       // [nterm]
  int* tfirst = tblk + g.nterm;                              // [nprod]
  int* tcount = tfirst + g.nprod;                            // [nprod]
  float* x = reinterpret_cast<float*>(tcount + g.nprod);     // [nblk][TR][LD]
  const int tid = threadIdx.x;
  // tables: term counts in parallel, offsets by one thread (shared memory only), terms in parallel
  for (int r = tid; r < g.nprod; r += blockDim.x) {
    const Prod p = a.prods[r];
    tcount[r] = SIDE == 0 ? p.na : p.nb;
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int r = 0; r < g.nprod; ++r) {
      tfirst[r] = acc;
      acc += tcount[r];
    }
  }
  __syncthreads();
  for (int r = tid; r < g.nprod; r += blockDim.x) {
    const Prod p = a.prods[r];
    const int t0 = SIDE == 0 ? p.a0 : p.b0, nt = tcount[r], f = tfirst[r];
    for (int t = 0; t < nt; ++t) {
      const Term tm = a.terms[t0 + t];
      tcoef[f + t] = tm.coef;
      tblk[f + t] = tm.row * g.block_cols + tm.col;
    }
  }
  const int row0 = blockIdx.y * TR, k0 = blockIdx.x * TK;
  // stage every block's tile, output orientation x[b][row][k]; zeros outside the block
  for (int b = 0; b < g.nblk; ++b) {
    const int br = b / g.block_cols, bc = b % g.block_cols;
    float* xb = x + (size_t)b * TR * LD;
    if (SIDE == 0) {  // A[(br ms + i) + (bc ks + k) lda]: lanes along i
      const int i = tid % TR;
#pragma unroll
      for (int kk = tid / TR; kk < TK; kk += 256 / TR) {
        const int row = row0 + i, k = k0 + kk;
        xb[i * LD + kk] = (row < a.rows && k < a.ks)
                              ? a.X[(long long)br * a.blk_row_stride + row + ((long long)bc * a.blk_col_stride + k) * a.ldx]
                              : 0.0f;
      }
    } else {  // B[(br ks + k) + (bc ns + j) ldb]: lanes along k
      const int kk = tid % TK;
#pragma unroll
      for (int j = tid / TK; j < TR; j += 256 / TK) {
        const int row = row0 + j, k = k0 + kk;
        xb[j * LD + kk] = (row < a.rows && k < a.ks)
                              ? a.X[(long long)br * a.blk_row_stride + k + ((long long)bc * a.blk_col_stride + row) * a.ldx]
                              : 0.0f;
      }
    }
  }
  __syncthreads();
  // one k pair per thread: rows TR x TK / 2 pairs = 256
  const int row = tid / (TK / 2), kk = 2 * (tid % (TK / 2));
  if (row0 + row >= a.rows) return;
  const float* xr = x + row * LD + kk;
  for (int r = 0; r < g.nprod; ++r) {
    double v0 = 0.0, v1 = 0.0;
    const int f = tfirst[r], nt = tcount[r];
    for (int t = 0; t < nt; ++t) {
      const float* xp = xr + (size_t)tblk[f + t] * TR * LD;
      const double w = tcoef[f + t];
      v0 = fma(w, (double)xp[0], v0);
      v1 = fma(w, (double)xp[1], v1);
    }
    store_split_pair(a, r, row0 + row, k0 + kk, v0, v1);
  }
}

}  // namespace fmms
