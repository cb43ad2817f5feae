// fmm_b200 device code: a persistent, warp-specialised FP64 DMMA GEMM whose producer
// warpgroup forms the U/V linear combinations of A and B sub-blocks while staging them
// into shared memory, and whose consumer warpgroups scatter each product into every C
// block with a nonzero W coefficient; plus the elementwise kernels of the AB / NAIVE
// pack types.  sm_100a only.
//
// Mapping of the reference's CPU design (fmm-gen):
//   * BLIS packing with fused sums (meta/abc_gen_mix.py:171-251, packA/B_add_stra_abc<r>)
//     -> producer warpgroup: cp.async of every U/V term tile into thread-private
//        shared-memory slots, folded into the operand stage (sum with coefficients),
//        released to the consumers with an mbarrier.
//   * AVX 8x4 micro-kernel (common/kernels/bl_dgemm_asm_8x4.c)
//     -> 128x128 CTA tile of mma.sync.m16n8k4 FP64 (DMMA) fragments, 8 consumer warps
//        with 64x32 warp tiles.
//   * multi-destination C update (meta/abc_micro_kernel_gen.py:147-244)
//     -> epilogue C_l += W[l,r] * M_r for every nonzero W of product r.  A work unit
//        owns one tile position in all C blocks for a range of products; when products
//        are split over several units, tickets per tile (or, in the direct variant with
//        few tile positions, per tile and C block) order the units' C updates (bounded
//        spin, error flag on timeout), so no two CTAs ever update the same C element at
//        once and every element receives its products in order r = 0..R-1.
//   * M_Add / S_Add / T_Add (meta/ab_gen_mix.py:341-372, meta/naive_gen_mix.py:60-137)
//     -> fmm_lincomb_kernel / fmm_lincomb_batch_kernel (operand sums formed in HBM, also
//        used by the ABC pack type for large sub-blocks), fmm_combine_staged_kernel and
//        fmm_combine_kernel (every C_l += W[l,r] M_r of the stored products in one pass, the
//        C blocks in groups that share products, running values in registers; the staged
//        form brings the M tiles in by bulk copies), fmm_scatter_kernel (one C block per
//        launch row, beyond the combine's tables).
//   * The direct variant (fmm_gemm_direct_kernel) runs when every operand is a single
//     aligned term (pre-summed operands): a deeper TMA pipeline and an epilogue on the
//     producer warps that overlaps the next product's DMMA.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace fmm {

constexpr int BM = 128;   // CTA tile rows (m)
constexpr int BN = 128;   // CTA tile columns (n)
constexpr int BK = 8;     // k depth of one operand stage
constexpr int NPROD = 256;               // producer threads (warpgroups 0, 1)
constexpr int NCONS = 256;               // consumer threads (warpgroups 2, 3)
constexpr int NTHREADS = NPROD + NCONS;  // 512
constexpr int LAUNCH_REGS = 65536 / NTHREADS;  // registers per thread at launch (128)
// Operand stages are dense: opA[k][m] (BK x BM) and opB[n][k] (BN x BK), exactly the
// layout a TMA box writes, so single-term operands are copied straight into a stage.
// (The consumers' FP64 fragment loads then see 4-way bank conflicts; shared-memory
// bandwidth has room for that: measured no loss against padded rows.)
constexpr int LDA_S = BM;      // opA[k][m]
constexpr int LDB_S = BK;      // opB[n][k]
constexpr int NSTAGE = 6;      // operand stages (producer -> consumers)
constexpr int NRAW = 6;        // cp.async path: thread-private raw term slots in flight
constexpr int EA = BM * BK / NPROD;  // A elements a producer thread stages per term (8)
constexpr int EB = BN * BK / NPROD;  // B elements a producer thread stages per term (8)
constexpr int OPA_SZ = BK * LDA_S;
constexpr int OPB_SZ = BN * LDB_S;
constexpr int STAGE_SZ = OPA_SZ + OPB_SZ;
constexpr int RAW_SZ = (EA + EB) * NPROD;
// TMA staging: one raw slot holds an A term box (BK x BM, m contiguous) and a B term box
// (BN columns of BK + 2 k values, k contiguous; two wider so that a box can start at the
// even k coordinate at or below an odd one).
constexpr int TB_K = BK + 2;
constexpr int TRAW_A = BK * BM;
constexpr int TRAW_SZ = TRAW_A + BN * TB_K;
constexpr int NRAW_TMA = 6;
constexpr int NFOLD = NPROD - 32;  // folding threads: producer warps 1..7 (warp 0 issues TMA)
constexpr int FPAIRS = (BM * BK / 2 + NFOLD - 1) / NFOLD;  // A element pairs per folding thread
constexpr int FELEMS = (BN * BK + NFOLD - 1) / NFOLD;      // B elements per folding thread
constexpr unsigned TMA_BYTES_A = TRAW_A * sizeof(double);
constexpr unsigned TMA_BYTES_B = BN * TB_K * sizeof(double);   // raw B box (k rounded down to even)
constexpr unsigned TMA_BYTES_B8 = BN * BK * sizeof(double);    // direct B box
static_assert((NSTAGE * STAGE_SZ * sizeof(double)) % 128 == 0, "raw slots must start 128-byte aligned");
static_assert((TRAW_SZ * sizeof(double)) % 128 == 0, "TMA raw slots must be 128-byte aligned");
static_assert((TRAW_A * sizeof(double)) % 128 == 0, "TMA B box must be 128-byte aligned");
constexpr int UQ_DEPTH = 16;  // work-unit ring entries (see UnitClaimer)
constexpr size_t RING_BYTES = 2 * UQ_DEPTH * sizeof(unsigned long long) + UQ_DEPTH * sizeof(int);
constexpr size_t SMEM_BYTES_CPASYNC = (size_t)(NSTAGE * STAGE_SZ + NRAW * RAW_SZ) * sizeof(double) +
                                      (2 * NSTAGE + 2 * NRAW_TMA) * sizeof(unsigned long long) + RING_BYTES;
// What the folding warps need to know about a raw slot, written by the issuer before
// the slot's TMA copies (published by the release of its arrive.expect_tx).
struct SlotMeta {
  double ca, cb;  // coefficients of the staged A and B terms
  int shift;      // B box starts one k before the term's first k
  int pad[3];
};
constexpr size_t SMEM_BYTES_TMA = (size_t)(NSTAGE * STAGE_SZ + NRAW_TMA * TRAW_SZ) * sizeof(double) +
                                  NRAW_TMA * sizeof(SlotMeta) +
                                  (2 * NSTAGE + 2 * NRAW_TMA) * sizeof(unsigned long long) + RING_BYTES;
constexpr size_t smem_bytes(bool tma) { return tma ? SMEM_BYTES_TMA : SMEM_BYTES_CPASYNC; }
constexpr int GROUP_M = 8;  // tile raster: groups of 8 tile rows for L2 reuse
constexpr int C_BATCH_J = 4;          // epilogue: 8-column groups per batch of C loads (4 elements each);
                                      // 4 (16 loads in flight per thread) measured 1-8 % faster than 2
constexpr int C_PREFETCH_STEPS = 24;  // k steps before a product's end at which its C tiles are prefetched
                                      // (at its first k step when it has fewer)
constexpr int PROD_REGS = 72;
constexpr int CONS_REGS = 184;
static_assert(NPROD * PROD_REGS + NCONS * CONS_REGS <= NTHREADS * LAUNCH_REGS,
              "register split exceeds the launch budget");
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ULL;  // bounded device-side waits give up after 4 s
// try_wait suspends the waiting thread until the phase completes or this many ns pass,
// so waiting warps do not take issue slots from the warps they wait for.
constexpr unsigned MBAR_SUSPEND_NS = 20000;

struct Term {
  int row;      // global block row in the composed grid
  int col;      // global block column
  double coef;  // coefficient
  int src;      // A/B terms: 0 = the operand matrix, 1 = the pre-summed workspace (S / T)
  int pad;      // C terms: this product's position among the products with a term in the
                // same C block (product order); the per-block tickets count up to it
};

struct Prod {
  int a0, na;   // A terms: terms[a0 .. a0+na)
  int b0, nb;   // B terms
  int c0, nc;   // C terms
};

enum Mode : int { MODE_ACCUM_C = 0, MODE_STORE_M = 1 };

// STATUS_TICKET_TIMEOUT: a wait for another CTA's C updates gave up (the kernel finishes,
// without the product order from then on); STATUS_WAIT_TIMEOUT: a wait inside a CTA's own
// pipeline gave up (every later wait returns at once and the kernel winds down).
// STATUS_TABLE: a kernel found an index outside its tables (clamped; the result is void)
enum StatusBits : unsigned { STATUS_TICKET_TIMEOUT = 1u, STATUS_WAIT_TIMEOUT = 2u, STATUS_TABLE = 4u };

// Time limit of the bounded device-side waits in ns: WAIT_LIMIT_NS unless a test lowers it
// (fmm_debug_set); read only on a wait's slow path.
__device__ unsigned long long g_wait_limit_ns = WAIT_LIMIT_NS;
__device__ __forceinline__ unsigned long long wait_limit_ns() {
  return *reinterpret_cast<volatile unsigned long long*>(&g_wait_limit_ns);
}

struct GemmArgs {
  CUtensorMap tmA;   // whole-matrix tensor maps (TMA path), FP64: A (m x k), box BM x BK
  CUtensorMap tmB;   // B (k x n), box BK x BN (direct loads)
  CUtensorMap tmB2;  // B (k x n), box (BK + 2) x BN (raw loads at even k)
  CUtensorMap tmAw;  // the same three for the pre-summed workspaces S (A side) and T (B side)
  CUtensorMap tmBw;
  CUtensorMap tmBw2;
  CUtensorMap tmA64;   // A and S again with a box of BM / 2 rows: the half-height units of the
  CUtensorMap tmAw64;  // direct variant (see Unit)
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  const double* Aw;  // pre-summed operands: S holds one ms x ks block per slot (block column),
  long long ldaw;    // T one ks x ns block per slot (block column); terms with src = 1 point here
  const double* Bw;
  long long ldbw;
  double* C;      // MODE_ACCUM_C: C blocks receive C_l += w * M_r
  long long ldc;
  double* M;      // MODE_STORE_M: product r stored at M + r * m_stride (ld = ldm)
  long long ldm;
  long long m_stride;
  int ms, ns, ks;   // sub-block sizes
  const Prod* prods;
  const Term* terms;
  int nprod;        // products [0, nprod)
  int tiles_m, tiles_n;
  int chunks;       // products are split into `chunks` consecutive ranges per tile
  int mode;
  int* tickets;     // per tile (nbt = 0): chunks completed; zeroed before launch; used when chunks > 1
  unsigned* status; // device status word (StatusBits)
  int nbt;          // > 0 (direct variant, one product per unit): tickets per (tile, C block),
  int nbc;          // nbt = C blocks, index tile * nbt + row * nbc + col, counting the block's
                    // updates in product order; 0: one ticket per tile
  int* counter;     // work units claimed so far in this launch (zeroed before launch)
  int bm;           // tile height: BM, or BM / 2 (direct variant only); 0 means BM
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async8(unsigned dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async16(unsigned dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(bar),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n}\n" ::"r"(bar)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(MBAR_SUSPEND_NS)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity.  Every phase is completed by another
// role of the same CTA, so in a correct run the wait ends; if it has not after the wait
// limit, the status word gets STATUS_WAIT_TIMEOUT and every later such wait of every CTA
// returns at once, so the kernel still finishes and the host reports FMM_E_TIMEOUT.  A
// ticket timeout alone (STATUS_TICKET_TIMEOUT) does not cut these waits short: the
// pipeline keeps running and every issued copy is consumed before the kernel ends.
__device__ __forceinline__ void mbar_wait(unsigned bar, unsigned parity, unsigned* status) {
  if (mbar_try_wait(bar, parity)) return;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if ((*(volatile unsigned*)status & STATUS_WAIT_TIMEOUT) != 0u) return;
    if (global_ns() - t0 > wait_limit_ns()) {
      atomicOr(status, STATUS_WAIT_TIMEOUT);
      return;
    }
  }
}

// Wait for a phase with a time limit only (no early exit on the status word): used at the
// end of a role for copies that may still be in flight (only on an error path, where
// other roles stopped consuming; in a normal run these phases have long completed).
__device__ __forceinline__ void mbar_wait_drain(unsigned bar, unsigned parity) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > wait_limit_ns()) return;
  }
}

__device__ __forceinline__ void named_bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait for a ticket written by another CTA: until *p >= target.  On timeout the
// status word gets STATUS_TICKET_TIMEOUT; once any status bit is set, ticket waits return
// at once.
__device__ __forceinline__ void ticket_spin(const int* p, int target, unsigned* status, unsigned sleep_ns) {
  if (ld_acquire(p) >= target) return;
  const unsigned long long t0 = global_ns();
  while (ld_acquire(p) < target) {
    if (*(volatile unsigned*)status != 0u) return;
    if (global_ns() - t0 > wait_limit_ns()) {
      atomicOr(status, STATUS_TICKET_TIMEOUT);
      return;
    }
    __nanosleep(sleep_ns);
  }
}

__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], const double (&a)[2], double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(b));
}

__device__ __forceinline__ int prod_T(const Prod& p) { return p.na > p.nb ? p.na : p.nb; }

// Work unit u -> (tile position, product range).  Chunk-major order: the units of one tile
// are a whole tile grid apart, so a later chunk is claimed well after the earlier one.
// unit_rows: the tile's rows inside the block (at most the tile height).  unit_half: the tile
// has at most BM / 2 rows (a job of half-height tiles, or the last tile row of a block whose
// height leaves <= 64 rows there); the direct variant then stages a BM / 2-row box of A and
// lets both rows of consumer warps cover those rows, each taking half of the column fragments
// (every element still gets a full tile's DMMAs in the same order).
struct Unit {
  int m0, n0, tile, r0, r1;
};

__device__ __forceinline__ int tile_height(const GemmArgs& a) { return a.bm > 0 ? a.bm : BM; }
// rows of the unit's tile inside the block, and whether that makes it a half-height unit
__device__ __forceinline__ int unit_rows(const GemmArgs& a, const Unit& w) { return min(tile_height(a), a.ms - w.m0); }
__device__ __forceinline__ bool unit_half(const GemmArgs& a, const Unit& w) { return unit_rows(a, w) <= BM / 2; }

// VARH: the job's tile height may be BM / 2 (direct variant); the other kernels use BM, known
// at compile time.
template <bool VARH = false>
__device__ __forceinline__ Unit decode_unit(const GemmArgs& a, int u) {
  const int ntiles = a.tiles_m * a.tiles_n;
  Unit w;
  int c, bid;
  if (a.mode == MODE_STORE_M) {
    c = u / ntiles;  // one product per unit
    bid = u % ntiles;
    w.r0 = c;
    w.r1 = c + 1;
  } else {
    c = u / ntiles;
    bid = u % ntiles;
    w.r0 = (int)((long long)a.nprod * c / a.chunks);
    w.r1 = (int)((long long)a.nprod * (c + 1) / a.chunks);
  }
  const int per_group = GROUP_M * a.tiles_n;
  const int grp = bid / per_group;
  const int first_m = grp * GROUP_M;
  const int rows_here = min(a.tiles_m - first_m, GROUP_M);
  const int in_grp = bid % per_group;
  const int tile_m = first_m + in_grp % rows_here;
  const int tile_n = in_grp / rows_here;
  w.m0 = tile_m * (VARH ? tile_height(a) : BM);
  w.n0 = tile_n * BN;
  w.tile = bid;
  return w;
}

__device__ __forceinline__ int num_units(const GemmArgs& a) {
  const int ntiles = a.tiles_m * a.tiles_n;
  return ntiles * (a.mode == MODE_STORE_M ? a.nprod : a.chunks);
}

// ------------------------------------------------------------------------------------
// Work-unit claims.  One thread of each CTA (the operand issuer) claims the launch's units
// in increasing order from a launch-wide counter and publishes each claimed index through
// a shared-memory ring; every other role of the CTA reads the ring in the same order
// (index -1 ends the sequence).  A unit waits only on tickets of lower-numbered units,
// which running CTAs claimed before it, so the launch makes progress whether or not all of
// its CTAs are resident at once (another kernel may hold some SMs).
//
// Ring depth: the issuer runs at most one operand pipeline (<= 6 stages of at least one
// unit each) plus the product-tile hand-off ahead of the slowest reader, so 16 entries never
// make it wait; if they did, the wait would end as the readers move on.
// ------------------------------------------------------------------------------------
struct UnitRing {
  unsigned base;  // shared address: UQ_DEPTH full barriers (entry published: 1 arrival, the
                  // claimer), UQ_DEPTH empty barriers (entry read by every reader warp), then
                  // UQ_DEPTH int entries
  __device__ __forceinline__ unsigned full(int s) const { return base + 8 * s; }
  __device__ __forceinline__ unsigned empty(int s) const { return base + 8 * (UQ_DEPTH + s); }
  __device__ __forceinline__ unsigned entry(int s) const { return base + 16 * UQ_DEPTH + 4 * s; }
};

__device__ __forceinline__ void st_shared_s32(unsigned addr, int v) {
  asm volatile("st.shared.s32 [%0], %1;\n" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_shared_s32(unsigned addr) {
  int v;
  asm volatile("ld.shared.s32 %0, [%1];\n" : "=r"(v) : "r"(addr) : "memory");
  return v;
}

// The claiming thread: next unit index of this CTA, or -1 when the launch has none left.
template <class Src>
struct UnitClaimer {
  const Src& src;
  UnitRing q;
  int n = 0;
  __device__ __forceinline__ int next() {
    const int slot = n % UQ_DEPTH;
    mbar_wait(q.empty(slot), (unsigned)(((n / UQ_DEPTH) & 1) ^ 1), src.status());
    int u = -1;
    if ((*(volatile unsigned*)src.status() & STATUS_WAIT_TIMEOUT) == 0u) {
      u = atomicAdd(src.counter(), 1);
      if (u >= src.total()) u = -1;
    }
    st_shared_s32(q.entry(slot), u);
    mbar_arrive(q.full(slot));  // release: the entry is visible to the readers' acquire
    ++n;
    return u;
  }
};

// A reader warp (all 32 lanes call next() together), or a lone thread (lone = true) whose
// warp has no other active lanes.  release = false reads an entry without freeing it (a
// second cursor of the same warp frees it later).
struct UnitReader {
  UnitRing q;
  unsigned* status;
  bool release;
  int n = 0;
  bool lone = false;
  __device__ __forceinline__ int next() {
    const int slot = n % UQ_DEPTH;
    mbar_wait(q.full(slot), (unsigned)((n / UQ_DEPTH) & 1), status);
    int u = ld_shared_s32(q.entry(slot));
    if ((*(volatile unsigned*)status & STATUS_WAIT_TIMEOUT) != 0u) u = -1;
    if (release) {
      if (lone) {
        mbar_arrive(q.empty(slot));
      } else {
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(q.empty(slot));
      }
    }
    ++n;
    return u;
  }
};

// Warp 0 of the per-thread-copy producer: lane 0 claims, the warp shares the index.
template <class Src>
struct WarpClaimer {
  UnitClaimer<Src> c;
  __device__ __forceinline__ int next() {
    int u = 0;
    if ((threadIdx.x & 31) == 0) u = c.next();
    return __shfl_sync(0xffffffffu, u, 0);
  }
};

__device__ __forceinline__ void unit_ring_init(const UnitRing& q, unsigned readers) {
  for (int s = 0; s < UQ_DEPTH; ++s) {
    mbar_init(q.full(s), 1);
    mbar_init(q.empty(s), readers);
  }
}

// ------------------------------------------------------------------------------------
// Producer: flattened stream of load units (k step s, term t) over the CTA's work units.
// ------------------------------------------------------------------------------------
struct LoadIter {
  int u;            // work unit index (global over the launch)
  int j;            // problem of the unit (0 for a single-problem launch)
  int nks;          // k steps per product of that problem
  Unit w;
  int r;            // product
  Prod p;
  int T;
  int s, t;
  bool valid;
  // term t of product r, fetched when the iterator moves so that the global loads are
  // off the producer's critical path
  Term ta, tb;
};

// Where a launch's work units come from.  OneJob: one problem, the kernel parameter (its
// fields stay in the parameter space).  JobBatch: many problems in global memory, problem
// j owning the units [unit_start[j], unit_start[j + 1]).
struct OneJob {
  const GemmArgs& a;
  __device__ __forceinline__ const GemmArgs& get(int) const { return a; }
  __device__ __forceinline__ int find(int) const { return 0; }
  __device__ __forceinline__ int first_unit(int) const { return 0; }
  __device__ __forceinline__ int total() const { return num_units(a); }
  __device__ __forceinline__ unsigned* status() const { return a.status; }
  __device__ __forceinline__ int* counter() const { return a.counter; }
  __device__ __forceinline__ void acquire_maps(int) const {}
};

struct JobBatch {
  const GemmArgs* jobs;
  const int* unit_start;
  int njobs, units;
  unsigned* st;
  int* ctr;
  __device__ __forceinline__ const GemmArgs& get(int j) const { return jobs[j]; }
  __device__ __forceinline__ int find(int u) const {  // last j with unit_start[j] <= u
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(unit_start + mid) <= u)
        lo = mid;
      else
        hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ int first_unit(int j) const { return __ldg(unit_start + j); }
  __device__ __forceinline__ int total() const { return units; }
  __device__ __forceinline__ unsigned* status() const { return st; }
  __device__ __forceinline__ int* counter() const { return ctr; }
  // The tensor maps were written into global memory by a copy before the launch; order
  // that write before the tensor-map proxy reads them.
  __device__ __forceinline__ void acquire_maps(int j) const {
    const CUtensorMap* m = &jobs[j].tmA;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(m + q) : "memory");
  }
};

__device__ __forceinline__ void load_terms(const GemmArgs& a, LoadIter& it) {
  if (it.t < it.p.na) it.ta = a.terms[it.p.a0 + it.t];
  if (it.t < it.p.nb) it.tb = a.terms[it.p.b0 + it.t];
}

template <bool VARH = false, class Src>
__device__ __forceinline__ void iter_enter_unit(const Src& src, LoadIter& it) {
  it.j = src.find(it.u);
  const GemmArgs& a = src.get(it.j);
  it.nks = (a.ks + BK - 1) / BK;
  it.w = decode_unit<VARH>(a, it.u - src.first_unit(it.j));
  it.r = it.w.r0;
  it.p = a.prods[it.r];
  it.T = prod_T(it.p);
  it.s = 0;
  it.t = 0;
  load_terms(a, it);
}

template <bool VARH = false, class Src, class Nx>
__device__ __forceinline__ void load_iter_start(const Src& src, LoadIter& it, Nx& nx) {
  it.u = nx.next();
  it.valid = it.u >= 0;
  if (it.valid) iter_enter_unit<VARH>(src, it);
}

template <class Src, class Nx>
__device__ __forceinline__ void load_iter_next(const Src& src, LoadIter& it, Nx& nx) {
  const GemmArgs& a = src.get(it.j);
  if (++it.t < it.T) {
    load_terms(a, it);
    return;
  }
  it.t = 0;
  if (++it.s < it.nks) {
    if (it.T > 1) load_terms(a, it);
    return;
  }
  it.s = 0;
  if (++it.r < it.w.r1) {
    it.p = a.prods[it.r];
    it.T = prod_T(it.p);
    load_terms(a, it);
    return;
  }
  it.u = nx.next();
  if (it.u < 0) {
    it.valid = false;
    return;
  }
  iter_enter_unit(src, it);
}

// Raw slot layout (thread-private, conflict-free): pair e of A at [e][pt] (16 B each),
// then the B pairs.  A term tile: 128 (m) x 8 (k) = 512 m-pairs, 4 per thread; B term
// tile: 8 (k) x 128 (n) = 512 k-pairs, 4 per thread.
constexpr int PA = EA / 2;  // A pairs per thread per term
constexpr int PB = EB / 2;

__device__ __forceinline__ void issue_unit(const GemmArgs& a, const LoadIter& it, double* raw_slot, int pt) {
  const unsigned sbase = smem_u32(raw_slot);
  if (it.t < it.p.na) {
    const double* M0 = it.ta.src ? a.Aw : a.A;
    const long long ld = it.ta.src ? a.ldaw : a.lda;
    const long long off = (long long)it.ta.row * a.ms + (long long)it.ta.col * a.ks * ld;
    const double* base = M0 + off;
    const bool al16 = ((off & 1) == 0) && ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(M0) & 15) == 0);
#pragma unroll
    for (int e = 0; e < PA; ++e) {
      const int q = e * NPROD + pt;        // pair index
      const int mm = 2 * (q % (BM / 2)), kk = q / (BM / 2);
      const int gm = it.w.m0 + mm, gk = it.s * BK + kk;
      const unsigned dst = sbase + (unsigned)(q * 16);
      if (al16) {
        const int nb = (gk < a.ks) ? ((gm + 1 < a.ms) ? 16 : (gm < a.ms ? 8 : 0)) : 0;
        cp_async16(dst, nb ? base + gm + (long long)gk * ld : M0, nb);
      } else {
        const bool v0 = (gk < a.ks) && (gm < a.ms), v1 = (gk < a.ks) && (gm + 1 < a.ms);
        cp_async8(dst, v0 ? base + gm + (long long)gk * ld : M0, v0 ? 8 : 0);
        cp_async8(dst + 8, v1 ? base + gm + 1 + (long long)gk * ld : M0, v1 ? 8 : 0);
      }
    }
  }
  if (it.t < it.p.nb) {
    const double* M0 = it.tb.src ? a.Bw : a.B;
    const long long ld = it.tb.src ? a.ldbw : a.ldb;
    const long long off = (long long)it.tb.row * a.ks + (long long)it.tb.col * a.ns * ld;
    const double* base = M0 + off;
    const bool al16 = ((off & 1) == 0) && ((ld & 1) == 0) && ((reinterpret_cast<uintptr_t>(M0) & 15) == 0);
#pragma unroll
    for (int e = 0; e < PB; ++e) {
      const int q = e * NPROD + pt;
      const int kk = 2 * (q % (BK / 2)), nn = q / (BK / 2);
      const int gk = it.s * BK + kk, gn = it.w.n0 + nn;
      const unsigned dst = sbase + (unsigned)((PA * NPROD + q) * 16);
      if (al16) {
        const int nb = (gn < a.ns) ? ((gk + 1 < a.ks) ? 16 : (gk < a.ks ? 8 : 0)) : 0;
        cp_async16(dst, nb ? base + gk + (long long)gn * ld : M0, nb);
      } else {
        const bool v0 = (gn < a.ns) && (gk < a.ks), v1 = (gn < a.ns) && (gk + 1 < a.ks);
        cp_async8(dst, v0 ? base + gk + (long long)gn * ld : M0, v0 ? 8 : 0);
        cp_async8(dst + 8, v1 ? base + gk + 1 + (long long)gn * ld : M0, v1 ? 8 : 0);
      }
    }
  }
}

// Fold one staged term into the operand stage.  A producer thread reads back only the
// elements it copied itself, so no barrier is needed between arrival and use; the
// stage itself belongs to the producer between its empty and full barrier phases.
__device__ __forceinline__ void fold_unit(const LoadIter& it, const double* raw_slot, double* opA, double* opB,
                                          int pt) {
  if (it.t < it.p.na) {
    const double c = it.ta.coef;
#pragma unroll
    for (int e = 0; e < PA; ++e) {
      const int q = e * NPROD + pt;
      const int mm = 2 * (q % (BM / 2)), kk = q / (BM / 2);
      const double2 v = reinterpret_cast<const double2*>(raw_slot)[q];
      double2* dst = reinterpret_cast<double2*>(opA + kk * LDA_S + mm);
      if (it.t == 0) {
        *dst = make_double2(c * v.x, c * v.y);
      } else {
        const double2 o = *dst;
        *dst = make_double2(fma(c, v.x, o.x), fma(c, v.y, o.y));
      }
    }
  }
  if (it.t < it.p.nb) {
    const double c = it.tb.coef;
#pragma unroll
    for (int e = 0; e < PB; ++e) {
      const int q = e * NPROD + pt;
      const int kk = 2 * (q % (BK / 2)), nn = q / (BK / 2);
      const double2 v = reinterpret_cast<const double2*>(raw_slot)[PA * NPROD + q];
      double2* dst = reinterpret_cast<double2*>(opB + nn * LDB_S + kk);
      if (it.t == 0) {
        *dst = make_double2(c * v.x, c * v.y);
      } else {
        const double2 o = *dst;
        *dst = make_double2(fma(c, v.x, o.x), fma(c, v.y, o.y));
      }
    }
  }
}

// The per-thread-copy producer's cursor that runs ahead (issuing copies): warp 0 claims the
// units, the other producer warps read the ring without freeing entries; the trailing
// cursor (folding) frees them.
template <class Src>
struct IssueCursor {
  WarpClaimer<Src> c;
  UnitReader r;
  bool claim;  // warp-uniform
  __device__ __forceinline__ int next() { return claim ? c.next() : r.next(); }
};

template <class Src>
__device__ __forceinline__ void producer(const Src& src, double* stages, double* raw, unsigned full0, unsigned empty0,
                                         int pt, const UnitRing& q) {
  IssueCursor<Src> inx{WarpClaimer<Src>{UnitClaimer<Src>{src, q}}, UnitReader{q, src.status(), false}, pt < 32};
  UnitReader cnx{q, src.status(), true};
  LoadIter iss, con;
  load_iter_start(src, iss, inx);
  load_iter_start(src, con, cnx);
  // prologue: NRAW - 1 load units in flight
#pragma unroll 1
  for (int i = 0; i < NRAW - 1; ++i) {
    if (iss.valid) {
      issue_unit(src.get(iss.j), iss, raw + (size_t)(i % NRAW) * RAW_SZ, pt);
      load_iter_next(src, iss, inx);
    }
    cp_async_commit();
  }
  long long kc = 0;  // operand stages filled so far
  int unit = 0;
#pragma unroll 1
  while (con.valid) {
    const int stage = (int)(kc % NSTAGE);
    double* opA = stages + (size_t)stage * STAGE_SZ;
    double* opB = opA + OPA_SZ;
    if (con.t == 0) mbar_wait(empty0 + 8 * stage, (unsigned)(((kc / NSTAGE) & 1) ^ 1), src.status());
    cp_async_wait<NRAW - 2>();
    fold_unit(con, raw + (size_t)(unit % NRAW) * RAW_SZ, opA, opB, pt);
    const bool last_term = (con.t == con.T - 1);
    if (iss.valid) {
      issue_unit(src.get(iss.j), iss, raw + (size_t)((unit + NRAW - 1) % NRAW) * RAW_SZ, pt);
      load_iter_next(src, iss, inx);
    }
    cp_async_commit();
    ++unit;
    if (last_term) {
      __syncwarp();
      if ((pt & 31) == 0) mbar_arrive(full0 + 8 * stage);
      ++kc;
    }
    load_iter_next(src, con, cnx);
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------------------------------
// TMA producer.  Warp 0, lane 0 is the issuer: per k step it copies single-term
// operands (coefficient 1, full k step, aligned) straight into the operand stage and
// every term of a summed operand into a raw slot.  Warps 1..7 fold the raw slots of a
// k step into registers (sum with coefficients, k tail masked) and store the result
// into the stage once.  The stage's full barrier completes on the issuer's arrival
// with its byte count plus one arrival per folding warp.
// ------------------------------------------------------------------------------------
struct KStep {
  bool dirA, dirB;  // operand copied straight into the stage
  int T;            // raw loads for the summed operands
};

__device__ __forceinline__ KStep kstep_info(const GemmArgs& a, const LoadIter& it) {
  KStep k;
  const bool whole = (it.s + 1) * BK <= a.ks;
  k.dirA = whole && it.p.na == 1 && it.ta.coef == 1.0;
  k.dirB = whole && it.p.nb == 1 && it.tb.coef == 1.0 && ((it.tb.row * a.ks) & 1) == 0;
  const int tA = k.dirA ? 0 : it.p.na, tB = k.dirB ? 0 : it.p.nb;
  k.T = tA > tB ? tA : tB;
  return k;
}

// Per-k-step iterator over (unit, product, k step); ta / tb hold the first A / B term.
template <bool VARH = false, class Src, class Nx>
__device__ __forceinline__ void kiter_next(const Src& src, LoadIter& it, Nx& nx) {
  it.t = 0;
  if (++it.s < it.nks) return;
  it.s = 0;
  const GemmArgs& a = src.get(it.j);
  if (++it.r < it.w.r1) {
    it.p = a.prods[it.r];
    it.T = prod_T(it.p);
    load_terms(a, it);
    return;
  }
  it.u = nx.next();
  if (it.u < 0) {
    it.valid = false;
    return;
  }
  iter_enter_unit<VARH>(src, it);
}

template <class Src>
__device__ __forceinline__ void tma_issuer(const Src& src, double* stages, double* raw, SlotMeta* meta, unsigned full0,
                                           unsigned empty0, unsigned rfull0, unsigned rempty0, const UnitRing& q) {
  UnitClaimer<Src> nx{src, q};
  LoadIter it;
  load_iter_start(src, it, nx);
  long long kc = 0, rc = 0;
  int mapped = -1;  // problem whose tensor maps were last acquired
#pragma unroll 1
  while (it.valid) {
    const GemmArgs& a = src.get(it.j);
    if (it.j != mapped) {
      src.acquire_maps(it.j);
      mapped = it.j;
    }
    const int stage = (int)(kc % NSTAGE);
    double* opA = stages + (size_t)stage * STAGE_SZ;
    const KStep ks = kstep_info(a, it);
    const int k0 = it.s * BK;
    mbar_wait(empty0 + 8 * stage, (unsigned)(((kc / NSTAGE) & 1) ^ 1), src.status());
    const unsigned fb = full0 + 8 * stage;
    mbar_arrive_expect_tx(fb, (ks.dirA ? TMA_BYTES_A : 0u) + (ks.dirB ? TMA_BYTES_B8 : 0u));
    if (ks.dirA)
      tma_load_2d(smem_u32(opA), it.ta.src ? &a.tmAw : &a.tmA, it.ta.row * a.ms + it.w.m0, it.ta.col * a.ks + k0,
                  fb);
    if (ks.dirB)
      tma_load_2d(smem_u32(opA + OPA_SZ), it.tb.src ? &a.tmBw : &a.tmB, it.tb.row * a.ks + k0,
                  it.tb.col * a.ns + it.w.n0, fb);
#pragma unroll 1
    for (int t = 0; t < ks.T; ++t, ++rc) {
      const int slot = (int)(rc % NRAW_TMA);
      if (rc >= NRAW_TMA) mbar_wait(rempty0 + 8 * slot, (unsigned)(((rc / NRAW_TMA) - 1) & 1), src.status());
      const bool hasA = !ks.dirA && t < it.p.na, hasB = !ks.dirB && t < it.p.nb;
      const unsigned rb = rfull0 + 8 * slot;
      double* rs = raw + (size_t)slot * TRAW_SZ;
      const Term tA = hasA ? (t == 0 ? it.ta : a.terms[it.p.a0 + t]) : Term{0, 0, 0.0, 0, 0};
      const Term tB = hasB ? (t == 0 ? it.tb : a.terms[it.p.b0 + t]) : Term{0, 0, 0.0, 0, 0};
      const int xk = tB.row * a.ks + k0;  // B box k coordinate, rounded down to even: TMA needs 16-byte x
      meta[slot].ca = tA.coef;
      meta[slot].cb = tB.coef;
      meta[slot].shift = xk & 1;
      mbar_arrive_expect_tx(rb, (hasA ? TMA_BYTES_A : 0u) + (hasB ? TMA_BYTES_B : 0u));
      if (hasA)
        tma_load_2d(smem_u32(rs), tA.src ? &a.tmAw : &a.tmA, tA.row * a.ms + it.w.m0, tA.col * a.ks + k0, rb);
      if (hasB) tma_load_2d(smem_u32(rs + TRAW_A), tB.src ? &a.tmBw2 : &a.tmB2, xk & ~1, tB.col * a.ns + it.w.n0, rb);
    }
    ++kc;
    kiter_next(src, it, nx);
  }
  // raw-slot copies still in flight (only on an error path) land before the CTA exits
  for (long long q = rc - NRAW_TMA; q < rc; ++q)
    if (q >= 0) mbar_wait_drain(rfull0 + 8 * (int)(q % NRAW_TMA), (unsigned)((q / NRAW_TMA) & 1));
}

// One raw slot folded into the running sums.  A: element pairs along m (16-byte
// loads, conflict-free); B: single elements with consecutive k per lane, which spreads
// the 80-byte box columns over all banks.  The k tail of a sub-block (k >= ks) only
// exists on a product's last k step and is masked there.
template <bool TAIL>
__device__ __forceinline__ void fold_slot(const double* rs, const SlotMeta& m, bool hasA, bool hasB, bool first,
                                          double2 (&accA)[FPAIRS], double (&accB)[FELEMS], int ft, int kvalid) {
  if (hasA) {
    const double c = m.ca;
#pragma unroll
    for (int e = 0; e < FPAIRS; ++e) {
      const int q = ft + e * NFOLD;
      if (q < BM * BK / 2) {
        const int mm = 2 * (q % (BM / 2)), kk = q / (BM / 2);
        double2 v = reinterpret_cast<const double2*>(rs)[(kk * BM + mm) / 2];
        if (TAIL && kk >= kvalid) v = make_double2(0.0, 0.0);
        accA[e] = first ? make_double2(c * v.x, c * v.y) : make_double2(fma(c, v.x, accA[e].x), fma(c, v.y, accA[e].y));
      }
    }
  }
  if (hasB) {
    const double c = m.cb;
    const double* rb = rs + TRAW_A + m.shift;
#pragma unroll
    for (int e = 0; e < FELEMS; ++e) {
      const int q = ft + e * NFOLD;
      if (q < BN * BK) {
        const int kk = q % BK, nn = q / BK;
        double v = rb[nn * TB_K + kk];
        if (TAIL && kk >= kvalid) v = 0.0;
        accB[e] = first ? c * v : fma(c, v, accB[e]);
      }
    }
  }
}

template <class Src>
__device__ __forceinline__ void tma_folder(const Src& src, double* stages, const double* raw, const SlotMeta* meta,
                                           unsigned full0, unsigned empty0, unsigned rfull0, unsigned rempty0, int ft,
                                           const UnitRing& q) {
  UnitReader nx{q, src.status(), true};
  LoadIter it;
  load_iter_start(src, it, nx);
  long long kc = 0, rc = 0;
  const int lane = ft & 31;
#pragma unroll 1
  while (it.valid) {
    const GemmArgs& a = src.get(it.j);
    const int stage = (int)(kc % NSTAGE);
    double* opA = stages + (size_t)stage * STAGE_SZ;
    double* opB = opA + OPA_SZ;
    const KStep ks = kstep_info(a, it);
    const int kvalid = a.ks - it.s * BK;  // valid k values in this step (>= BK except at the tail)
    // Every folding warp waits for the stage to be released before it arrives on the
    // stage's full barrier, even when it has nothing to fold: an arrival made earlier
    // could land in the barrier's previous phase (whose issuer arrival and bytes may
    // still be outstanding) and break that phase's transaction accounting.
    mbar_wait(empty0 + 8 * stage, (unsigned)(((kc / NSTAGE) & 1) ^ 1), src.status());
    if (ks.T > 0) {
      double2 accA[FPAIRS];
      double accB[FELEMS];
#pragma unroll 1
      for (int t = 0; t < ks.T; ++t, ++rc) {
        const int slot = (int)(rc % NRAW_TMA);
        mbar_wait(rfull0 + 8 * slot, (unsigned)((rc / NRAW_TMA) & 1), src.status());
        const double* rs = raw + (size_t)slot * TRAW_SZ;
        const bool hasA = !ks.dirA && t < it.p.na, hasB = !ks.dirB && t < it.p.nb;
        if (kvalid >= BK)
          fold_slot<false>(rs, meta[slot], hasA, hasB, t == 0, accA, accB, ft, kvalid);
        else
          fold_slot<true>(rs, meta[slot], hasA, hasB, t == 0, accA, accB, ft, kvalid);
        __threadfence_block();  // raw-slot loads complete before the slot can be refilled
        __syncwarp();
        if (lane == 0) mbar_arrive(rempty0 + 8 * slot);
      }
      if (!ks.dirA) {
#pragma unroll
        for (int e = 0; e < FPAIRS; ++e) {
          const int q = ft + e * NFOLD;
          if (q < BM * BK / 2) {
            const int mm = 2 * (q % (BM / 2)), kk = q / (BM / 2);
            *reinterpret_cast<double2*>(opA + kk * LDA_S + mm) = accA[e];
          }
        }
      }
      if (!ks.dirB) {
#pragma unroll
        for (int e = 0; e < FELEMS; ++e) {
          const int q = ft + e * NFOLD;
          if (q < BN * BK) opB[(q / BK) * LDB_S + q % BK] = accB[e];
        }
      }
      // The stage is written here through the generic proxy and later refilled by TMA
      // (async proxy): order these stores before any later async-proxy access to it.
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(full0 + 8 * stage);
    ++kc;
    kiter_next(src, it, nx);
  }
}

// ------------------------------------------------------------------------------------
// Consumers: DMMA over the stages, then the multi-destination epilogue.
//
// Consumer warp (wm, wn) owns tile rows wm*64 + 16i + 0..15 and tile columns
// frag_col(wn, j) + 0..7 for fragments i, j = 0..3.  The columns are interleaved (warp wn
// owns wn*8 + 32j) so that a tile cut short by the block edge still spreads its column
// fragments over all four warps of a row half; with the warp-to-scheduler mapping (warp
// % 4, i.e. wn) every SM sub-partition then skips about the same share of an edge tile.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int frag_col(int wn, int j) { return wn * 8 + j * 32; }

// Fragments of warp (wm, wn) that hold rows < vr and columns < vc of the tile: i < im, j < jn.
__device__ __forceinline__ void frag_counts(int vr, int vc, int wm, int wn, int& im, int& jn) {
  const int rrem = vr - wm * 64, crem = vc - wn * 8;
  im = rrem <= 0 ? 0 : min(4, (rrem + 15) >> 4);
  jn = crem <= 0 ? 0 : min(4, (crem + 31) >> 5);
}

// One operand stage into the fragments i < IM, j < JN of the accumulator (IM = JN = 4:
// the whole 64 x 32 warp tile; fewer for the warps of an edge tile, whose other
// fragments stay as they were and are never written out).  Compile-time counts keep each
// form straight-line code: shared-memory loads and DMMAs with no predicates.
// jb: first column fragment (the half-height form gives each row of warps two of the four).
template <int IM, int JN, int LDA = LDA_S>
__device__ __forceinline__ void mma_stage_t(const double* opA, const double* opB, double (&acc)[4][4][4], int wm,
                                            int wn, int g, int t4, int jb = 0) {
#pragma unroll
  for (int kq = 0; kq < BK / 4; ++kq) {
    double af[4][2], bf[4];
#pragma unroll
    for (int i = 0; i < IM; ++i) {
      const int row = wm * 64 + i * 16 + g;
      af[i][0] = opA[(kq * 4 + t4) * LDA + row];
      af[i][1] = opA[(kq * 4 + t4) * LDA + row + 8];
    }
#pragma unroll
    for (int j = 0; j < JN; ++j) bf[j] = opB[(frag_col(wn, jb + j) + g) * LDB_S + kq * 4 + t4];
#pragma unroll
    for (int i = 0; i < IM; ++i)
#pragma unroll
      for (int j = 0; j < JN; ++j) dmma_16x8x4(acc[i][j], af[i], bf[j]);
  }
}

template <int IM_, int JN_>
struct Frags {
  static constexpr int IM = IM_, JN = JN_;
};

// Calls f(Frags<IM, JN>{}) with IM >= im, JN >= jn, so that a k loop written once is
// compiled for the edge shapes: full tiles (4, 4), bottom-edge (1..3, 4), right-edge
// (4, 1..3) and idle warps (0, 0); a corner takes the cheaper of its two edge forms.
// Extra fragments are harmless, and eight forms instead of all seventeen keep the
// consumer code small: on B200 the full set cost 1.5 % on short-k shapes.
template <class F>
__device__ __forceinline__ void with_frags(int im, int jn, F&& f) {
  if (im == 4 && jn == 4) {
    f(Frags<4, 4>{});
    return;
  }
  if (im <= 0 || jn <= 0) {
    f(Frags<0, 0>{});
    return;
  }
  if (jn < 4 && (im == 4 || jn < im)) {
    switch (jn) {
      case 1: f(Frags<4, 1>{}); break;
      case 2: f(Frags<4, 2>{}); break;
      default: f(Frags<4, 3>{}); break;
    }
    return;
  }
  switch (im) {
    case 1: f(Frags<1, 4>{}); break;
    case 2: f(Frags<2, 4>{}); break;
    case 3: f(Frags<3, 4>{}); break;
    default: f(Frags<4, 4>{}); break;
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
            const int cc = n0 + frag_col(wn, j) + t4 * 2 + q;
            if (rr < a.ms && cc < a.ns) Mr[rr + (long long)cc * a.ldm] = acc[i][j][2 * h + q];
          }
    return;
  }
  // C_l += w * M_r, 4 * C_BATCH_J elements at a time: all loads of a batch are issued before
  // any store, so a batch costs one memory round trip instead of one per element.
#pragma unroll 1
  for (int c = 0; c < p.nc; ++c) {
    const Term tm = a.terms[p.c0 + c];
    const double w = tm.coef;
    double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jb = 0; jb < 4; jb += C_BATCH_J) {
        double cv[C_BATCH_J][4];
#pragma unroll
        for (int j = 0; j < C_BATCH_J; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int rr = m0 + wm * 64 + i * 16 + g + 8 * h;
              const int cc = n0 + frag_col(wn, jb + j) + t4 * 2 + q;
              cv[j][2 * h + q] = (rr < a.ms && cc < a.ns) ? Cb[rr + (long long)cc * a.ldc] : 0.0;
            }
#pragma unroll
        for (int j = 0; j < C_BATCH_J; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int rr = m0 + wm * 64 + i * 16 + g + 8 * h;
              const int cc = n0 + frag_col(wn, jb + j) + t4 * 2 + q;
              if (rr < a.ms && cc < a.ns)
                Cb[rr + (long long)cc * a.ldc] = fma(w, acc[i][jb + j][2 * h + q], cv[j][2 * h + q]);
            }
      }
  }
}

// Pull the C tiles an epilogue will update into L2 while the product's last k steps run.
__device__ __forceinline__ void prefetch_c_tiles(const GemmArgs& a, const Prod& p, int m0, int n0, int ct) {
  if (a.mode != MODE_ACCUM_C) return;
  for (int c = 0; c < p.nc; ++c) {
    const Term tm = a.terms[p.c0 + c];
    const double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc;
#pragma unroll
    for (int e = 0; e < (BN * BM / 16) / NCONS; ++e) {  // 128-byte lines: 16 rows of one column
      const int l = ct + e * NCONS;
      const int rr = m0 + (l % (BM / 16)) * 16, cc = n0 + l / (BM / 16);
      if (rr < a.ms && cc < a.ns)
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(Cb + rr + (long long)cc * a.ldc));
    }
  }
}

// Wait until the previous product chunk of this tile has finished its C updates.
__device__ __forceinline__ void ticket_wait(const GemmArgs& a, int tile, int chunk, int ct) {
  if (ct == 0) ticket_spin(a.tickets + tile, chunk, a.status, 256);
  named_bar_sync(1, NCONS);
}

__device__ __forceinline__ void ticket_release(const GemmArgs& a, int tile, int chunk, int ct) {
  __threadfence();
  named_bar_sync(1, NCONS);
  if (ct == 0) st_release(a.tickets + tile, chunk + 1);
}

template <class Src>
__device__ __forceinline__ void consumer(const Src& src, const double* stages, unsigned full0, unsigned empty0,
                                         int ct, const UnitRing& q) {
  const int warp = ct >> 5, lane = ct & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  UnitReader nx{q, src.status(), true};
  long long kc = 0;
  double acc[4][4][4];
#pragma unroll 1
  for (int u = nx.next(); u >= 0; u = nx.next()) {
    const int job = src.find(u);
    const GemmArgs& a = src.get(job);
    const int ul = u - src.first_unit(job);
    const int ntiles = a.tiles_m * a.tiles_n;
    const bool ordered = (a.mode == MODE_ACCUM_C) && a.chunks > 1;
    const int nks = (a.ks + BK - 1) / BK;
    const Unit w = decode_unit(a, ul);
    const int chunk = ul / ntiles;
#pragma unroll 1
    for (int r = w.r0; r < w.r1; ++r) {
      const Prod p = a.prods[r];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
#pragma unroll 1
      for (int s = 0; s < nks; ++s) {
        const int stage = (int)(kc % NSTAGE);
        const double* opA = stages + (size_t)stage * STAGE_SZ;
        const double* opB = opA + OPA_SZ;
        mbar_wait(full0 + 8 * stage, (unsigned)((kc / NSTAGE) & 1), src.status());
        if (s == (nks > C_PREFETCH_STEPS ? nks - C_PREFETCH_STEPS : 0)) prefetch_c_tiles(a, p, w.m0, w.n0, ct);
        mma_stage_t<4, 4>(opA, opB, acc, wm, wn, g, t4);
        // The stage is refilled by TMA as soon as every warp has arrived; the fence
        // makes this warp's shared-memory fragment loads complete before its arrival
        // (measured: without it a refill could overwrite fragments still in flight).
        __threadfence_block();
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * stage);
        ++kc;
      }
      if (ordered && r == w.r0) ticket_wait(a, w.tile, chunk, ct);
      epilogue(a, p, r, acc, w.m0, w.n0, wm, wn, g, t4);
    }
    if (ordered) ticket_release(a, w.tile, chunk, ct);
  }
}

// Persistent: one CTA per SM takes work units in claim order (UnitClaimer) until none is left.
// TMA = true stages operands with tensor copies (A, B 16-byte aligned, even leading
// dimensions); TMA = false with per-thread cp.async (any alignment).
template <bool TMA, class Src>
__device__ __forceinline__ void gemm_cta(const Src& src) {
  extern __shared__ __align__(128) double smem[];
  double* stages = smem;                                  // [NSTAGE][STAGE_SZ]
  double* raw = stages + (size_t)NSTAGE * STAGE_SZ;       // [NRAW][RAW_SZ] or [NRAW_TMA][TRAW_SZ]
  SlotMeta* meta = reinterpret_cast<SlotMeta*>(raw + (TMA ? (size_t)NRAW_TMA * TRAW_SZ : (size_t)NRAW * RAW_SZ));
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(meta + (TMA ? NRAW_TMA : 0));
  const unsigned full0 = smem_u32(bars);
  const unsigned empty0 = smem_u32(bars + NSTAGE);
  const unsigned rfull0 = smem_u32(bars + 2 * NSTAGE);
  const unsigned rempty0 = smem_u32(bars + 2 * NSTAGE + NRAW_TMA);
  const UnitRing q{smem_u32(bars + 2 * NSTAGE + 2 * NRAW_TMA)};
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      // full: TMA path = issuer (1) + folding warps; cp.async path = the 4 producer warps
      mbar_init(full0 + 8 * s, TMA ? 1 + NFOLD / 32 : NPROD / 32);
      mbar_init(empty0 + 8 * s, NCONS / 32);
    }
    if (TMA) {
      for (int s = 0; s < NRAW_TMA; ++s) {
        mbar_init(rfull0 + 8 * s, 1);
        mbar_init(rempty0 + 8 * s, NFOLD / 32);
      }
    }
    // ring readers: folding + consumer warps (TMA); every producer and consumer warp (cp.async)
    unit_ring_init(q, TMA ? (NFOLD + NCONS) / 32 : (NPROD + NCONS) / 32);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid < NPROD) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(PROD_REGS));
    if (TMA) {
      if (tid == 0)
        tma_issuer(src, stages, raw, meta, full0, empty0, rfull0, rempty0, q);
      else if (tid >= 32)
        tma_folder(src, stages, raw, meta, full0, empty0, rfull0, rempty0, tid - 32, q);
    } else {
      producer(src, stages, raw, full0, empty0, tid, q);
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(CONS_REGS));
    consumer(src, stages, full0, empty0, tid - NPROD, q);
  }
}

template <bool TMA>
__global__ void __launch_bounds__(NTHREADS, 1) fmm_gemm_kernel(const __grid_constant__ GemmArgs a) {
  gemm_cta<TMA>(OneJob{a});
}

// Many independent problems (each with its own plan tables, operands, sizes, tensor maps
// and tickets) in one persistent launch: the units of all problems form one sequence,
// problem j owning [unit_start[j], unit_start[j + 1]).
struct BatchArgs {
  const GemmArgs* jobs;    // global memory, 64-byte aligned (tensor maps inside)
  const int* unit_start;   // njobs + 1 entries
  int njobs;
  int units;
  unsigned* status;
  int* counter;            // work units claimed so far (zeroed before launch)
};

template <bool TMA>
__global__ void __launch_bounds__(NTHREADS, 1) fmm_gemm_batch_kernel(const BatchArgs b) {
  gemm_cta<TMA>(JobBatch{b.jobs, b.unit_start, b.njobs, b.units, b.status, b.counter});
}

// ------------------------------------------------------------------------------------
// Direct variant: every operand of every product is one unit-coefficient block staged by
// TMA straight into the stage (the pre-summed ABC path and the classical plan) and ks is a
// multiple of BK, so no term is folded.  The seven folding warps then run the
// multi-destination C epilogue instead: the consumers write each finished product tile
// into shared memory (one 128 x 128 FP64 buffer, in place of the raw slots and two of the
// stages) and go straight on with the next product, while warps 1..7 add W[l,r] * M_r into
// the C blocks from it.  The epilogue overlaps the DMMAs of the next product.
// ------------------------------------------------------------------------------------
constexpr int NSTAGE_D = 4;
constexpr int MS_LD = BM + 1;  // product tile in shared memory: column-major, padded
constexpr int NEPI_D = NFOLD;  // epilogue threads (warps 1..7)
static_assert((size_t)(NSTAGE_D * STAGE_SZ + BN * (BM + 1)) * sizeof(double) + 80 <= 232448, "direct variant shared memory");
constexpr size_t SMEM_BYTES_DIRECT = (size_t)(NSTAGE_D * STAGE_SZ + BN * MS_LD) * sizeof(double) +
                                     (2 * NSTAGE_D + 2) * sizeof(unsigned long long) + RING_BYTES;

template <class Src>
__device__ __forceinline__ void direct_issuer(const Src& src, double* stages, unsigned full0, unsigned empty0,
                                              const UnitRing& q) {
  UnitClaimer<Src> nx{src, q};
  LoadIter it;
  load_iter_start<true>(src, it, nx);
  long long kc = 0;
  int mapped = -1;
#pragma unroll 1
  while (it.valid) {
    const GemmArgs& a = src.get(it.j);
    if (it.j != mapped) {
      src.acquire_maps(it.j);
      mapped = it.j;
    }
    const int stage = (int)(kc % NSTAGE_D);
    double* opA = stages + (size_t)stage * STAGE_SZ;
    const int k0 = it.s * BK;
    mbar_wait(empty0 + 8 * stage, (unsigned)(((kc / NSTAGE_D) & 1) ^ 1), src.status());
    const unsigned fb = full0 + 8 * stage;
    const bool half = unit_half(a, it.w);  // half-height unit: a BM / 2-row A box, dense [k][BM / 2]
    mbar_arrive_expect_tx(fb, (half ? TMA_BYTES_A / 2 : TMA_BYTES_A) + TMA_BYTES_B8);
    const CUtensorMap* ma = it.ta.src ? (half ? &a.tmAw64 : &a.tmAw) : (half ? &a.tmA64 : &a.tmA);
    tma_load_2d(smem_u32(opA), ma, it.ta.row * a.ms + it.w.m0, it.ta.col * a.ks + k0, fb);
    tma_load_2d(smem_u32(opA + OPA_SZ), it.tb.src ? &a.tmBw : &a.tmB, it.tb.row * a.ks + k0,
                it.tb.col * a.ns + it.w.n0, fb);
    ++kc;
    kiter_next<true>(src, it, nx);
  }
  // copies still in flight (only on an error path) land before the CTA exits
  for (long long q = kc - NSTAGE_D; q < kc; ++q)
    if (q >= 0) mbar_wait_drain(full0 + 8 * (int)(q % NSTAGE_D), (unsigned)((q / NSTAGE_D) & 1));
}

template <class Src>
__device__ __forceinline__ void direct_consumer(const Src& src, const double* stages, double* Ms, unsigned full0,
                                                unsigned empty0, unsigned mfull, unsigned mempty, int ct,
                                                const UnitRing& uq) {
  const int warp = ct >> 5, lane = ct & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  UnitReader nx{uq, src.status(), true};
  long long kc = 0, q = 0;
  double acc[4][4][4];
#pragma unroll 1
  for (int u = nx.next(); u >= 0; u = nx.next()) {
    const int job = src.find(u);
    const GemmArgs& a = src.get(job);
    const int nks = (a.ks + BK - 1) / BK;
    const Unit w = decode_unit<true>(a, u - src.first_unit(job));
    const bool half = unit_half(a, w);
    int im, jn;
    frag_counts(a.ms - w.m0, a.ns - w.n0, wm, wn, im, jn);
#pragma unroll 1
    for (int r = w.r0; r < w.r1; ++r, ++q) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
      if (half) {
        // both rows of warps on the tile's BM / 2 rows, warp row wm taking the column
        // fragments 2 wm, 2 wm + 1 of its warp column: each element gets the DMMAs of a full
        // tile in the same order (results equal a full tile's bit for bit), in half the time
#pragma unroll 1
        for (int s = 0; s < nks; ++s, ++kc) {
          const int stage = (int)(kc % NSTAGE_D);
          const double* opA = stages + (size_t)stage * STAGE_SZ;
          mbar_wait(full0 + 8 * stage, (unsigned)((kc / NSTAGE_D) & 1), src.status());
          mma_stage_t<4, 2, BM / 2>(opA, opA + OPA_SZ, acc, 0, wn, g, t4, 2 * wm);
          __threadfence_block();
          __syncwarp();
          if (lane == 0) mbar_arrive(empty0 + 8 * stage);
        }
      } else {
        with_frags(im, jn, [&](auto fr) {
          using FR = decltype(fr);
#pragma unroll 1
          for (int s = 0; s < nks; ++s, ++kc) {
            const int stage = (int)(kc % NSTAGE_D);
            const double* opA = stages + (size_t)stage * STAGE_SZ;
            mbar_wait(full0 + 8 * stage, (unsigned)((kc / NSTAGE_D) & 1), src.status());
            mma_stage_t<FR::IM, FR::JN>(opA, opA + OPA_SZ, acc, wm, wn, g, t4);
            __threadfence_block();  // fragment loads complete before the stage can be refilled
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * stage);
          }
        });
      }
      // hand the product tile to the epilogue warps once they are done with the previous one
      mbar_wait(mempty, (unsigned)((q & 1) ^ 1), src.status());
      if (half) {  // rows 0..63, this warp's two column fragments
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
              for (int e = 0; e < 2; ++e)
                Ms[(frag_col(wn, 2 * wm + j) + t4 * 2 + e) * MS_LD + i * 16 + g + 8 * h] = acc[i][j][2 * h + e];
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int rr = wm * 64 + i * 16 + g + 8 * h;
                const int cc = frag_col(wn, j) + t4 * 2 + e;
                Ms[cc * MS_LD + rr] = acc[i][j][2 * h + e];
              }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(mfull);
    }
  }
}

template <class Src>
__device__ __forceinline__ void direct_epilogue(const Src& src, const double* Ms, unsigned mfull, unsigned mempty,
                                                int et, const UnitRing& uq) {
  const int ew = et >> 5, lane = et & 31;
  constexpr int NW = NEPI_D / 32;  // 7 warps
  UnitReader nx{uq, src.status(), true};
  long long q = 0;
#pragma unroll 1
  for (int u = nx.next(); u >= 0; u = nx.next()) {
    const int job = src.find(u);
    const GemmArgs& a = src.get(job);
    const int ul = u - src.first_unit(job);
    const int ntiles = a.tiles_m * a.tiles_n;
    const bool ordered = (a.mode == MODE_ACCUM_C) && a.chunks > 1;
    const Unit w = decode_unit<true>(a, ul);
    const int rows = unit_rows(a, w);
    const int chunk = ul / ntiles;
#pragma unroll 1
    for (int r = w.r0; r < w.r1; ++r, ++q) {
      const Prod p = a.prods[r];
      // the unit's C tiles into L2 while its product is still being computed
      for (int c = 0; a.mode == MODE_ACCUM_C && c < p.nc; ++c) {
        const Term tm = a.terms[p.c0 + c];
        const double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc;
        for (int l = et; l < (BM / 16) * BN; l += NEPI_D) {
          const int ri = (l % (BM / 16)) * 16, cc = w.n0 + l / (BM / 16);
          if (ri < rows && cc < a.ns)
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(Cb + w.m0 + ri + (long long)cc * a.ldc));
        }
      }
      mbar_wait(mfull, (unsigned)(q & 1), src.status());
      if (a.mode == MODE_STORE_M) {  // the product tile to its workspace (the AB pack type)
        double* Mr = a.M + (long long)r * a.m_stride + w.m0 + lane;
        const int rmax = rows - lane;
#pragma unroll 1
        for (int col = ew; col < BN; col += NW) {
          if (w.n0 + col >= a.ns) continue;
          double* mp = Mr + (long long)(w.n0 + col) * a.ldm;
#pragma unroll
          for (int ch = 0; ch < 4; ++ch)
            if (ch * 32 < rmax) mp[ch * 32] = Ms[col * MS_LD + lane + ch * 32];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(mempty);
        continue;
      }
      const bool per_block = ordered && a.nbt > 0;
      if (ordered && !per_block && r == w.r0) {
        if (et == 0) ticket_spin(a.tickets + w.tile, chunk, a.status, 256);
        named_bar_sync(2, NEPI_D);
      }
      // C_l += w * M_r: warp ew takes columns ew, ew + 7, ... four at a time; a lane owns rows
      // lane, lane + 32, lane + 64, lane + 96, so loads and stores are 256-byte coalesced and
      // 16 loads are in flight per lane before the stores
#pragma unroll 1
      for (int c = 0; c < p.nc; ++c) {
        const Term tm = a.terms[p.c0 + c];
        const double wgt = tm.coef;
        int* tk = nullptr;
        if (per_block) {  // wait for the previous product that updates this C block
          tk = a.tickets + (long long)w.tile * a.nbt + tm.row * a.nbc + tm.col;
          if (et == 0) ticket_spin(tk, tm.pad, a.status, 128);
          named_bar_sync(2, NEPI_D);
        }
        double* Cb = a.C + (long long)tm.row * a.ms + (long long)tm.col * a.ns * a.ldc + w.m0 + lane;
        const int rmax = rows - lane;  // rows of this lane inside the tile: rr < rmax
#pragma unroll 1
        for (int col0 = ew; col0 < BN; col0 += NW * 4) {
          double cv[4][4];
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) {
            const int col = col0 + cb * NW;
            const bool cok = col < BN && w.n0 + col < a.ns;
            const double* cp = Cb + (long long)(w.n0 + col) * a.ldc;
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) cv[cb][ch] = (cok && ch * 32 < rmax) ? cp[ch * 32] : 0.0;
          }
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) {
            const int col = col0 + cb * NW;
            if (!(col < BN && w.n0 + col < a.ns)) continue;
            double* cp = Cb + (long long)(w.n0 + col) * a.ldc;
            const double* mp = Ms + col * MS_LD + lane;
#pragma unroll
            for (int ch = 0; ch < 4; ++ch)
              if (ch * 32 < rmax) cp[ch * 32] = fma(wgt, mp[ch * 32], cv[cb][ch]);
          }
        }
        if (tk) {  // this block's update is visible before the next product may start its own
          __threadfence();
          named_bar_sync(2, NEPI_D);
          if (et == 0) st_release(tk, tm.pad + 1);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(mempty);  // the buffer can take the next product
    }
    if (ordered && a.nbt == 0) {
      __threadfence();
      named_bar_sync(2, NEPI_D);
      if (et == 0) st_release(a.tickets + w.tile, chunk + 1);
    }
  }
}

template <class Src>
__device__ __forceinline__ void gemm_cta_direct(const Src& src) {
  extern __shared__ __align__(128) double smem[];
  double* stages = smem;                                        // [NSTAGE_D][STAGE_SZ]
  double* Ms = stages + (size_t)NSTAGE_D * STAGE_SZ;            // [BN][MS_LD]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(Ms + (size_t)BN * MS_LD);
  const unsigned full0 = smem_u32(bars);
  const unsigned empty0 = smem_u32(bars + NSTAGE_D);
  const unsigned mfull = smem_u32(bars + 2 * NSTAGE_D);
  const unsigned mempty = smem_u32(bars + 2 * NSTAGE_D + 1);
  const UnitRing q{smem_u32(bars + 2 * NSTAGE_D + 2)};
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE_D; ++s) {
      mbar_init(full0 + 8 * s, 1);             // the issuer's arrival + TMA bytes
      mbar_init(empty0 + 8 * s, NCONS / 32);
    }
    mbar_init(mfull, NCONS / 32);
    mbar_init(mempty, NEPI_D / 32);
    unit_ring_init(q, (NEPI_D + NCONS) / 32);  // ring readers: epilogue + consumer warps
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (tid < NPROD) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(PROD_REGS));
    if (tid == 0)
      direct_issuer(src, stages, full0, empty0, q);
    else if (tid >= 32)
      direct_epilogue(src, Ms, mfull, mempty, tid - 32, q);
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(CONS_REGS));
    direct_consumer(src, stages, Ms, full0, empty0, mfull, mempty, tid - NPROD, q);
  }
}

__global__ void __launch_bounds__(NTHREADS, 1) fmm_gemm_direct_kernel(const __grid_constant__ GemmArgs a) {
  gemm_cta_direct(OneJob{a});
}

__global__ void __launch_bounds__(NTHREADS, 1) fmm_gemm_direct_batch_kernel(const BatchArgs b) {
  gemm_cta_direct(JobBatch{b.jobs, b.unit_start, b.njobs, b.units, b.status, b.counter});
}

// Operand sums in HBM: out_j = sum_t coef_t * X_{blk_t} for the A terms (side 0) or the
// B terms (side 1) of product plist[j] (j = blockIdx.y).  Used for the NAIVE pack
// type's S_r / T_r temporaries and for the pre-summed operands of the ABC pack type.
// Each thread handles two consecutive rows of a column (16-byte loads and stores when
// the addresses allow).
struct LincombArgs {
  const double* X;
  long long ldx;
  int rows, cols;          // sub-block size
  int blk_row_stride;      // rows per block row (ms for A, ks for B)
  int blk_col_stride;      // cols per block column (ks for A, ns for B)
  double* out;
  long long ldo;
  long long out_stride;    // per output
  const Prod* prods;
  const Term* terms;
  const int* plist;        // product of each output; nullptr = output j is product j
  int side;
};

// Elements per block: output j = blockIdx.x varies fastest in the grid, so the blocks
// resident at one time cover the same element range for many outputs and read each input
// element from HBM about once (the other reads hit L2).
constexpr int LINCOMB_CHUNK = 256 * 16;  // row pairs per block

__device__ __forceinline__ long long lincomb_pairs(const LincombArgs& a) {
  return (long long)((a.rows + 1) / 2) * a.cols;
}

__device__ __forceinline__ void lincomb_body(const LincombArgs& a, int j, long long chunk) {
  const int r = a.plist ? a.plist[j] : j;
  const Prod p = a.prods[r];
  const int t0 = a.side == 0 ? p.a0 : p.b0;
  const int nt = a.side == 0 ? p.na : p.nb;
  double* out = a.out + (long long)j * a.out_stride;
  const int hr = (a.rows + 1) / 2;  // row pairs per column
  const long long total = lincomb_pairs(a);
  const long long e1 = min(total, (chunk + 1) * LINCOMB_CHUNK);
  long long e = chunk * LINCOMB_CHUNK + threadIdx.x;
  int ip = (int)(e % hr);  // row pair and column of element e, then stepped without division
  long long c = e / hr;
  for (; e < e1; e += blockDim.x) {
    const int i = 2 * ip;
    const bool two = i + 1 < a.rows;
    double v0 = 0.0, v1 = 0.0;
    // terms in groups of four: the group's loads are issued before its fmas, so a thread
    // keeps several loads in flight (the sum order is unchanged)
    for (int tg = 0; tg < nt; tg += 4) {
      double x0[4], x1[4], cf[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        x0[q] = x1[q] = cf[q] = 0.0;
        if (tg + q < nt) {
          const Term tm = a.terms[t0 + tg + q];
          cf[q] = tm.coef;
          const double* x =
              a.X + (long long)tm.row * a.blk_row_stride + i + ((long long)tm.col * a.blk_col_stride + c) * a.ldx;
          if (two && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
            const double2 xx = *reinterpret_cast<const double2*>(x);
            x0[q] = xx.x;
            x1[q] = xx.y;
          } else {
            x0[q] = x[0];
            if (two) x1[q] = x[1];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int t = tg + q;
        if (t < nt) {
          v0 = (t == 0) ? cf[q] * x0[q] : fma(cf[q], x0[q], v0);
          v1 = (t == 0) ? cf[q] * x1[q] : fma(cf[q], x1[q], v1);
        }
      }
    }
    double* o = out + i + c * a.ldo;
    if (two && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
      *reinterpret_cast<double2*>(o) = make_double2(v0, v1);
    } else {
      o[0] = v0;
      if (two) o[1] = v1;
    }
    ip += blockDim.x;
    while (ip >= hr) {
      ip -= hr;
      ++c;
    }
  }
}

__global__ void fmm_lincomb_kernel(const LincombArgs a) {
  const long long nchunk = (lincomb_pairs(a) + LINCOMB_CHUNK - 1) / LINCOMB_CHUNK;
  for (long long c = blockIdx.y; c < nchunk; c += gridDim.y) lincomb_body(a, blockIdx.x, c);
}

// The operand sums of many problems in one launch: task blockIdx.z, output blockIdx.x
// (tasks with fewer outputs return at once), element chunks over blockIdx.y.
struct LincombTask {
  LincombArgs a;
  int nout;
  int pad;
};

__global__ void fmm_lincomb_batch_kernel(const LincombTask* tasks) {
  const LincombTask& tk = tasks[blockIdx.z];
  if ((int)blockIdx.x >= tk.nout) return;
  const long long nchunk = (lincomb_pairs(tk.a) + LINCOMB_CHUNK - 1) / LINCOMB_CHUNK;
  for (long long c = blockIdx.y; c < nchunk; c += gridDim.y) lincomb_body(tk.a, blockIdx.x, c);
}

// Column-major copies between pitches, many in one launch (task blockIdx.y): used to give
// operands with an odd leading dimension the even pitch (16-byte column starts) that
// tensor-memory-access staging needs.
struct PitchCopy {
  const double* src;
  long long lds;
  double* dst;
  long long ldd;
  int rows, cols;
};

__device__ __forceinline__ void pitch_copy_body(const PitchCopy& t) {
  for (int j = blockIdx.x; j < t.cols; j += gridDim.x) {
    const double* s = t.src + (long long)j * t.lds;
    double* d = t.dst + (long long)j * t.ldd;
    for (int i = threadIdx.x; i < t.rows; i += blockDim.x) d[i] = s[i];
  }
}

__global__ void fmm_pitch_copy_kernel(const PitchCopy* tasks) { pitch_copy_body(tasks[blockIdx.y]); }
__global__ void fmm_pitch_copy1_kernel(const PitchCopy t) { pitch_copy_body(t); }

// C_l += sum_r W[l, r] * M_r for every C block, the blocks in groups of up to COMBINE_GROUP: a
// thread owns P element positions and walks the groups; for a group it keeps the running values of
// its member blocks in registers, walks the union of their products in increasing r (one
// load of M_r per position, COMBINE_G_BATCH loads in flight) and applies M_r to every member
// whose W[l, r] is nonzero, c_l = fma(W[l, r], M_r, c_l).  Each block still gets exactly the
// epilogue's fma sequence (products in increasing r), so the result is bit-identical to the
// direct schedule.  The host groups blocks that share products (greedy by overlap), which
// cuts the M loads per position from nnz(W) toward R (222-1 x 333-1: 540 -> 299 in 5
// groups) with no shared-memory read-modify-write.  Tables (shared memory, per CTA):
//   group g: gdesc[g * GDESC + 0..3] = first entry, #entries, #members, first chunk;
//            gdesc[g * GDESC + 4 + q] = block id of member q (row * grid_n + col)
//   entry e: er[e] = product r, em[e] = member mask | (first coefficient of e) << 8,
//            the coefficients of its set bits, member order, from ec[first coefficient]
constexpr int COMBINE_GROUP = 8;
constexpr int GDESC = 4 + COMBINE_GROUP;
constexpr int COMBINE_G_THREADS = 256;
constexpr int COMBINE_G_BATCH = 16;

struct CombineGroupArgs {
  double* C;
  long long ldc;
  int ms, ns;
  const double* M;
  long long ldm;
  long long m_stride;
  int grid_n;
  int ngroup, nent, ncoef;
  const int* gdesc;
  const int* er;
  const int* em;
  const double* ec;
  int nprod;  // products (slabs of M)
  // staged kernel: the entries of each group in chunks of CST_CHUNK
  int nchunk;
  const int* chr;                 // [nchunk][CST_CHUNK] products (past a group's end: its last)
  const unsigned long long* chm;  // [nchunk] byte q: slots that update member q
  const double* chc;              // [nchunk][COMBINE_GROUP][CST_CHUNK] coefficients
};

__host__ __device__ constexpr size_t combine_group_smem_bytes(int ngroup, int nent, int ncoef) {
  return sizeof(double) * (size_t)ncoef + sizeof(int) * (2 * (size_t)nent + (size_t)GDESC * ngroup) + 16;
}

template <int P>
__global__ void __launch_bounds__(COMBINE_G_THREADS) fmm_combine_kernel(const CombineGroupArgs a) {
  extern __shared__ __align__(16) double gtab[];
  double* sc = gtab;                               // [ncoef]
  int* sr = reinterpret_cast<int*>(sc + a.ncoef);  // [nent]
  int* sm = sr + a.nent;                           // [nent]
  int* sg = sm + a.nent;                           // [GDESC * ngroup]
  for (int q = threadIdx.x; q < a.ncoef; q += blockDim.x) sc[q] = a.ec[q];
  for (int q = threadIdx.x; q < a.nent; q += blockDim.x) {
    sr[q] = a.er[q];
    sm[q] = a.em[q];
  }
  for (int q = threadIdx.x; q < GDESC * a.ngroup; q += blockDim.x) sg[q] = a.gdesc[q];
  __syncthreads();
  const int nt = blockDim.x;
  const long long total = (long long)a.ms * a.ns;
  for (long long e0 = (long long)blockIdx.x * nt * P; e0 < total; e0 += (long long)gridDim.x * nt * P) {
    // position p of this thread: e0 + threadIdx.x + p * nt (clamped to the last one, whose
    // stores then repeat the same values)
    long long cofs[P], mofs[P];
    bool live[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const long long e = e0 + threadIdx.x + (long long)p * nt;
      live[p] = e < total;
      const long long ee = live[p] ? e : total - 1;
      const int i = (int)(ee % a.ms);
      const long long j = ee / a.ms;
      cofs[p] = i + j * a.ldc;
      mofs[p] = i + j * a.ldm;
    }
    if (!live[0]) continue;
#pragma unroll 1
    for (int g = 0; g < a.ngroup; ++g) {
      const int* gd = sg + g * GDESC;
      const int ef = gd[0], ne = gd[1], nm = gd[2];
      double c[COMBINE_GROUP][P];
      long long cb[COMBINE_GROUP];
#pragma unroll
      for (int q = 0; q < COMBINE_GROUP; ++q) {
        const int b = gd[4 + (q < nm ? q : 0)];
        cb[q] = (long long)(b / a.grid_n) * a.ms + (long long)(b % a.grid_n) * a.ns * a.ldc;
#pragma unroll
        for (int p = 0; p < P; ++p) c[q][p] = q < nm ? a.C[cb[q] + cofs[p]] : 0.0;
      }
#pragma unroll 1
      for (int q0 = 0; q0 < ne; q0 += COMBINE_G_BATCH) {
        double mv[COMBINE_G_BATCH][P];
#pragma unroll
        for (int t = 0; t < COMBINE_G_BATCH; ++t) {
          const long long mo = (long long)sr[ef + min(q0 + t, ne - 1)] * a.m_stride;
#pragma unroll
          for (int p = 0; p < P; ++p) mv[t][p] = __ldcg(a.M + mo + mofs[p]);
        }
#pragma unroll
        for (int t = 0; t < COMBINE_G_BATCH; ++t) {
          if (q0 + t >= ne) break;
          const int mk = sm[ef + q0 + t];
          int k = mk >> 8;
#pragma unroll
          for (int q = 0; q < COMBINE_GROUP; ++q)
            if (mk & (1 << q)) {
              const double w = sc[k++];
#pragma unroll
              for (int p = 0; p < P; ++p) c[q][p] = fma(w, mv[t][p], c[q][p]);
            }
        }
      }
#pragma unroll
      for (int q = 0; q < COMBINE_GROUP; ++q)
        if (q < nm) {
#pragma unroll
          for (int p = 0; p < P; ++p)
            if (live[p]) a.C[cb[q] + cofs[p]] = c[q][p];
        }
    }
  }
}

// The same combine with the M values staged in shared memory by bulk copies: a tile of
// CST_TILE consecutive element positions (M_r[e0 .. e0 + CST_TILE) is contiguous when
// ldm == ms), walked group by group and, within a group, CST_CHUNK products at a time; a
// producer warp copies each chunk's M_r tiles (cp.async.bulk, 2 KB each) into a ring of
// CST_STAGES stages while the compute warps apply earlier chunks, so the loads in flight per
// SM are bounded by shared memory instead of registers.  A compute thread owns one position
// of the tile and keeps its group's running C values in registers; the arithmetic per block
// is the register kernel's (bit-identical).  Waits are bounded (status word on timeout).
constexpr int CST_THREADS = 256;  // compute threads, one position each
constexpr int CST_TILE = CST_THREADS;
constexpr int CST_CHUNK = 8;      // products per stage
constexpr int CST_STAGES = 3;  // 48 KB of stages: three CTAs per SM (24 compute warps)
constexpr size_t CST_STAGE_DOUBLES = (size_t)CST_CHUNK * CST_TILE;
static_assert(COMBINE_GROUP * CST_CHUNK <= 64, "one 64-bit word of slot bits per chunk");

__host__ __device__ constexpr size_t combine_staged_smem_bytes(int ngroup, int nchunk) {
  return sizeof(double) * CST_STAGE_DOUBLES * CST_STAGES + 16 * CST_STAGES +
         (sizeof(double) * COMBINE_GROUP * CST_CHUNK + sizeof(unsigned long long) + sizeof(int) * CST_CHUNK) *
             (size_t)nchunk +
         sizeof(int) * GDESC * (size_t)ngroup + 16;
}

__device__ __forceinline__ void bulk_load_1d(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// CombineGroupArgs plus the status word; requires ldm == ms, M and m_stride 16-byte
// multiples (in doubles: m_stride even) and ms * ns even (every tile's byte count a multiple
// of 16).
__global__ void __launch_bounds__(CST_THREADS + 32) fmm_combine_staged_kernel(const CombineGroupArgs a,
                                                                              unsigned* status) {
  extern __shared__ __align__(128) double cst[];
  double* stages = cst;                                                    // [STAGES][CHUNK][TILE]
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(stages + CST_STAGE_DOUBLES * CST_STAGES);
  double* sc = reinterpret_cast<double*>(bars + 2 * CST_STAGES);           // [nchunk][GROUP][CHUNK]
  unsigned long long* smk = reinterpret_cast<unsigned long long*>(sc + (size_t)a.nchunk * COMBINE_GROUP * CST_CHUNK);
  int* sr = reinterpret_cast<int*>(smk + a.nchunk);                        // [nchunk][CHUNK]
  int* sg = sr + (size_t)a.nchunk * CST_CHUNK;                             // [GDESC * ngroup]
  const unsigned full0 = smem_u32(bars), empty0 = smem_u32(bars + CST_STAGES);
  const int tid = threadIdx.x;
  for (int q = tid; q < a.nchunk * COMBINE_GROUP * CST_CHUNK; q += blockDim.x) sc[q] = a.chc[q];
  for (int q = tid; q < a.nchunk; q += blockDim.x) smk[q] = a.chm[q];
  for (int q = tid; q < a.nchunk * CST_CHUNK; q += blockDim.x) sr[q] = a.chr[q];
  for (int q = tid; q < GDESC * a.ngroup; q += blockDim.x) sg[q] = a.gdesc[q];
  if (tid == 0) {
    for (int s = 0; s < CST_STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, CST_THREADS / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const long long total = (long long)a.ms * a.ns;
  const long long ntile = (total + CST_TILE - 1) / CST_TILE;
  long long k = 0;  // stage step of this CTA
  if (tid >= CST_THREADS) {  // producer warp: lane 0 issues the copies
    if (tid != CST_THREADS) return;
    for (long long t = blockIdx.x; t < ntile; t += gridDim.x) {
      const long long e0 = t * CST_TILE;
      const unsigned bytes = (unsigned)(8 * min((long long)CST_TILE, total - e0));
      for (int g = 0; g < a.ngroup; ++g) {
        const int ne = sg[g * GDESC + 1], c0 = sg[g * GDESC + 3];
        for (int q0 = 0; q0 < ne; q0 += CST_CHUNK, ++k) {
          const int s = (int)(k % CST_STAGES);
          mbar_wait(empty0 + 8 * s, (unsigned)(((k / CST_STAGES) & 1) ^ 1), status);
          const int nq = min(CST_CHUNK, ne - q0);
          const int* rr = sr + (size_t)(c0 + q0 / CST_CHUNK) * CST_CHUNK;
          mbar_arrive_expect_tx(full0 + 8 * s, bytes * nq);
          for (int q = 0; q < nq; ++q) {
            int r = rr[q];
            if ((unsigned)r >= (unsigned)a.nprod) {  // never with host-checked tables
              atomicOr(status, STATUS_TABLE);
              r = 0;
            }
            bulk_load_1d(smem_u32(stages + (size_t)s * CST_STAGE_DOUBLES + (size_t)q * CST_TILE),
                         a.M + (long long)r * a.m_stride + e0, bytes, full0 + 8 * s);
          }
        }
      }
    }
    // copies still in flight (only on an error path) land before the CTA exits
    for (long long q = k - CST_STAGES; q < k; ++q)
      if (q >= 0) mbar_wait_drain(full0 + 8 * (int)(q % CST_STAGES), (unsigned)((q / CST_STAGES) & 1));
    return;
  }
  const int lane = tid & 31;
  for (long long t = blockIdx.x; t < ntile; t += gridDim.x) {
    const long long e = t * CST_TILE + tid;
    const bool live = e < total;
    const long long ee = live ? e : total - 1;
    const long long cofs = (ee % a.ms) + (ee / a.ms) * a.ldc;
    for (int g = 0; g < a.ngroup; ++g) {
      const int* gd = sg + g * GDESC;
      const int ne = gd[1], nm = gd[2], c0 = gd[3];
      double c[COMBINE_GROUP];
      long long cb[COMBINE_GROUP];
#pragma unroll
      for (int q = 0; q < COMBINE_GROUP; ++q) {
        const int b = gd[4 + (q < nm ? q : 0)];
        cb[q] = (long long)(b / a.grid_n) * a.ms + (long long)(b % a.grid_n) * a.ns * a.ldc + cofs;
        c[q] = q < nm ? a.C[cb[q]] : 0.0;
      }
      for (int q0 = 0; q0 < ne; q0 += CST_CHUNK, ++k) {
        const int s = (int)(k % CST_STAGES);
        const int ch = c0 + q0 / CST_CHUNK;
        const unsigned long long bits = smk[ch];
        const double* cf = sc + (size_t)ch * COMBINE_GROUP * CST_CHUNK;
        mbar_wait(full0 + 8 * s, (unsigned)((k / CST_STAGES) & 1), status);
        const double* st = stages + (size_t)s * CST_STAGE_DOUBLES + tid;
        // per member only its set slots (warp-uniform bit loops): the M value and the
        // coefficient come from shared memory at the slot's index, the running value stays in
        // a register (members unrolled); slots past the group's end have no bits
#pragma unroll
        for (int b = 0; b < COMBINE_GROUP; ++b) {
          unsigned bq = (unsigned)(bits >> (8 * b)) & 0xffu;
          while (bq) {
            const int q = __ffs(bq) - 1;
            bq &= bq - 1;
            c[b] = fma(cf[b * CST_CHUNK + q], st[(size_t)q * CST_TILE], c[b]);
          }
        }
        __threadfence_block();  // the stage's loads complete before it can be refilled
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * s);
      }
      if (live) {
#pragma unroll
        for (int q = 0; q < COMBINE_GROUP; ++q)
          if (q < nm) a.C[cb[q]] = c[q];
      }
    }
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
