// fmm_b200 host runtime and C ABI (declared in include/fmm_b200.h).
//
// Reference interfaces replaced (fmm-gen):
//   bl_dgemm                       common/dgemm/my_dgemm.c:115-210
//   bl_dgemm_strassen_abc/ab/naive common/include/bl_dgemm.h:96-130 (generated bodies:
//                                  meta/abc_gen_mix.py:448-472, meta/ab_gen_mix.py:430-456,
//                                  meta/naive_gen_mix.py:412-429)
//   fringe split + peeling         meta/common_mix.py:124-171, common/dgemm/bl_dgemm_util.c:316-353
//   packing pool                   common/dgemm/bl_dgemm_util.c:375-394 (here: stream-ordered
//                                  device allocations, freed after each call)
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <iterator>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "../../include/fmm_b200.h"
#include "fmm_kernels.cuh"
#include "fmm_split_bf16.cuh"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kBatchCounters = 2;  // a batch's per-phase work-unit counters, ahead of its tickets
constexpr int kMR = 8;  // register-tile granularity of the FMM/fringe split (bl_config.h:16-17)
constexpr int kNR = 4;

std::atomic<long long> g_launches{0};
thread_local int t_last_error = FMM_OK;
// Byte written into every ticket before a launch (fmm_debug_set): 0 in normal operation.
int g_ticket_fill = 0;
// Cap on the pre-summed operand workspace of one call (fmm_set_workspace_limit), and the
// workspace bytes the last call on this thread used.
constexpr long long kDefaultWorkspaceLimit = 8LL << 30;
std::atomic<long long> g_ws_limit{kDefaultWorkspaceLimit};
thread_local long long t_last_ws = 0;

// Optional per-kernel timing: when enabled, every launch is bracketed by CUDA events on
// its own stream; fmm_profile_end() sums the durations per kernel kind.
enum KernelKind {
  K_GEMM_FMM = 0,
  K_GEMM_CLASSICAL = 1,
  K_LINCOMB = 2,
  K_SCATTER = 3,
  K_SPLIT_OPERANDS = 4,
  K_GEMM_SPLIT = 5,
  K_GEMM_BATCH = 6,
  K_LINCOMB_BATCH = 7,
  K_PITCH_COPY = 8,
  K_COMBINE = 9,
  K_GEMM_FMM_DIRECT = 10,        // the same launches when they run the direct variant
  K_GEMM_CLASSICAL_DIRECT = 11,
  K_NUM = 12
};
const char* const kKernelNames[K_NUM] = {"fmm_gemm_kernel[fmm products]", "fmm_gemm_kernel[classical]",
                                         "fmm_lincomb_kernel", "fmm_scatter_kernel",
                                         "fmm_split_operands_kernel", "fmm_split_gemm_kernel",
                                         "fmm_gemm_batch_kernel", "fmm_lincomb_batch_kernel",
                                         "fmm_pitch_copy_kernel", "fmm_combine_kernel",
                                         "fmm_gemm_direct_kernel[fmm products]",
                                         "fmm_gemm_direct_kernel[classical]"};
struct ProfRec {
  int kind;
  cudaEvent_t e0, e1;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;

struct ProfScope {
  int kind;
  cudaStream_t st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ProfScope(int k, cudaStream_t s) : kind(k), st(s) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_on) return;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      e0 = e1 = nullptr;
      return;
    }
    cudaEventRecord(e0, st);
  }
  ~ProfScope() {
    if (!e0) return;
    cudaEventRecord(e1, st);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof.push_back(ProfRec{kind, e0, e1});
  }
};

struct DevTables {
  fmm::Prod* prods = nullptr;
  fmm::Term* terms = nullptr;
  int* cblk = nullptr;
  int* ent_r = nullptr;
  double* ent_w = nullptr;
  int* cg_desc = nullptr;  // grouped combine tables
  int* cg_r = nullptr;
  int* cg_m = nullptr;
  double* cg_c = nullptr;
  int* ch_r = nullptr;
  unsigned long long* ch_m = nullptr;
  double* ch_c = nullptr;
  fmm::Prod* prods_ps = nullptr;  // products over pre-summed operands (one A and one B term each)
  fmm::Term* terms_ps = nullptr;
  int* plistA = nullptr;          // products whose A operand is pre-summed, in slot order
  int* plistB = nullptr;
  fmm::Prod* prods_all = nullptr;  // every product over pre-summed slots (slot r = product r)
  fmm::Term* terms_all = nullptr;
  int* plist_all = nullptr;        // 0 .. R-1
  bool ready = false;
};

// Tables of a k split (see ksplit_tables): base tables (one of the TableBase forms) with
// every product r split into S products (r, p) over k range p of its operands.
enum TableBase : int { BASE_ORIG = 0, BASE_PS = 1, BASE_ALL = 2, BASE_GROUP = 3 };
struct KSplitTables {
  int base = 0, S = 0, g1 = 0, dev = -1;  // BASE_GROUP: products [S, g1) (see group_build)
  fmm::Prod* prods = nullptr;
  fmm::Term* terms = nullptr;
};

}  // namespace

struct fmm_plan {
  int dims[3];
  int rank;
  std::vector<fmm::Prod> prods;
  std::vector<fmm::Term> terms;
  // Per C block lists of (product, coefficient), products in order: used by the scatter.
  std::vector<int> cblk;     // 4 ints per block
  std::vector<int> ent_r;
  std::vector<double> ent_w;
  int n_cblk = 0;
  int n_cterms = 0;  // C terms over all products
  // The same lists with the blocks in groups that share products (fmm_combine_kernel's
  // tables: group descriptors, merged entries and their coefficients; see build_combine_groups).
  std::vector<int> cg_desc, cg_r, cg_m;
  std::vector<double> cg_c;
  int n_cgroup = 0;
  std::vector<int> ch_r;                 // staged kernel: CST_CHUNK products per chunk
  std::vector<unsigned long long> ch_m;  // one byte of slot bits per member
  std::vector<double> ch_c;              // COMBINE_GROUP x CST_CHUNK coefficients per chunk
  // Pre-summed form: each product's A operand is either its single A block (src 0) or
  // slot j of the workspace S (src 1) that holds sum_i U[i,r] A_i; likewise for B / T.
  std::vector<fmm::Prod> prods_ps;
  std::vector<fmm::Term> terms_ps;
  std::vector<int> plistA, plistB;
  // Every product pre-summed (slot r = product r): used when ks is not a multiple of the
  // k step, so that zero-padded workspaces keep each k step inside its operand block.
  std::vector<fmm::Prod> prods_all;
  std::vector<fmm::Term> terms_all;
  std::mutex mu;
  DevTables dev[kMaxDevices];
  std::vector<KSplitTables> ksplit;  // uploaded k-split tables (any device), built on first use
};

namespace {

fmm_plan* g_default_plan = nullptr;
std::mutex g_default_mu;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return FMM_OK;
  if (e == cudaErrorMemoryAllocation) return FMM_E_NOMEM;
  return FMM_E_CUDA;
}

#define FMM_CUDA_TRY(expr)                  \
  do {                                      \
    cudaError_t _e = (expr);                \
    if (_e != cudaSuccess) return cuda_status(_e); \
  } while (0)

int upload_tables(fmm_plan* p, DevTables& d) {
  std::lock_guard<std::mutex> lk(p->mu);
  if (d.ready) return FMM_OK;
  FMM_CUDA_TRY(cudaMalloc(&d.prods, sizeof(fmm::Prod) * p->prods.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.terms, sizeof(fmm::Term) * p->terms.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.cblk, sizeof(int) * (p->cblk.size() ? p->cblk.size() : 1)));
  FMM_CUDA_TRY(cudaMalloc(&d.ent_r, sizeof(int) * (p->ent_r.size() ? p->ent_r.size() : 1)));
  FMM_CUDA_TRY(cudaMalloc(&d.ent_w, sizeof(double) * (p->ent_w.size() ? p->ent_w.size() : 1)));
  FMM_CUDA_TRY(cudaMemcpy(d.prods, p->prods.data(), sizeof(fmm::Prod) * p->prods.size(), cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemcpy(d.terms, p->terms.data(), sizeof(fmm::Term) * p->terms.size(), cudaMemcpyHostToDevice));
  if (!p->cblk.empty())
    FMM_CUDA_TRY(cudaMemcpy(d.cblk, p->cblk.data(), sizeof(int) * p->cblk.size(), cudaMemcpyHostToDevice));
  if (!p->ent_r.empty()) {
    FMM_CUDA_TRY(cudaMemcpy(d.ent_r, p->ent_r.data(), sizeof(int) * p->ent_r.size(), cudaMemcpyHostToDevice));
    FMM_CUDA_TRY(cudaMemcpy(d.ent_w, p->ent_w.data(), sizeof(double) * p->ent_w.size(), cudaMemcpyHostToDevice));
  }
  {
    auto up = [](auto** dst, const auto& v) -> cudaError_t {
      using T = typename std::decay_t<decltype(v)>::value_type;
      cudaError_t e = cudaMalloc(dst, sizeof(T) * (v.size() ? v.size() : 1));
      if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
      return e;
    };
    FMM_CUDA_TRY(up(&d.cg_desc, p->cg_desc));
    FMM_CUDA_TRY(up(&d.cg_r, p->cg_r));
    FMM_CUDA_TRY(up(&d.cg_m, p->cg_m));
    FMM_CUDA_TRY(up(&d.cg_c, p->cg_c));
    FMM_CUDA_TRY(up(&d.ch_r, p->ch_r));
    FMM_CUDA_TRY(up(&d.ch_m, p->ch_m));
    FMM_CUDA_TRY(up(&d.ch_c, p->ch_c));
  }
  FMM_CUDA_TRY(cudaMalloc(&d.prods_ps, sizeof(fmm::Prod) * p->prods_ps.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.terms_ps, sizeof(fmm::Term) * p->terms_ps.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.plistA, sizeof(int) * (p->plistA.size() + 1)));
  FMM_CUDA_TRY(cudaMalloc(&d.plistB, sizeof(int) * (p->plistB.size() + 1)));
  FMM_CUDA_TRY(cudaMemcpy(d.prods_ps, p->prods_ps.data(), sizeof(fmm::Prod) * p->prods_ps.size(),
                          cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemcpy(d.terms_ps, p->terms_ps.data(), sizeof(fmm::Term) * p->terms_ps.size(),
                          cudaMemcpyHostToDevice));
  if (!p->plistA.empty())
    FMM_CUDA_TRY(cudaMemcpy(d.plistA, p->plistA.data(), sizeof(int) * p->plistA.size(), cudaMemcpyHostToDevice));
  if (!p->plistB.empty())
    FMM_CUDA_TRY(cudaMemcpy(d.plistB, p->plistB.data(), sizeof(int) * p->plistB.size(), cudaMemcpyHostToDevice));
  std::vector<int> all(p->rank);
  for (int r = 0; r < p->rank; ++r) all[r] = r;
  FMM_CUDA_TRY(cudaMalloc(&d.prods_all, sizeof(fmm::Prod) * p->prods_all.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.terms_all, sizeof(fmm::Term) * p->terms_all.size()));
  FMM_CUDA_TRY(cudaMalloc(&d.plist_all, sizeof(int) * all.size()));
  FMM_CUDA_TRY(cudaMemcpy(d.prods_all, p->prods_all.data(), sizeof(fmm::Prod) * p->prods_all.size(),
                          cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemcpy(d.terms_all, p->terms_all.data(), sizeof(fmm::Term) * p->terms_all.size(),
                          cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemcpy(d.plist_all, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice));
  d.ready = true;
  return FMM_OK;
}

int device_tables(const fmm_plan* cp, DevTables** out) {
  fmm_plan* p = const_cast<fmm_plan*>(cp);
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return FMM_E_UNSUPPORTED;
  DevTables& d = p->dev[dev];
  if (!d.ready) {
    int rc = upload_tables(p, d);
    if (rc != FMM_OK) return rc;
  }
  *out = &d;
  return FMM_OK;
}

// k split of a plan's products: product r (k extent ks) becomes S products (r, p), p = 0..S-1,
// each over k range [p ks/S, (p+1) ks/S) of r's operands, with r's C terms.  A work unit then
// covers a product's k range part, so a launch with too few units for whole waves of the
// SMs gets S times as many, shorter ones.  The C update is linear in the product, so the
// parts' updates, applied in order (r, 0), (r, 1), ... under the same tickets, sum to r's.
// With the part depth ks' = ks / S every operand term keeps its block and indexes part p by
// its k block coordinate: an A term (row, col) becomes (row, col S + p) (A column offset
// col ks + p ks' = (col S + p) ks'), a B term (row, col) becomes (row S + p, col); this holds
// for blocks of A and B and for the slots of the pre-summed workspaces alike.  C terms keep
// their block; their per-block ticket position (pad) counts the split products.
void ksplit_build(const fmm_plan* p, int base, int S, std::vector<fmm::Prod>* op, std::vector<fmm::Term>* ot) {
  const std::vector<fmm::Prod>& prods = base == BASE_PS ? p->prods_ps : base == BASE_ALL ? p->prods_all : p->prods;
  const std::vector<fmm::Term>& terms = base == BASE_PS ? p->terms_ps : base == BASE_ALL ? p->terms_all : p->terms;
  std::vector<int> cnt((size_t)p->dims[0] * p->dims[2], 0);
  // part-major: split product (r, q) is q * R + r, so the S parts of one (tile, product) are
  // R tiles' worth of units apart and do not run at the same time (their C updates are
  // ordered by tickets, so parts claimed together would wait on each other)
  for (int q = 0; q < S; ++q) {
    for (const fmm::Prod& pr : prods) {
      fmm::Prod v = pr;
      v.a0 = (int)ot->size();
      for (int t = 0; t < pr.na; ++t) {
        fmm::Term x = terms[pr.a0 + t];
        x.col = x.col * S + q;
        ot->push_back(x);
      }
      v.b0 = (int)ot->size();
      for (int t = 0; t < pr.nb; ++t) {
        fmm::Term x = terms[pr.b0 + t];
        x.row = x.row * S + q;
        ot->push_back(x);
      }
      v.c0 = (int)ot->size();
      for (int t = 0; t < pr.nc; ++t) {
        fmm::Term x = terms[pr.c0 + t];
        x.pad = cnt[(size_t)x.row * p->dims[2] + x.col]++;
        ot->push_back(x);
      }
      op->push_back(v);
    }
  }
}

// Tables of products [g0, g1) over the slots of a group workspace: product r reads slot
// r - g0 of S and of T (src 1), keeps its C terms, and counts its per-block ticket positions
// within the group (each group is a launch of its own).
void group_build(const fmm_plan* p, int g0, int g1, std::vector<fmm::Prod>* op, std::vector<fmm::Term>* ot) {
  std::vector<int> cnt((size_t)p->dims[0] * p->dims[2], 0);
  for (int r = g0; r < g1; ++r) {
    const fmm::Prod& pr = p->prods[r];
    fmm::Prod v{};
    v.a0 = (int)ot->size();
    v.na = 1;
    ot->push_back(fmm::Term{0, r - g0, 1.0, 1, 0});
    v.b0 = (int)ot->size();
    v.nb = 1;
    ot->push_back(fmm::Term{0, r - g0, 1.0, 1, 0});
    v.c0 = (int)ot->size();
    v.nc = pr.nc;
    for (int t = 0; t < pr.nc; ++t) {
      fmm::Term x = p->terms[pr.c0 + t];
      x.pad = cnt[(size_t)x.row * p->dims[2] + x.col]++;
      ot->push_back(x);
    }
    op->push_back(v);
  }
}

// Derived tables of a plan on the current device (uploaded on first use): the k split S of a
// base form (ksplit_build), or with base == BASE_GROUP the group [S, g1) (group_build).
int ksplit_tables(const fmm_plan* cp, int base, int S, const fmm::Prod** prods, const fmm::Term** terms,
                  int g1 = 0) {
  fmm_plan* p = const_cast<fmm_plan*>(cp);
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(p->mu);
  for (const auto& t : p->ksplit)
    if (t.base == base && t.S == S && t.g1 == g1 && t.dev == dev) {
      *prods = t.prods;
      *terms = t.terms;
      return FMM_OK;
    }
  std::vector<fmm::Prod> vp;
  std::vector<fmm::Term> vt;
  if (base == BASE_GROUP)
    group_build(p, S, g1, &vp, &vt);
  else
    ksplit_build(p, base, S, &vp, &vt);
  KSplitTables t;
  t.base = base;
  t.S = S;
  t.g1 = g1;
  t.dev = dev;
  FMM_CUDA_TRY(cudaMalloc(&t.prods, sizeof(fmm::Prod) * vp.size()));
  cudaError_t e = cudaMalloc(&t.terms, sizeof(fmm::Term) * vt.size());
  if (e == cudaSuccess) e = cudaMemcpy(t.prods, vp.data(), sizeof(fmm::Prod) * vp.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t.terms, vt.data(), sizeof(fmm::Term) * vt.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(t.prods);
    if (t.terms) cudaFree(t.terms);
    return cuda_status(e);
  }
  p->ksplit.push_back(t);
  *prods = t.prods;
  *terms = t.terms;
  return FMM_OK;
}

// Blocks of the C grid in groups of up to fmm::COMBINE_GROUP that share products, for
// fmm_combine_kernel: greedily merge the two groups whose product sets overlap most (while
// the merged group fits), up to 64 blocks; beyond that, consecutive blocks.  Then one merged
// entry per product of a group's union (increasing r) with the mask of the members it
// updates and their coefficients in member order.
void build_combine_groups(fmm_plan* p) {
  const int nb = p->n_cblk;
  std::vector<std::vector<int>> mem(nb), uni(nb);
  for (int b = 0; b < nb; ++b) {
    mem[b] = {b};
    const int e0 = p->cblk[4 * b + 2], ne = p->cblk[4 * b + 3];
    uni[b].assign(p->ent_r.begin() + e0, p->ent_r.begin() + e0 + ne);  // increasing r
  }
  auto overlap = [](const std::vector<int>& x, const std::vector<int>& y) {
    size_t i = 0, j = 0;
    int n = 0;
    while (i < x.size() && j < y.size()) {
      if (x[i] == y[j]) ++n, ++i, ++j;
      else if (x[i] < y[j]) ++i;
      else ++j;
    }
    return n;
  };
  if (nb <= 64) {
    for (;;) {
      int best = 0, bi = -1, bj = -1;
      for (int i = 0; i < (int)mem.size(); ++i)
        for (int j = i + 1; j < (int)mem.size(); ++j) {
          if ((int)(mem[i].size() + mem[j].size()) > fmm::COMBINE_GROUP) continue;
          const int ov = overlap(uni[i], uni[j]);
          if (ov > best) best = ov, bi = i, bj = j;
        }
      if (bi < 0) break;
      mem[bi].insert(mem[bi].end(), mem[bj].begin(), mem[bj].end());
      std::vector<int> u;
      std::set_union(uni[bi].begin(), uni[bi].end(), uni[bj].begin(), uni[bj].end(), std::back_inserter(u));
      uni[bi] = u;
      mem.erase(mem.begin() + bj);
      uni.erase(uni.begin() + bj);
    }
  } else {
    std::vector<std::vector<int>> m2, u2;
    for (int b = 0; b < nb; b += fmm::COMBINE_GROUP) {
      std::vector<int> g, u;
      for (int q = b; q < std::min(nb, b + fmm::COMBINE_GROUP); ++q) {
        g.push_back(q);
        std::vector<int> t;
        std::set_union(u.begin(), u.end(), uni[q].begin(), uni[q].end(), std::back_inserter(t));
        u = t;
      }
      m2.push_back(g);
      u2.push_back(u);
    }
    mem = m2;
    uni = u2;
  }
  p->cg_desc.clear();
  p->ch_r.clear();
  p->ch_m.clear();
  p->ch_c.clear();
  p->cg_r.clear();
  p->cg_m.clear();
  p->cg_c.clear();
  for (size_t g = 0; g < mem.size(); ++g) {
    const int first = (int)p->cg_r.size();
    std::vector<size_t> pos(mem[g].size(), 0);  // cursor into each member's (increasing r) list
    for (int r : uni[g]) {
      int mask = 0;
      const int k0 = (int)p->cg_c.size();
      for (size_t q = 0; q < mem[g].size(); ++q) {
        const int b = mem[g][q];
        const int e0 = p->cblk[4 * b + 2], ne = p->cblk[4 * b + 3];
        if (pos[q] < (size_t)ne && p->ent_r[e0 + pos[q]] == r) {
          mask |= 1 << q;
          p->cg_c.push_back(p->ent_w[e0 + pos[q]]);
          ++pos[q];
        }
      }
      p->cg_r.push_back(r);
      p->cg_m.push_back(mask | (k0 << 8));
    }
    // the group's entries in chunks of CST_CHUNK (the staged kernel's stage): per chunk the
    // products, one byte per member (bit t: slot t updates it) and a member-major
    // CST_CHUNK x CST_CHUNK coefficient block (0 where the bit is clear)
    const int first_chunk = (int)(p->ch_r.size() / fmm::CST_CHUNK);
    {
      const int ne = (int)p->cg_r.size() - first;
      for (int q0 = 0; q0 < ne; q0 += fmm::CST_CHUNK) {
        unsigned long long bits = 0;
        std::vector<double> cf((size_t)fmm::COMBINE_GROUP * fmm::CST_CHUNK, 0.0);
        for (int t = 0; t < fmm::CST_CHUNK; ++t) {
          const int e = first + std::min(q0 + t, ne - 1);
          p->ch_r.push_back(p->cg_r[e]);
          if (q0 + t >= ne) continue;
          const int mk = p->cg_m[e];
          int kc = mk >> 8;
          for (int q = 0; q < fmm::COMBINE_GROUP; ++q)
            if (mk & (1 << q)) {
              bits |= 1ULL << (8 * q + t);
              cf[(size_t)q * fmm::CST_CHUNK + t] = p->cg_c[kc++];
            }
        }
        p->ch_m.push_back(bits);
        p->ch_c.insert(p->ch_c.end(), cf.begin(), cf.end());
      }
    }
    p->cg_desc.push_back(first);
    p->cg_desc.push_back((int)p->cg_r.size() - first);
    p->cg_desc.push_back((int)mem[g].size());
    p->cg_desc.push_back(first_chunk);
    for (int q = 0; q < fmm::COMBINE_GROUP; ++q) {
      const int b = q < (int)mem[g].size() ? mem[g][q] : mem[g][0];
      p->cg_desc.push_back(p->cblk[4 * b] * p->dims[2] + p->cblk[4 * b + 1]);
    }
  }
  p->n_cgroup = (int)mem.size();
  // the kernels index their tables with these values: check them here (a plan whose tables
  // fail falls back to the per-block scatter)
  bool ok = p->ch_r.size() == (size_t)fmm::CST_CHUNK * p->ch_m.size() &&
            p->ch_c.size() == (size_t)fmm::COMBINE_GROUP * fmm::CST_CHUNK * p->ch_m.size();
  for (int r : p->ch_r) ok = ok && r >= 0 && r < p->rank;
  for (int r : p->cg_r) ok = ok && r >= 0 && r < p->rank;
  for (int g = 0; ok && g < p->n_cgroup; ++g) {
    const int* gd = p->cg_desc.data() + (size_t)g * fmm::GDESC;
    const int nch = (gd[1] + fmm::CST_CHUNK - 1) / fmm::CST_CHUNK;
    ok = gd[1] > 0 && gd[0] + gd[1] <= (int)p->cg_r.size() && gd[2] >= 1 && gd[2] <= fmm::COMBINE_GROUP &&
         gd[3] >= 0 && gd[3] + nch <= (int)p->ch_m.size();
    for (int q = 0; ok && q < fmm::COMBINE_GROUP; ++q) ok = gd[4 + q] >= 0 && gd[4 + q] < p->dims[0] * p->dims[2];
  }
  if (!ok) p->n_cgroup = 0;
}

int build_plan(const int dims[3], int rank, const int* nterms, const int* rows, const int* cols,
               const double* coefs, fmm_plan** out) {
  if (!dims || !nterms || !rows || !cols || !coefs || !out || rank <= 0) return FMM_E_INVALID;
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return FMM_E_PLAN;
  fmm_plan* p = new (std::nothrow) fmm_plan();
  if (!p) return FMM_E_NOMEM;
  std::memcpy(p->dims, dims, sizeof(p->dims));
  p->rank = rank;
  int pos = 0;
  const int lim[3][2] = {{dims[0], dims[1]}, {dims[1], dims[2]}, {dims[0], dims[2]}};
  for (int r = 0; r < rank; ++r) {
    fmm::Prod pr{};
    int* first[3] = {&pr.a0, &pr.b0, &pr.c0};
    int* count[3] = {&pr.na, &pr.nb, &pr.nc};
    for (int s = 0; s < 3; ++s) {
      const int n = nterms[3 * r + s];
      if (n <= 0) {
        delete p;
        return FMM_E_PLAN;
      }
      *first[s] = (int)p->terms.size();
      *count[s] = n;
      for (int q = 0; q < n; ++q, ++pos) {
        if (rows[pos] < 0 || rows[pos] >= lim[s][0] || cols[pos] < 0 || cols[pos] >= lim[s][1]) {
          delete p;
          return FMM_E_PLAN;
        }
        p->terms.push_back(fmm::Term{rows[pos], cols[pos], coefs[pos], 0, 0});
      }
    }
    // A single operand term whose coefficient is a power of two moves its coefficient
    // into the product's W coefficients (exact), so the operand can be staged as is.
    for (int side = 0; side < 2; ++side) {
      const int n = side == 0 ? pr.na : pr.nb;
      fmm::Term& t = p->terms[side == 0 ? pr.a0 : pr.b0];
      int e2 = 0;
      if (n == 1 && t.coef != 1.0 && t.coef != 0.0 && std::frexp(std::fabs(t.coef), &e2) == 0.5) {
        for (int q = 0; q < pr.nc; ++q) p->terms[pr.c0 + q].coef *= t.coef;
        t.coef = 1.0;
      }
    }
    p->prods.push_back(pr);
  }
  for (const auto& pr : p->prods) p->n_cterms += pr.nc;
  // C block lists for the scatter (products in increasing order per block).
  const int nblk = dims[0] * dims[2];
  std::vector<std::vector<std::pair<int, double>>> lists(nblk);
  for (int r = 0; r < rank; ++r) {
    const fmm::Prod& pr = p->prods[r];
    for (int q = 0; q < pr.nc; ++q) {
      fmm::Term& t = p->terms[pr.c0 + q];
      auto& list = lists[t.row * dims[2] + t.col];
      t.pad = (int)list.size();  // position among the block's products (per-block tickets)
      list.push_back({r, t.coef});
    }
  }
  for (int b = 0; b < nblk; ++b) {
    if (lists[b].empty()) continue;
    p->cblk.push_back(b / dims[2]);
    p->cblk.push_back(b % dims[2]);
    p->cblk.push_back((int)p->ent_r.size());
    p->cblk.push_back((int)lists[b].size());
    for (auto& e : lists[b]) {
      p->ent_r.push_back(e.first);
      p->ent_w.push_back(e.second);
    }
    ++p->n_cblk;
  }
  build_combine_groups(p);
  for (int r = 0; r < rank; ++r) {
    const fmm::Prod& pr = p->prods[r];
    fmm::Prod q{};
    q.a0 = (int)p->terms_ps.size();
    q.na = 1;
    const fmm::Term& ta = p->terms[pr.a0];
    if (pr.na == 1 && ta.coef == 1.0) {
      p->terms_ps.push_back(ta);
    } else {
      p->terms_ps.push_back(fmm::Term{0, (int)p->plistA.size(), 1.0, 1, 0});
      p->plistA.push_back(r);
    }
    q.b0 = (int)p->terms_ps.size();
    q.nb = 1;
    const fmm::Term& tb = p->terms[pr.b0];
    if (pr.nb == 1 && tb.coef == 1.0) {
      p->terms_ps.push_back(tb);
    } else {
      p->terms_ps.push_back(fmm::Term{0, (int)p->plistB.size(), 1.0, 1, 0});
      p->plistB.push_back(r);
    }
    q.c0 = (int)p->terms_ps.size();
    q.nc = pr.nc;
    for (int c = 0; c < pr.nc; ++c) p->terms_ps.push_back(p->terms[pr.c0 + c]);
    p->prods_ps.push_back(q);
    fmm::Prod qa{};
    qa.a0 = (int)p->terms_all.size();
    qa.na = 1;
    p->terms_all.push_back(fmm::Term{0, r, 1.0, 1, 0});
    qa.b0 = (int)p->terms_all.size();
    qa.nb = 1;
    p->terms_all.push_back(fmm::Term{0, r, 1.0, 1, 0});
    qa.c0 = (int)p->terms_all.size();
    qa.nc = pr.nc;
    for (int c = 0; c < pr.nc; ++c) p->terms_all.push_back(p->terms[pr.c0 + c]);
    p->prods_all.push_back(qa);
  }
  *out = p;
  return FMM_OK;
}

fmm_plan* classical_plan() {
  static fmm_plan* p = [] {
    const int dims[3] = {1, 1, 1};
    const int nt[3] = {1, 1, 1};
    const int rows[3] = {0, 0, 0}, cols[3] = {0, 0, 0};
    const double coefs[3] = {1.0, 1.0, 1.0};
    fmm_plan* q = nullptr;
    build_plan(dims, 1, nt, rows, cols, coefs, &q);
    return q;
  }();
  return p;
}

bool smem_configured[kMaxDevices];
int sm_count[kMaxDevices];
unsigned* dev_status[kMaxDevices];
std::mutex g_attr_mu;

PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

int configure_kernel(int* dev_out) {
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return FMM_E_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (!smem_configured[dev]) {
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmm::smem_bytes(false)));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmm::smem_bytes(true)));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_direct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmm::SMEM_BYTES_DIRECT));
    if (!g_encode_tiled) {
      cudaDriverEntryPointQueryResult q;
      void* fn = nullptr;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
          q == cudaDriverEntryPointSuccess)
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    FMM_CUDA_TRY(cudaDeviceGetAttribute(&sm_count[dev], cudaDevAttrMultiProcessorCount, dev));
    // Workspaces come from the device's stream-ordered pool; keep freed blocks mapped
    // instead of returning them to the driver at every synchronisation, so repeated
    // calls do not pay for mapping gigabytes of workspace again.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      cuuint64_t keep = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    FMM_CUDA_TRY(cudaMalloc(&dev_status[dev], sizeof(unsigned)));
    FMM_CUDA_TRY(cudaMemset(dev_status[dev], 0, sizeof(unsigned)));
    smem_configured[dev] = true;
  }
  *dev_out = dev;
  return FMM_OK;
}

// Column-major FP64 matrix (rows x cols, leading dimension ld) as a 2-D tensor map with
// the given box.  Returns false when TMA cannot address it (then cp.async staging runs).
bool make_tensor_map(CUtensorMap* map, const double* base, long long rows, long long cols, long long ld,
                     unsigned box_rows, unsigned box_cols) {
  if (!g_encode_tiled) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (ld & 1) != 0) return false;
  if (rows <= 0 || cols <= 0 || rows >= (1LL << 31) || cols >= (1LL << 31) || ld * 8 >= (1LL << 40)) return false;
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(double)};
  cuuint32_t box[2] = {box_rows, box_cols};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode_tiled(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Work units take one product each (product-major order): the CTAs running at one time
// then work on one or two products, whose operand panels stay in L2, and the per-tile
// tickets keep the C updates in product order.  Measured on B200 against units of many
// products: 16384^3 222-1 x 333-1 35.6 -> 36.5 TFLOP/s, 222-2 41.0 -> 41.3.
int choose_chunks(int ntiles, int nprod, int nsm) {
  (void)ntiles;
  (void)nsm;
  return nprod;
}

// k split (ksplit_build) for a launch of `units` work units of ks deep products on nsm SMs.
// A launch of few units spends its last wave partly idle: 222-1 at 2048^3 has 448 units
// on 148 SMs, 3.03 waves whose last holds 4 units.  Splitting every product's k range into S
// parts gives S times the units, each S times shorter; the modelled time
// ceil(units S / nsm) (ks / (8 S) + kUnitOverheadSteps) k steps picks S in 1..8 (parts of
// whole k steps, at least kMinPartSteps deep; a split must gain 3 %).  Launches of many waves
// keep S = 1.
constexpr int kUnitOverheadSteps = 4;  // per-unit cost beyond its k steps (hand-off, C tile traffic)
constexpr int kMinPartSteps = 16;
std::atomic<int> g_split_form{0};     // fmm_debug_set FMM_DEBUG_SPLIT_OPERANDS: 1 = one product per CTA
std::atomic<int> g_force_ksplit{0};  // fmm_debug_set FMM_DEBUG_KSPLIT: S for every split launch (0: model)
int choose_ksplit(long long units, int ks, int nsm) {
  if (units <= 0 || nsm <= 0 || units >= 8LL * nsm || ks % fmm::BK != 0) return 1;
  const long long nks = ks / fmm::BK;
  const int forced = g_force_ksplit.load();
  if (forced > 0) return (nks % forced == 0 && nks / forced >= kMinPartSteps) ? forced : 1;
  auto cost = [&](int S) { return ((units * S + nsm - 1) / nsm) * (double)(nks / S + kUnitOverheadSteps); };
  int best = 1;
  double best_cost = cost(1);
  for (int S = 2; S <= 8; ++S) {
    if (nks % S != 0 || nks / S < kMinPartSteps) continue;
    const double c = cost(S);
    if (c < 0.97 * best_cost) {
      best = S;
      best_cost = c;
    }
  }
  return best;
}

// Launch the persistent DMMA GEMM over sub-blocks of size ms x ks x ns.
// Workspaces of pre-summed operands (slot j of S: ms x ks, of T: ks x ns, block columns).
struct PresumOps {
  const int* plistA = nullptr;  // products of the slots (device); nullptr: the plan's lists
  const int* plistB = nullptr;
  int kslot = 0;                // columns per S slot and rows per T slot; 0: ks
  const double* S = nullptr;
  long long ldS = 0;
  int nslotA = 0;
  const double* T = nullptr;
  long long ldT = 0;
  int nslotB = 0;
};

// Every k step of a product reads only its own operand blocks: ks is a multiple of BK, or
// the block grid is 1 x 1 x 1, where the tensor maps end at the operands' last k column / row
// and a partial last step reads TMA's zero fill.
bool whole_k_steps(const int grid_dims[3], int ks) {
  return ks % fmm::BK == 0 || (grid_dims[0] == 1 && grid_dims[1] == 1 && grid_dims[2] == 1);
}

// direct_ok: every product's operands are single unit-coefficient blocks (pre-summed
// products, the classical plan), so with TMA staging and whole k steps the direct variant
// (epilogue on the otherwise idle folding warps, overlapping the next product) can run.
// ksplit > 1: prods / terms are k-split tables (ksplit_tables) with nprod = R * ksplit products
// of depth ks / ksplit, a whole number of k steps; ks is the operands' full depth.
int launch_gemm(int kind, const fmm::Prod* prods, const fmm::Term* terms, const int grid_dims[3], int nprod,
                int mode, const double* A, long long lda, const double* B, long long ldb, const PresumOps& ps,
                double* C, long long ldc, double* M, long long ldm, long long m_stride, int ms, int ns, int ks,
                cudaStream_t st, bool direct_ok = false, int ks_orig = -1, int ksplit = 1) {
  if (ms <= 0 || ns <= 0 || ks <= 0 || nprod <= 0) return FMM_OK;
  if (ksplit < 1 || ks % ksplit != 0 || (ksplit > 1 && (ks / ksplit) % fmm::BK != 0)) return FMM_E_INVALID;
  int dev = 0;
  int rc = configure_kernel(&dev);
  if (rc != FMM_OK) return rc;
  fmm::GemmArgs a{};
  a.A = A;
  a.lda = lda;
  a.B = B;
  a.ldb = ldb;
  a.C = C;
  a.ldc = ldc;
  a.M = M;
  a.ldm = ldm;
  a.m_stride = m_stride;
  a.ms = ms;
  a.ns = ns;
  a.ks = ks / ksplit;
  a.prods = prods;
  a.terms = terms;
  a.Aw = ps.S ? ps.S : A;
  a.ldaw = ps.S ? ps.ldS : lda;
  a.Bw = ps.T ? ps.T : B;
  a.ldbw = ps.T ? ps.ldT : ldb;
  a.nprod = nprod;
  a.tiles_m = (ms + fmm::BM - 1) / fmm::BM;
  a.tiles_n = (ns + fmm::BN - 1) / fmm::BN;
  a.mode = mode;
  a.status = dev_status[dev];
  const int ntiles = a.tiles_m * a.tiles_n;
  a.chunks = (mode == fmm::MODE_ACCUM_C) ? choose_chunks(ntiles, nprod, sm_count[dev]) : 1;
  const long long units = (long long)ntiles * (mode == fmm::MODE_STORE_M ? nprod : a.chunks);
  if (units > INT32_MAX) return FMM_E_UNSUPPORTED;
  const unsigned grid = (unsigned)(units < sm_count[dev] ? units : sm_count[dev]);
  // A spans grid_dims[0] x grid_dims[1] blocks of ms x ks; B grid_dims[1] x grid_dims[2] of ks x ns
  // the operands' own maps cover the operands (their k extent is the real one when the
  // products read zero-padded pre-summed slots)
  const long long am = (long long)grid_dims[0] * ms, ak = (long long)grid_dims[1] * (ks_orig >= 0 ? ks_orig : ks),
                  bn = (long long)grid_dims[2] * ns;
  bool tma = make_tensor_map(&a.tmA, A, am, ak, lda, fmm::BM, fmm::BK) &&
             make_tensor_map(&a.tmA64, A, am, ak, lda, fmm::BM / 2, fmm::BK) &&
             make_tensor_map(&a.tmB, B, ak, bn, ldb, fmm::BK, fmm::BN) &&
             make_tensor_map(&a.tmB2, B, ak, bn, ldb, fmm::TB_K, fmm::BN);
  if (tma) {
    if (ps.S && ps.nslotA > 0)
      tma = make_tensor_map(&a.tmAw, ps.S, ms, (long long)ps.nslotA * ks, ps.ldS, fmm::BM, fmm::BK) &&
            make_tensor_map(&a.tmAw64, ps.S, ms, (long long)ps.nslotA * ks, ps.ldS, fmm::BM / 2, fmm::BK);
    else
      a.tmAw = a.tmA, a.tmAw64 = a.tmA64;
  }
  if (tma) {
    if (ps.T && ps.nslotB > 0)
      tma = make_tensor_map(&a.tmBw, ps.T, ks, (long long)ps.nslotB * ns, ps.ldT, fmm::BK, fmm::BN) &&
            make_tensor_map(&a.tmBw2, ps.T, ks, (long long)ps.nslotB * ns, ps.ldT, fmm::TB_K, fmm::BN);
    else
      a.tmBw = a.tmB, a.tmBw2 = a.tmB2;
  }
  const bool direct = direct_ok && tma && whole_k_steps(grid_dims, a.ks);
  // Per-tile tickets keep a tile's C updates in product order.  With few tile positions
  // (at most half as many as SMs) the units of one position run at the same time and their
  // epilogues form one chain of all R products; there the direct variant (one product per
  // unit) orders the updates per (tile, C block) instead, so only products that update the
  // same C block wait for one another.  Each C element still receives its products'
  // updates in product order (same results).  Measured on B200, per tile -> per block:
  // 222-1 x 333-1 3000^3 3.21 -> 2.13 ms, 4000 x 3840 x 2000 3.29 -> 2.67 ms, 4096^3 5.42
  // -> 5.08 ms; 222-2 2048^3 0.88 -> 0.60 ms; 222-1 1024^3 0.17 -> 0.14 ms.  With more
  // positions the extra barrier per C term costs more than it frees (14400^2 x 480, 361
  // positions: 12.5 -> 14.0 ms; 4000 x 16000 x 2000, 126 positions: 9.5 -> 9.9 ms).
  // [0]: the launch's work-unit counter; then the tickets
  size_t nt = 0;
  if (mode == fmm::MODE_ACCUM_C && a.chunks > 1) {
    if (direct && a.chunks == nprod && 2 * ntiles <= sm_count[dev]) {
      a.nbt = grid_dims[0] * grid_dims[2];
      a.nbc = grid_dims[2];
    }
    nt = (size_t)ntiles * (a.nbt > 0 ? a.nbt : 1);
  }
  int* tickets = nullptr;
  FMM_CUDA_TRY(cudaMallocAsync((void**)&tickets, sizeof(int) * (nt + 1), st));
  FMM_CUDA_TRY(cudaMemsetAsync(tickets, 0, sizeof(int) * (nt + 1), st));
  if (nt > 0 && g_ticket_fill != 0)
    FMM_CUDA_TRY(cudaMemsetAsync(tickets + 1, g_ticket_fill, sizeof(int) * nt, st));
  a.counter = tickets;
  a.tickets = nt > 0 ? tickets + 1 : nullptr;
  {
    const int pkind = !direct ? kind : (kind == K_GEMM_FMM ? K_GEMM_FMM_DIRECT : K_GEMM_CLASSICAL_DIRECT);
    ProfScope ps(pkind, st);
    if (direct)
      fmm::fmm_gemm_direct_kernel<<<grid, fmm::NTHREADS, fmm::SMEM_BYTES_DIRECT, st>>>(a);
    else if (tma)
      fmm::fmm_gemm_kernel<true><<<grid, fmm::NTHREADS, fmm::smem_bytes(true), st>>>(a);
    else
      fmm::fmm_gemm_kernel<false><<<grid, fmm::NTHREADS, fmm::smem_bytes(false), st>>>(a);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  rc = cuda_status(cudaGetLastError());
  if (tickets) {
    cudaError_t fe = cudaFreeAsync(tickets, st);
    if (rc == FMM_OK) rc = cuda_status(fe);
  }
  return rc;
}

const int kUnitGrid[3] = {1, 1, 1};

int call_ksplit(const fmm_plan* plan, int ms, int ns, int ks, bool presum, int kk, int nsm);  // below

int sm_count_current() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  return sm_count[dev];
}

int plain_gemm(int m, int n, int k, const double* A, long long lda, const double* B, long long ldb, double* C,
               long long ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0 || k <= 0) return FMM_OK;
  DevTables* d = nullptr;
  int rc = device_tables(classical_plan(), &d);
  if (rc != FMM_OK) return rc;
  int dev = 0;
  rc = configure_kernel(&dev);
  if (rc != FMM_OK) return rc;
  const int S = call_ksplit(classical_plan(), m, n, k, false, k, sm_count[dev]);
  if (S > 1) {
    const fmm::Prod* vp = nullptr;
    const fmm::Term* vt = nullptr;
    rc = ksplit_tables(classical_plan(), BASE_ORIG, S, &vp, &vt);
    if (rc != FMM_OK) return rc;
    return launch_gemm(K_GEMM_CLASSICAL, vp, vt, kUnitGrid, S, fmm::MODE_ACCUM_C, A, lda, B, ldb, PresumOps{}, C,
                       ldc, nullptr, 0, 0, m, n, k, st, true, -1, S);
  }
  return launch_gemm(K_GEMM_CLASSICAL, d->prods, d->terms, kUnitGrid, 1, fmm::MODE_ACCUM_C, A, lda, B, ldb,
                     PresumOps{}, C, ldc, nullptr, 0, 0, m, n, k, st, true);
}

int grid_for(long long total, int threads) {
  long long b = (total + threads - 1) / threads;
  if (b > 148LL * 16) b = 148LL * 16;
  if (b < 1) b = 1;
  return (int)b;
}

// Blocks along the element dimension of fmm_lincomb_kernel (each covers LINCOMB_CHUNK
// row pairs; beyond the grid limit the blocks loop).
unsigned lincomb_chunks(long long pairs) {
  const long long c = (pairs + fmm::LINCOMB_CHUNK - 1) / fmm::LINCOMB_CHUNK;
  return (unsigned)std::max<long long>(1, std::min<long long>(c, 65535));
}

// Fringe GEMMs, same regions and order as the reference's dynamic peeling.
int peel(int m, int n, int k, const double* A, long long lda, const double* B, long long ldb, double* C,
         long long ldc, int dim1, int dim2, int dim3, cudaStream_t st) {
  const int mr = m % dim1, kr = k % dim2, nr = n % dim3;
  const int ms = m - mr, ns = n - nr, ks = k - kr;
  int rc = FMM_OK;
  if (kr > 0 && ms > 0 && ns > 0) {
    rc = plain_gemm(ms, ns, kr, A + (long long)ks * lda, lda, B + ks, ldb, C, ldc, st);
    if (rc != FMM_OK) return rc;
  }
  if (nr > 0) {
    rc = plain_gemm(m, nr, k, A, lda, B + (long long)ns * ldb, ldb, C + (long long)ns * ldc, ldc, st);
    if (rc != FMM_OK) return rc;
  }
  if (mr > 0 && ns > 0) {
    rc = plain_gemm(mr, ns, k, A + ms, lda, B, ldb, C + ms, ldc, st);
    if (rc != FMM_OK) return rc;
  }
  return FMM_OK;
}

// C_l += sum_r W[l,r] * M_r for every C block at once (fmm_combine_kernel); false when the
// plan's grouped tables do not fit the kernel's shared memory (the caller then uses the
// per-block scatter).
bool combine_fits(const fmm_plan* plan) {
  return plan->n_cgroup > 0 &&
         fmm::combine_group_smem_bytes(plan->n_cgroup, (int)plan->cg_r.size(), (int)plan->cg_c.size()) <= 200 * 1024;
}

bool combine_configured[kMaxDevices];
// element positions per thread of the combine (fmm_debug_set FMM_DEBUG_COMBINE_POSITIONS; 0: 1)
std::atomic<int> g_combine_positions{0};

int launch_combine(const fmm_plan* plan, const DevTables& d, double* C, long long ldc, int ms, int ns,
                   const double* M, long long ldm, long long m_stride, cudaStream_t st) {
  int dev = 0;
  int rc0 = configure_kernel(&dev);
  if (rc0 != FMM_OK) return rc0;
  {
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (!combine_configured[dev]) {
      FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_combine_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
      FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_combine_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
      FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_combine_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024));
      combine_configured[dev] = true;
    }
  }
  fmm::CombineGroupArgs ga{};
  ga.C = C;
  ga.ldc = ldc;
  ga.ms = ms;
  ga.ns = ns;
  ga.M = M;
  ga.ldm = ldm;
  ga.m_stride = m_stride;
  ga.grid_n = plan->dims[2];
  ga.ngroup = plan->n_cgroup;
  ga.nent = (int)plan->cg_r.size();
  ga.ncoef = (int)plan->cg_c.size();
  ga.gdesc = d.cg_desc;
  ga.er = d.cg_r;
  ga.em = d.cg_m;
  ga.ec = d.cg_c;
  ga.nprod = plan->rank;
  const long long total = (long long)ms * ns;
  ga.nchunk = (int)plan->ch_m.size();
  ga.chr = d.ch_r;
  ga.chm = d.ch_m;
  ga.chc = d.ch_c;
  const size_t ssm = fmm::combine_staged_smem_bytes(ga.ngroup, ga.nchunk);
  // staged form: the M tiles of a position range are contiguous 16-byte-aligned runs
  const bool staged = g_combine_positions.load() == 0 && ldm == ms && m_stride % 2 == 0 && total % 2 == 0 &&
                      ((uintptr_t)M & 15) == 0 && ssm <= 200 * 1024 && total > 0;
  if (staged) {
    const long long ntile = (total + fmm::CST_TILE - 1) / fmm::CST_TILE;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(ntile, (long long)sm_count[dev] * 3));
    {
      ProfScope pf(K_COMBINE, st);
      fmm::fmm_combine_staged_kernel<<<grid, fmm::CST_THREADS + 32, ssm, st>>>(ga, dev_status[dev]);
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cuda_status(cudaGetLastError());
  }
  const int P = g_combine_positions.load() == 2 ? 2 : 1;
  const size_t smem = fmm::combine_group_smem_bytes(ga.ngroup, ga.nent, ga.ncoef);
  const long long per = (long long)fmm::COMBINE_G_THREADS * P;
  const long long blocks = ((long long)ms * ns + per - 1) / per;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(blocks, (long long)sm_count_current() * 8));
  {
    ProfScope pf(K_COMBINE, st);
    if (P == 2)
      fmm::fmm_combine_kernel<2><<<grid, fmm::COMBINE_G_THREADS, smem, st>>>(ga);
    else
      fmm::fmm_combine_kernel<1><<<grid, fmm::COMBINE_G_THREADS, smem, st>>>(ga);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cuda_status(cudaGetLastError());
}

// Pre-summing pays off once the sub-blocks are large enough that the extra pass over HBM
// (each operand sum written once, then read by every tile that uses it) costs less than
// folding the sums while staging, which limits the producer warps, and it lets the
// direct kernel variant run.  Measured on B200 (pre-summed vs folded): 222-1 x 333-1
// 4096^3 11.7 -> 5.4 ms, 4000 x 3840 x 2000 5.6 -> 3.3 ms, 14400 x 14400 x 480 22.5 ->
// 19.1 ms; 222-2 2048^3 1.34 -> 0.88 ms; 222-1 1024^3 0.24 -> 0.17 ms (ms * ns = 2^18).
bool use_presum(const fmm_plan* plan, int ms, int ns, int ks) {
  if (plan->plistA.empty() && plan->plistB.empty()) return false;
  return (long long)ms * ns >= (1LL << 17) && ks >= 64;
}

// ABC schedule for pre-summed products: the multi-destination epilogue (C_l += W[l,r] M_r
// straight from each product tile) or, when that C traffic dominates, the products stored
// to a workspace and one combine pass (every M_r and C element crossing HBM once).  The
// epilogue moves 16 nnz(W) ms ns bytes of C while the DMMAs run; the stored schedule writes
// 8 R ms ns bytes of product tiles (also during the DMMAs), then the combine pass moves
// 8 (R + 2 blocks) ms ns bytes.  Model fitted to B200 measurements (222-1 x 333-1, DMMA
// products 33 TFLOP/s executed, epilogue C traffic 4.6 TB/s, product stores 6 TB/s, combine
// 2.6 TB/s): the direct launch takes max(t_mma, t_epi) + 1.05 min^2 / max (the two overlap
// less as they approach each other: 4000 x 16000 x 2000 7.76 ms for t_mma 5.75 and t_epi
// 3.32, 14400 x 14400 x 480 12.4 ms, 8192^3 24.2 ms), the storing launch 1.08 max(t_mma,
// t_store) (6.16 and 4.92 ms).  The stored schedule must gain 3 % and its product workspace
// (8 R ms ns bytes) must fit the workspace cap.  It is the reference's own trade between its
// ABC and AB variants (meta/model_gen.py:87-95 counts the C memory operations of each).
bool prefer_stored_products(const fmm_plan* plan, int ms, int ns, int ks) {
  const double mn = (double)ms * ns;
  const int nblk = plan->dims[0] * plan->dims[2];
  if (8.0 * plan->rank * mn > (double)g_ws_limit.load()) return false;
  const double t_mma = 2.0 * plan->rank * mn * ks / 33e12;
  const double t_epi = 16.0 * plan->n_cterms * mn / 4.6e12;
  const double t_store = 8.0 * plan->rank * mn / 6.0e12;
  const double t_comb = 8.0 * (plan->rank + 2.0 * nblk) * mn / 2.6e12;
  const double hi = std::max(t_mma, t_epi), lo = std::min(t_mma, t_epi);
  const double t_direct = hi + 1.05 * lo * lo / hi;
  return 1.08 * std::max(t_mma, t_store) + t_comb < 0.97 * t_direct;
}

// One operand's sums (fmm_lincomb_kernel): output j = blockIdx.x, element chunks over y.
int launch_lincomb(const fmm_plan* plan, const fmm::LincombArgs& la, int nout, cudaStream_t st) {
  (void)plan;
  if (nout <= 0) return FMM_OK;
  const long long pairs = (long long)(la.rows + 1) / 2 * la.cols;
  {
    ProfScope pf(K_LINCOMB, st);
    fmm::fmm_lincomb_kernel<<<dim3((unsigned)nout, lincomb_chunks(pairs)), 256, 0, st>>>(la);
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cuda_status(cudaGetLastError());
}

int presum(const fmm_plan* plan, const DevTables& d, const double* A, long long lda, const double* B, long long ldb,
           const PresumOps& ps, int ms, int ns, int ks, cudaStream_t st) {
  if (ps.nslotA > 0) {
    fmm::LincombArgs la{};
    la.X = A;
    la.ldx = lda;
    la.rows = ms;
    la.cols = ks;
    la.blk_row_stride = ms;
    la.blk_col_stride = ks;
    la.out = const_cast<double*>(ps.S);
    la.ldo = ps.ldS;
    la.out_stride = ps.ldS * (ps.kslot ? ps.kslot : ks);
    la.prods = d.prods;
    la.terms = d.terms;
    la.plist = ps.plistA ? ps.plistA : d.plistA;
    la.side = 0;
    const int rc = launch_lincomb(plan, la, ps.nslotA, st);
    if (rc != FMM_OK) return rc;
  }
  if (ps.nslotB > 0) {
    fmm::LincombArgs lb{};
    lb.X = B;
    lb.ldx = ldb;
    lb.rows = ks;
    lb.cols = ns;
    lb.blk_row_stride = ks;
    lb.blk_col_stride = ns;
    lb.out = const_cast<double*>(ps.T);
    lb.ldo = ps.ldT;
    lb.out_stride = ps.ldT * ns;
    lb.prods = d.prods;
    lb.terms = d.terms;
    lb.plist = ps.plistB ? ps.plistB : d.plistB;
    lb.side = 1;
    const int rc = launch_lincomb(plan, lb, ps.nslotB, st);
    if (rc != FMM_OK) return rc;
  }
  return cuda_status(cudaGetLastError());
}

// Pre-summed operands for the products of one call: the workspace, the operand sums and the
// tables the products kernel reads them with.  When ks is not a multiple of the k step every
// product gets its own slot whose k extent is padded with zeros (kk = ks rounded up), so all
// k steps stay inside the slot and the direct variant can run.
struct PresumPlan {
  PresumOps ps;
  const fmm::Prod* prods = nullptr;
  const fmm::Term* terms = nullptr;
  int kk = 0;
  char* ws = nullptr;
};

int presum_prepare(const fmm_plan* plan, const DevTables& d, const double* A, long long lda, const double* B,
                   long long ldb, int ms, int ns, int ks, cudaStream_t st, PresumPlan* out) {
  const int R = plan->rank;
  PresumOps& ps = out->ps;
  int rc = FMM_OK;
  if (ks % fmm::BK != 0) {
    const int kp = (ks + fmm::BK - 1) / fmm::BK * fmm::BK;
    ps.plistA = d.plist_all;
    ps.plistB = d.plist_all;
    ps.kslot = kp;
    const size_t sbytes = sizeof(double) * (size_t)ms * kp * R;
    const size_t tbytes = sizeof(double) * (size_t)kp * ns * R;
    FMM_CUDA_TRY(cudaMallocAsync((void**)&out->ws, sbytes + tbytes + 16, st));
    ps.S = reinterpret_cast<double*>(out->ws);
    ps.ldS = ms;
    ps.nslotA = R;
    ps.T = reinterpret_cast<double*>(out->ws + sbytes);
    ps.ldT = kp;
    ps.nslotB = R;
    // zero padding: S slot r columns [ks, kp); T rows [ks, kp) of every column
    rc = cuda_status(cudaMemset2DAsync(out->ws + sizeof(double) * (size_t)ms * ks, sizeof(double) * (size_t)ms * kp,
                                       0, sizeof(double) * (size_t)ms * (kp - ks), R, st));
    if (rc == FMM_OK)
      rc = cuda_status(cudaMemset2DAsync(out->ws + sbytes + sizeof(double) * ks, sizeof(double) * kp, 0,
                                         sizeof(double) * (kp - ks), (size_t)R * ns, st));
    out->prods = d.prods_all;
    out->terms = d.terms_all;
    out->kk = kp;
  } else {
    const int nA = (int)plan->plistA.size(), nB = (int)plan->plistB.size();
    const long long ldT = ks + (ks & 1);
    const size_t sbytes = sizeof(double) * (size_t)ms * ks * nA;
    const size_t tbytes = sizeof(double) * (size_t)ldT * ns * nB;
    FMM_CUDA_TRY(cudaMallocAsync((void**)&out->ws, sbytes + tbytes + 16, st));
    ps.S = reinterpret_cast<double*>(out->ws);
    ps.ldS = ms;
    ps.nslotA = nA;
    ps.T = reinterpret_cast<double*>(out->ws + sbytes);
    ps.ldT = ldT;
    ps.nslotB = nB;
    out->prods = d.prods_ps;
    out->terms = d.terms_ps;
    out->kk = ks;
  }
  if (rc == FMM_OK) rc = presum(plan, d, A, lda, B, ldb, ps, ms, ns, ks, st);
  return rc;
}

// Bytes presum_prepare would allocate for one call.
size_t presum_bytes(const fmm_plan* plan, int ms, int ns, int ks) {
  if (ks % fmm::BK != 0) {
    const size_t kp = (ks + fmm::BK - 1) / fmm::BK * fmm::BK;
    return sizeof(double) * kp * ((size_t)ms + ns) * plan->rank + 16;
  }
  return sizeof(double) * ((size_t)ms * ks * plan->plistA.size() + (size_t)(ks + (ks & 1)) * ns * plan->plistB.size()) +
         16;
}

// The k split a single call gives products of ms x ks x ns: the pre-summed direct launch
// (unless the call stores its products or runs them in workspace groups) and the classical
// plan split as choose_ksplit decides; other forms keep S = 1.  Batches apply the same split
// per job.
int call_ksplit(const fmm_plan* plan, int ms, int ns, int ks, bool presum, int kk, int nsm) {
  const long long tiles = (long long)((ms + fmm::BM - 1) / fmm::BM) * ((ns + fmm::BN - 1) / fmm::BN);
  if (plan->rank == 1) return choose_ksplit(tiles, ks, nsm);
  if (!presum) return 1;
  if (combine_fits(plan) && prefer_stored_products(plan, ms, ns, ks)) return 1;
  if ((long long)presum_bytes(plan, ms, ns, ks) > g_ws_limit.load()) return 1;
  return choose_ksplit(tiles * plan->rank, kk, nsm);
}

// Pre-summed products in groups, when one call's whole operand workspace would exceed the
// workspace limit: the R products run as groups of G consecutive products, each group's
// operand sums (one slot per product, k extent padded to whole k steps) formed into one of
// two workspace halves while the previous group's products run.  The sums go on a second
// stream, which waits for the products that last read that half; each group's products
// wait for their sums.  Groups run in product order on the caller's stream, so every C
// element still receives its products' updates in order r = 0..R-1 (results are those of
// the ungrouped call).  Workspace 2 G (ms + ns) kk 8 bytes, within the limit for G >= 1.
int run_presum_groups(const fmm_plan* plan, const DevTables& d, const double* A, long long lda, const double* B,
                      long long ldb, double* C, long long ldc, int ms, int ns, int ks, cudaStream_t st) {
  const int R = plan->rank;
  const int kk = (ks + fmm::BK - 1) / fmm::BK * fmm::BK;
  const size_t sb = sizeof(double) * (size_t)ms * kk, tb = sizeof(double) * (size_t)kk * ns;
  long long G = g_ws_limit.load() / (long long)(2 * (sb + tb));
  G = std::max<long long>(1, std::min<long long>(G, R));
  const int ng = (int)((R + G - 1) / G);
  const int nbuf = ng > 1 ? 2 : 1;
  const size_t half = (size_t)G * (sb + tb);
  char* ws = nullptr;
  FMM_CUDA_TRY(cudaMallocAsync((void**)&ws, nbuf * half + 16, st));
  t_last_ws = (long long)(nbuf * half);
  int rc = FMM_OK;
  auto ok = [&](cudaError_t e) {
    if (rc == FMM_OK && e != cudaSuccess) rc = cuda_status(e);
    return rc == FMM_OK;
  };
  // zero padding once per half: S slot columns [ks, kk), T slot rows [ks, kk) (the sums fill [0, ks))
  for (int b = 0; b < nbuf && kk != ks; ++b) {
    char* S = ws + b * half;
    ok(cudaMemset2DAsync(S + sizeof(double) * (size_t)ms * ks, sb, 0, sizeof(double) * (size_t)ms * (kk - ks), G,
                         st)) &&
        ok(cudaMemset2DAsync(S + G * sb + sizeof(double) * ks, sizeof(double) * kk, 0, sizeof(double) * (kk - ks),
                             (size_t)G * ns, st));
  }
  cudaStream_t side = nullptr;
  cudaEvent_t ev_start = nullptr, ev_sum[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr};
  ok(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) &&
      ok(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming)) &&
      ok(cudaEventCreateWithFlags(&ev_sum[0], cudaEventDisableTiming)) &&
      ok(cudaEventCreateWithFlags(&ev_sum[1], cudaEventDisableTiming)) &&
      ok(cudaEventCreateWithFlags(&ev_done[0], cudaEventDisableTiming)) &&
      ok(cudaEventCreateWithFlags(&ev_done[1], cudaEventDisableTiming)) && ok(cudaEventRecord(ev_start, st)) &&
      ok(cudaStreamWaitEvent(side, ev_start, 0));
  for (int g = 0; g < ng && rc == FMM_OK; ++g) {
    const int g0 = (int)(g * G), g1 = (int)std::min<long long>(R, (g + 1) * G), n = g1 - g0, b = g % 2;
    char* S = ws + b * half;
    PresumOps ps;
    ps.plistA = d.plist_all + g0;
    ps.plistB = d.plist_all + g0;
    ps.kslot = kk;
    ps.S = reinterpret_cast<const double*>(S);
    ps.ldS = ms;
    ps.nslotA = n;
    ps.T = reinterpret_cast<const double*>(S + G * sb);
    ps.ldT = kk;
    ps.nslotB = n;
    if (g >= 2 && !ok(cudaStreamWaitEvent(side, ev_done[b], 0))) break;
    rc = presum(plan, d, A, lda, B, ldb, ps, ms, ns, ks, side);
    if (!ok(cudaEventRecord(ev_sum[b], side)) || !ok(cudaStreamWaitEvent(st, ev_sum[b], 0))) break;
    const fmm::Prod* gp = nullptr;
    const fmm::Term* gt = nullptr;
    if (rc == FMM_OK) rc = ksplit_tables(plan, BASE_GROUP, g0, &gp, &gt, g1);
    if (rc == FMM_OK)
      rc = launch_gemm(K_GEMM_FMM, gp, gt, plan->dims, n, fmm::MODE_ACCUM_C, A, lda, B, ldb, ps, C, ldc, nullptr, 0,
                       0, ms, ns, kk, st, true, ks);
    if (rc == FMM_OK) ok(cudaEventRecord(ev_done[b], st));
  }
  // every sum was waited for by the caller's stream, so freeing there comes after all uses
  cudaError_t fe = cudaFreeAsync(ws, st);
  if (rc == FMM_OK) rc = cuda_status(fe);
  for (cudaEvent_t e : {ev_start, ev_sum[0], ev_sum[1], ev_done[0], ev_done[1]})
    if (e) cudaEventDestroy(e);
  if (side) cudaStreamDestroy(side);
  return rc;
}

int check_args(int m, int n, int k, const void* A, long long lda, const void* B, long long ldb, const void* C,
               long long ldc) {
  if (m < 0 || n < 0 || k < 0) return FMM_E_INVALID;
  if (m == 0 || n == 0 || k == 0) return FMM_OK;
  if (!A || !B || !C) return FMM_E_INVALID;
  if (lda < m || ldb < k || ldc < m) return FMM_E_INVALID;
  return FMM_OK;
}

int run_fmm(const fmm_plan* plan, int pack, int m, int n, int k, const double* A, long long lda, const double* B,
            long long ldb, double* C, long long ldc, cudaStream_t st) {
  if (!plan) return FMM_E_NOPLAN;
  if (pack != FMM_PACK_ABC && pack != FMM_PACK_AB && pack != FMM_PACK_NAIVE) return FMM_E_UNSUPPORTED;
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK) return rc;
  if (m == 0 || n == 0 || k == 0) return FMM_OK;
  const int pm = plan->dims[0] * kMR, pk = plan->dims[1], pn = plan->dims[2] * kNR;
  const int md = m - m % pm, kd = k - k % pk, nd = n - n % pn;
  const int ms = md / plan->dims[0], ks = kd / plan->dims[1], ns = nd / plan->dims[2];
  DevTables* d = nullptr;
  rc = device_tables(plan, &d);
  if (rc != FMM_OK) return rc;
  const int R = plan->rank;
  t_last_ws = 0;
  if (ms > 0 && ns > 0 && ks > 0) {
    if (pack == FMM_PACK_ABC) {
      const int nA = (int)plan->plistA.size(), nB = (int)plan->plistB.size();
      if (use_presum(plan, ms, ns, ks) && combine_fits(plan) && prefer_stored_products(plan, ms, ns, ks)) {
        // C-traffic-bound shapes (small k per product): operand sums in HBM, each product
        // stored by the direct variant, W applied by one combine pass
        const long long mstride = (long long)ms * ns;
        char* mws = nullptr;
        FMM_CUDA_TRY(cudaMallocAsync((void**)&mws, sizeof(double) * (size_t)mstride * R, st));
        double* M = reinterpret_cast<double*>(mws);
        PresumPlan pp;
        t_last_ws = (long long)presum_bytes(plan, ms, ns, ks);
        rc = presum_prepare(plan, *d, A, lda, B, ldb, ms, ns, ks, st, &pp);
        if (rc == FMM_OK)
          rc = launch_gemm(K_GEMM_FMM, pp.prods, pp.terms, plan->dims, R, fmm::MODE_STORE_M, A, lda, B, ldb, pp.ps,
                           C, ldc, M, ms, mstride, ms, ns, pp.kk, st, true, ks);
        if (rc == FMM_OK) rc = launch_combine(plan, *d, C, ldc, ms, ns, M, ms, mstride, st);
        if (pp.ws) {
          cudaError_t fe = cudaFreeAsync(pp.ws, st);
          if (rc == FMM_OK) rc = cuda_status(fe);
        }
        cudaError_t fe = cudaFreeAsync(mws, st);
        if (rc == FMM_OK) rc = cuda_status(fe);
      } else if (use_presum(plan, ms, ns, ks) && (long long)presum_bytes(plan, ms, ns, ks) > g_ws_limit.load()) {
        rc = run_presum_groups(plan, *d, A, lda, B, ldb, C, ldc, ms, ns, ks, st);  // workspace within the limit
      } else if (use_presum(plan, ms, ns, ks)) {
        // U/V sums formed once per product in HBM (bandwidth-bound), then every
        // product reads single operands; products scattered into C in the epilogue.
        t_last_ws = (long long)presum_bytes(plan, ms, ns, ks);
        PresumPlan pp;
        rc = presum_prepare(plan, *d, A, lda, B, ldb, ms, ns, ks, st, &pp);
        const int S = call_ksplit(plan, ms, ns, ks, true, pp.kk, sm_count_current());
        const fmm::Prod* vp = pp.prods;
        const fmm::Term* vt = pp.terms;
        if (rc == FMM_OK && S > 1) rc = ksplit_tables(plan, pp.kk != ks ? BASE_ALL : BASE_PS, S, &vp, &vt);
        if (rc == FMM_OK)
          rc = launch_gemm(K_GEMM_FMM, vp, vt, plan->dims, R * S, fmm::MODE_ACCUM_C, A, lda, B, ldb, pp.ps, C, ldc,
                           nullptr, 0, 0, ms, ns, pp.kk, st, true, ks, S);
        if (pp.ws) {
          cudaError_t fe = cudaFreeAsync(pp.ws, st);
          if (rc == FMM_OK) rc = cuda_status(fe);
        }
      } else {
        rc = launch_gemm(K_GEMM_FMM, d->prods, d->terms, plan->dims, R, fmm::MODE_ACCUM_C, A, lda, B, ldb,
                         PresumOps{}, C, ldc, nullptr, 0, 0, ms, ns, ks, st);
      }
      if (rc != FMM_OK) return rc;
    } else {
      const long long mstride = (long long)ms * ns;
      size_t bytes = sizeof(double) * (size_t)mstride * R;
      size_t s_bytes = 0, t_bytes = 0;
      if (pack == FMM_PACK_NAIVE) {
        s_bytes = sizeof(double) * (size_t)ms * ks * R;
        t_bytes = sizeof(double) * (size_t)ks * ns * R;
      }
      char* ws = nullptr;
      FMM_CUDA_TRY(cudaMallocAsync((void**)&ws, bytes + s_bytes + t_bytes, st));
      double* M = reinterpret_cast<double*>(ws);
      if (pack == FMM_PACK_AB && use_presum(plan, ms, ns, ks)) {
        // large sub-blocks: operands pre-summed as for ABC, each product stored to M by the
        // direct variant, W applied by the combine pass below
        PresumPlan pp;
        rc = presum_prepare(plan, *d, A, lda, B, ldb, ms, ns, ks, st, &pp);
        if (rc == FMM_OK)
          rc = launch_gemm(K_GEMM_FMM, pp.prods, pp.terms, plan->dims, R, fmm::MODE_STORE_M, A, lda, B, ldb, pp.ps,
                           C, ldc, M, ms, mstride, ms, ns, pp.kk, st, true, ks);
        if (pp.ws) {
          cudaError_t fe = cudaFreeAsync(pp.ws, st);
          if (rc == FMM_OK) rc = cuda_status(fe);
        }
      } else if (pack == FMM_PACK_AB) {
        rc = launch_gemm(K_GEMM_FMM, d->prods, d->terms, plan->dims, R, fmm::MODE_STORE_M, A, lda, B, ldb,
                         PresumOps{}, C, ldc, M, ms, mstride, ms, ns, ks, st);
      } else {
        double* S = reinterpret_cast<double*>(ws + bytes);
        double* T = reinterpret_cast<double*>(ws + bytes + s_bytes);
        fmm::LincombArgs la{};
        la.X = A;
        la.ldx = lda;
        la.rows = ms;
        la.cols = ks;
        la.blk_row_stride = ms;
        la.blk_col_stride = ks;
        la.out = S;
        la.ldo = ms;
        la.out_stride = (long long)ms * ks;
        la.prods = d->prods;
        la.terms = d->terms;
        la.side = 0;
        la.plist = nullptr;
        rc = launch_lincomb(plan, la, R, st);
        fmm::LincombArgs lb = la;
        lb.X = B;
        lb.ldx = ldb;
        lb.rows = ks;
        lb.cols = ns;
        lb.blk_row_stride = ks;
        lb.blk_col_stride = ns;
        lb.out = T;
        lb.ldo = ks;
        lb.out_stride = (long long)ks * ns;
        lb.side = 1;
        if (rc == FMM_OK) rc = launch_lincomb(plan, lb, R, st);
        // Product r: M_r = S_r * T_r, with S_r the block (0, r) of an ms x (R*ks) matrix.
        if (rc == FMM_OK) {
          DevTables* dc = nullptr;
          rc = device_tables(classical_plan(), &dc);
          for (int r = 0; rc == FMM_OK && r < R; ++r) {
            rc = launch_gemm(K_GEMM_FMM, dc->prods, dc->terms, kUnitGrid, 1, fmm::MODE_STORE_M,
                             S + (long long)r * ms * ks, ms, T + (long long)r * ks * ns, ks, PresumOps{}, nullptr, 0,
                             M + (long long)r * mstride, ms, 0, ms, ns, ks, st);
          }
        }
      }
      if (rc == FMM_OK && combine_fits(plan)) {
        rc = launch_combine(plan, *d, C, ldc, ms, ns, M, ms, mstride, st);
      } else if (rc == FMM_OK) {
        fmm::ScatterArgs sa{};
        sa.C = C;
        sa.ldc = ldc;
        sa.ms = ms;
        sa.ns = ns;
        sa.M = M;
        sa.ldm = ms;
        sa.m_stride = mstride;
        sa.cblk = d->cblk;
        sa.ent_r = d->ent_r;
        sa.ent_w = d->ent_w;
        const dim3 gs((unsigned)grid_for(mstride, 256), (unsigned)plan->n_cblk);
        {
          ProfScope ps(K_SCATTER, st);
          fmm::fmm_scatter_kernel<<<gs, 256, 0, st>>>(sa);
        }
        g_launches.fetch_add(1, std::memory_order_relaxed);
        rc = cuda_status(cudaGetLastError());
      }
      cudaError_t fe = cudaFreeAsync(ws, st);
      if (rc == FMM_OK) rc = cuda_status(fe);
      if (rc != FMM_OK) return rc;
    }
  }
  return peel(m, n, k, A, lda, B, ldb, C, ldc, pm, pk, pn, st);
}

int noalloc_status(int dev, bool clear);  // the no-allocation entry point's status word (below)

int device_status(bool clear) {
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return FMM_E_UNSUPPORTED;
  unsigned v = 0;
  if (smem_configured[dev]) {
    FMM_CUDA_TRY(cudaMemcpy(&v, dev_status[dev], sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (clear && v) FMM_CUDA_TRY(cudaMemset(dev_status[dev], 0, sizeof(unsigned)));
  }
  const int rn = noalloc_status(dev, clear);
  if (rn != FMM_OK && rn != FMM_E_TIMEOUT) return rn;
  if (v & fmm::STATUS_TABLE) return FMM_E_PLAN;
  return (v || rn == FMM_E_TIMEOUT) ? FMM_E_TIMEOUT : FMM_OK;
}

// Host-pointer execution: stage A, B, C into device memory, run, copy C back.
//
// Large problems run as a grid of R row panels x P column panels of C, each block
// C[I, J] += A[I, :] * B[:, J] a GEMM of its own (partitioned like any |I| x |J| x k call), so
// that the copies overlap the compute.  Blocks run column panel by column panel, the row
// panels inside: the copy-in stream brings, in that order, each block's operands that are not
// on the device yet (A[I, :] at its first use, B[:, J] at its first use, C[I, J]); the
// calling thread's stream computes block b once its copies have landed while the next
// blocks' operands come in; a copy-out stream returns C[I, J] after its block (host-to-
// device and device-to-host copies run at the same time).  Before the first kernel only
// A[I_0, :], B[:, J_0] and C[I_0, J_0] are copied: with two row panels half of A instead of
// all of it (16384^3: 1.8 instead of 3.2 GB).  Row and column edges fall on multiples of 128 x
// (block rows / columns of the plan), so every block's sub-blocks are whole 128-row tiles
// where the size allows.
#ifndef FMM_HOST_PANELS
#define FMM_HOST_PANELS 4
#endif
constexpr int kHostPanelMinCols = 2048;              // column panels at least this wide
constexpr long long kHostPanelMinElems = 1LL << 22;  // C of at least 32 MB
constexpr long long kHostRowSplitMinA = 1LL << 26;   // two row panels once A has 2^26 elements (512 MB)
constexpr int kHostRowPanelMinRows = 4096;

void split_edges(int total, int parts, int unit, std::vector<int>* edges) {
  edges->assign(1, 0);
  for (int j = 1; j < parts; ++j) {
    long long e = (long long)total * j / parts;
    if (total / parts >= unit) e -= e % unit;
    if (e > edges->back() && e < total) edges->push_back((int)e);
  }
  edges->push_back(total);
}

int host_panels(const fmm_plan* plan, bool plain, int m, int n, int k, std::vector<int>* rows,
                std::vector<int>* cols) {
  int P = 1, R = 1;
  if ((long long)m * n >= kHostPanelMinElems) P = std::max(1, std::min(FMM_HOST_PANELS, n / kHostPanelMinCols));
  if (P > 1 && (long long)m * k >= kHostRowSplitMinA && m >= 2 * kHostRowPanelMinRows) R = 2;
  split_edges(m, R, 128 * ((plain || !plan) ? 1 : plan->dims[0]), rows);
  split_edges(n, P, 128 * ((plain || !plan) ? 1 : plan->dims[2]), cols);
  return (int)(rows->size() - 1) * (int)(cols->size() - 1);
}

int run_host(const fmm_plan* plan, int pack, bool plain, int m, int n, int k, const double* A, int lda,
             const double* B, int ldb, double* C, int ldc) {
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK) return rc;
  if (m == 0 || n == 0 || k == 0) return FMM_OK;
  if (!plain && !plan) return FMM_E_NOPLAN;
  cudaStream_t st = cudaStreamPerThread;
  // even device pitches for A and B: tensor copies need 16-byte column starts
  const int pa = m + (m & 1), pb = k + (k & 1);
  const size_t szA = sizeof(double) * (size_t)pa * k, szB = sizeof(double) * (size_t)pb * n,
               szC = sizeof(double) * (size_t)m * n;
  std::vector<int> re, ce;
  const int NB = host_panels(plan, plain, m, n, k, &re, &ce);
  const int R = (int)re.size() - 1;
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  cudaStream_t sin = nullptr, sout = nullptr;
  std::vector<cudaEvent_t> ev;  // [0]: allocations made; [1 + b]: block b copied in; [1 + NB + b]: block b done
  auto ok = [&](cudaError_t e) {
    if (rc == FMM_OK && e != cudaSuccess) rc = cuda_status(e);
    return rc == FMM_OK;
  };
  ok(cudaMallocAsync((void**)&dA, szA, st)) && ok(cudaMallocAsync((void**)&dB, szB, st)) &&
      ok(cudaMallocAsync((void**)&dC, szC, st));
  if (rc == FMM_OK && NB > 1) {
    ok(cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking)) &&
        ok(cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking));
    ev.assign(1 + 2 * NB, nullptr);
    for (auto& e : ev)
      if (!ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) break;
  }
  cudaStream_t cin = NB > 1 ? sin : st, cout = NB > 1 ? sout : st;
  if (rc == FMM_OK && NB > 1) ok(cudaEventRecord(ev[0], st)) && ok(cudaStreamWaitEvent(sin, ev[0], 0));
  // block b = column panel b / R, row panel b % R
  for (int b = 0; b < NB && rc == FMM_OK; ++b) {
    const int i = b % R, j = b / R;
    const int r0 = re[i], mi = re[i + 1] - re[i], c0 = ce[j], nj = ce[j + 1] - ce[j];
    if (j == 0)  // A[I, :] at its first use
      ok(cudaMemcpy2DAsync(dA + r0, sizeof(double) * pa, A + r0, sizeof(double) * lda, sizeof(double) * mi, k,
                           cudaMemcpyHostToDevice, cin));
    if (i == 0 && rc == FMM_OK)  // B[:, J] at its first use
      ok(cudaMemcpy2DAsync(dB + (size_t)c0 * pb, sizeof(double) * pb, B + (size_t)c0 * ldb, sizeof(double) * ldb,
                           sizeof(double) * k, nj, cudaMemcpyHostToDevice, cin));
    if (rc == FMM_OK)
      ok(cudaMemcpy2DAsync(dC + r0 + (size_t)c0 * m, sizeof(double) * m, C + r0 + (size_t)c0 * ldc,
                           sizeof(double) * ldc, sizeof(double) * mi, nj, cudaMemcpyHostToDevice, cin));
    if (NB > 1 && rc == FMM_OK) ok(cudaEventRecord(ev[1 + b], sin));
  }
  for (int b = 0; b < NB && rc == FMM_OK; ++b) {
    const int i = b % R, j = b / R;
    const int r0 = re[i], mi = re[i + 1] - re[i], c0 = ce[j], nj = ce[j + 1] - ce[j];
    if (NB > 1 && !ok(cudaStreamWaitEvent(st, ev[1 + b], 0))) break;
    double* Cb = dC + r0 + (size_t)c0 * m;
    rc = plain ? plain_gemm(mi, nj, k, dA + r0, pa, dB + (size_t)c0 * pb, pb, Cb, m, st)
               : run_fmm(plan, pack, mi, nj, k, dA + r0, pa, dB + (size_t)c0 * pb, pb, Cb, m, st);
    if (rc != FMM_OK) break;
    if (NB > 1) ok(cudaEventRecord(ev[1 + NB + b], st)) && ok(cudaStreamWaitEvent(sout, ev[1 + NB + b], 0));
    if (rc == FMM_OK)
      ok(cudaMemcpy2DAsync(C + r0 + (size_t)c0 * ldc, sizeof(double) * ldc, Cb, sizeof(double) * m,
                           sizeof(double) * mi, nj, cudaMemcpyDeviceToHost, cout));
  }
  // join: every copy has finished before the buffers go back to the pool
  if (sin) ok(cudaStreamSynchronize(sin));
  if (sout) ok(cudaStreamSynchronize(sout));
  if (dA) cudaFreeAsync(dA, st);
  if (dB) cudaFreeAsync(dB, st);
  if (dC) cudaFreeAsync(dC, st);
  ok(cudaStreamSynchronize(st));
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  if (sin) cudaStreamDestroy(sin);
  if (sout) cudaStreamDestroy(sout);
  if (rc == FMM_OK) rc = device_status(true);
  return rc;
}

// Operands whose leading dimension is odd cannot be staged by tensor copies (columns
// must start on 16 bytes) and fall back to per-thread copies at about half the speed.
// Large ones are copied once, stream-ordered, into an even-pitch workspace instead
// (bandwidth-bound, a few percent of the GEMM); small ones stay in place.
constexpr long long kRepitchMinElems = 1LL << 18;

struct Repitched {
  const double* A;
  long long lda;
  const double* B;
  long long ldb;
  char* ws = nullptr;
};

int repitch(int m, int n, int k, const double* A, long long lda, const double* B, long long ldb, cudaStream_t st,
            Repitched* out) {
  out->A = A;
  out->lda = lda;
  out->B = B;
  out->ldb = ldb;
  const bool a_odd = (lda & 1) && (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (long long)m * k >= kRepitchMinElems;
  const bool b_odd = (ldb & 1) && (reinterpret_cast<uintptr_t>(B) & 15) == 0 && (long long)k * n >= kRepitchMinElems;
  if (!a_odd && !b_odd) return FMM_OK;
  const long long pa = m + (m & 1), pb = k + (k & 1);
  const size_t sa = a_odd ? ((sizeof(double) * (size_t)pa * k + 255) & ~(size_t)255) : 0;
  const size_t sb = b_odd ? sizeof(double) * (size_t)pb * n : 0;
  FMM_CUDA_TRY(cudaMallocAsync((void**)&out->ws, sa + sb, st));
  if (a_odd) {
    double* dst = reinterpret_cast<double*>(out->ws);
    fmm::fmm_pitch_copy1_kernel<<<256, 256, 0, st>>>(fmm::PitchCopy{A, lda, dst, pa, m, k});
    g_launches.fetch_add(1, std::memory_order_relaxed);
    out->A = dst;
    out->lda = pa;
  }
  if (b_odd) {
    double* dst = reinterpret_cast<double*>(out->ws + sa);
    fmm::fmm_pitch_copy1_kernel<<<256, 256, 0, st>>>(fmm::PitchCopy{B, ldb, dst, pb, k, n});
    g_launches.fetch_add(1, std::memory_order_relaxed);
    out->B = dst;
    out->ldb = pb;
  }
  return cuda_status(cudaGetLastError());
}

int release(Repitched& r, int rc, cudaStream_t st) {
  if (!r.ws) return rc;
  cudaError_t e = cudaFreeAsync(r.ws, st);
  return rc == FMM_OK ? cuda_status(e) : rc;
}

}  // namespace

extern "C" {

int fmm_plan_create(const int dims[3], int rank, const int* nterms, const int* rows, const int* cols,
                    const double* coefs, fmm_plan** out) {
  return build_plan(dims, rank, nterms, rows, cols, coefs, out);
}

int fmm_plan_destroy(fmm_plan* plan) {
  if (!plan) return FMM_E_INVALID;
  {
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (g_default_plan == plan) g_default_plan = nullptr;
  }
  for (auto& d : plan->dev) {
    if (!d.ready) continue;
    cudaFree(d.prods);
    cudaFree(d.terms);
    cudaFree(d.cblk);
    cudaFree(d.ent_r);
    cudaFree(d.ent_w);
    cudaFree(d.cg_desc);
    cudaFree(d.cg_r);
    cudaFree(d.cg_m);
    cudaFree(d.cg_c);
    cudaFree(d.ch_r);
    cudaFree(d.ch_m);
    cudaFree(d.ch_c);
    cudaFree(d.prods_ps);
    cudaFree(d.terms_ps);
    cudaFree(d.plistA);
    cudaFree(d.plistB);
    cudaFree(d.prods_all);
    cudaFree(d.terms_all);
    cudaFree(d.plist_all);
  }
  for (auto& t : plan->ksplit) {
    cudaFree(t.prods);
    cudaFree(t.terms);
  }
  delete plan;
  return FMM_OK;
}

int fmm_plan_rank(const fmm_plan* plan) { return plan ? plan->rank : FMM_E_INVALID; }

int fmm_plan_combine_info(const fmm_plan* plan, int* groups, int* entries, int* chunks) {
  if (!plan) return FMM_E_INVALID;
  if (groups) *groups = plan->n_cgroup;
  if (entries) *entries = plan->n_cgroup ? (int)plan->cg_r.size() : 0;
  if (chunks) *chunks = plan->n_cgroup ? (int)plan->ch_m.size() : 0;
  return FMM_OK;
}

int fmm_bind_default_plan(fmm_plan* plan) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  g_default_plan = plan;
  return FMM_OK;
}

fmm_plan* fmm_default_plan(void) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  return g_default_plan;
}

int fmm_dgemm_dev(const fmm_plan* plan, int pack_type, int m, int n, int k, const double* A, long lda,
                  const double* B, long ldb, double* C, long ldc, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK || m == 0 || n == 0 || k == 0 || !plan) return run_fmm(plan, pack_type, m, n, k, A, lda, B, ldb, C, ldc, st);
  Repitched r;
  rc = repitch(m, n, k, A, lda, B, ldb, st, &r);
  if (rc == FMM_OK) rc = run_fmm(plan, pack_type, m, n, k, r.A, r.lda, r.B, r.ldb, C, ldc, st);
  return release(r, rc, st);
}

int fmm_plain_dgemm_dev(int m, int n, int k, const double* A, long lda, const double* B, long ldb, double* C,
                        long ldc, void* stream) {
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK || m == 0 || n == 0 || k == 0) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Repitched r;
  rc = repitch(m, n, k, A, lda, B, ldb, st, &r);
  if (rc == FMM_OK) rc = plain_gemm(m, n, k, r.A, r.lda, r.B, r.ldb, C, ldc, st);
  return release(r, rc, st);
}

int fmm_dgemm_host(const fmm_plan* plan, int pack_type, int m, int n, int k, const double* A, int lda,
                   const double* B, int ldb, double* C, int ldc) {
  return run_host(plan, pack_type, false, m, n, k, A, lda, B, ldb, C, ldc);
}

void bl_dgemm(int m, int n, int k, double* A, int lda, double* B, int ldb, double* C, int ldc) {
  t_last_error = run_host(nullptr, 0, true, m, n, k, A, lda, B, ldb, C, ldc);
}

void bl_dgemm_strassen_abc(int m, int n, int k, double* A, int lda, double* B, int ldb, double* C, int ldc) {
  t_last_error = run_host(fmm_default_plan(), FMM_PACK_ABC, false, m, n, k, A, lda, B, ldb, C, ldc);
}

void bl_dgemm_strassen_ab(int m, int n, int k, double* A, int lda, double* B, int ldb, double* C, int ldc) {
  t_last_error = run_host(fmm_default_plan(), FMM_PACK_AB, false, m, n, k, A, lda, B, ldb, C, ldc);
}

void bl_dgemm_strassen_naive(int m, int n, int k, double* A, int lda, double* B, int ldb, double* C, int ldc) {
  t_last_error = run_host(fmm_default_plan(), FMM_PACK_NAIVE, false, m, n, k, A, lda, B, ldb, C, ldc);
}

void bl_dynamic_peeling(int m, int n, int k, double* A, int lda, double* B, int ldb, double* C, int ldc, int dim1,
                        int dim2, int dim3) {
  if (dim1 <= 0 || dim2 <= 0 || dim3 <= 0) {
    t_last_error = FMM_E_INVALID;
    return;
  }
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK || m == 0 || n == 0 || k == 0) {
    t_last_error = rc;
    return;
  }
  cudaStream_t st = cudaStreamPerThread;
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  const int pa = m + (m & 1), pb = k + (k & 1);  // even device pitches (16-byte column starts)
  const size_t szA = sizeof(double) * (size_t)pa * k, szB = sizeof(double) * (size_t)pb * n,
               szC = sizeof(double) * (size_t)m * n;
  rc = cuda_status(cudaMallocAsync((void**)&dA, szA, st));
  if (rc == FMM_OK) rc = cuda_status(cudaMallocAsync((void**)&dB, szB, st));
  if (rc == FMM_OK) rc = cuda_status(cudaMallocAsync((void**)&dC, szC, st));
  if (rc == FMM_OK)
    rc = cuda_status(cudaMemcpy2DAsync(dA, sizeof(double) * pa, A, sizeof(double) * lda, sizeof(double) * m, k,
                                       cudaMemcpyHostToDevice, st));
  if (rc == FMM_OK)
    rc = cuda_status(cudaMemcpy2DAsync(dB, sizeof(double) * pb, B, sizeof(double) * ldb, sizeof(double) * k, n,
                                       cudaMemcpyHostToDevice, st));
  if (rc == FMM_OK)
    rc = cuda_status(cudaMemcpy2DAsync(dC, sizeof(double) * m, C, sizeof(double) * ldc, sizeof(double) * m, n,
                                       cudaMemcpyHostToDevice, st));
  if (rc == FMM_OK) rc = peel(m, n, k, dA, pa, dB, pb, dC, m, dim1, dim2, dim3, st);
  if (rc == FMM_OK)
    rc = cuda_status(cudaMemcpy2DAsync(C, sizeof(double) * ldc, dC, sizeof(double) * m, sizeof(double) * m, n,
                                       cudaMemcpyDeviceToHost, st));
  if (dA) cudaFreeAsync(dA, st);
  if (dB) cudaFreeAsync(dB, st);
  if (dC) cudaFreeAsync(dC, st);
  cudaError_t se = cudaStreamSynchronize(st);
  if (rc == FMM_OK) rc = cuda_status(se);
  if (rc == FMM_OK) rc = device_status(true);
  t_last_error = rc;
}

int fmm_last_error(void) { return t_last_error; }

const char* fmm_error_string(int code) {
  switch (code) {
    case FMM_OK: return "ok";
    case FMM_E_INVALID: return "invalid argument (dimension, leading dimension or pointer)";
    case FMM_E_NOPLAN: return "no FMM plan bound";
    case FMM_E_CUDA: return "CUDA runtime error";
    case FMM_E_NOMEM: return "out of memory";
    case FMM_E_PLAN: return "malformed plan tables";
    case FMM_E_UNSUPPORTED: return "unsupported pack type or option";
    case FMM_E_TIMEOUT: return "device-side wait timed out";
    case FMM_E_TOO_LARGE: return "problem exceeds the no-allocation scratch limits";
    default: return "unknown error";
  }
}

long long fmm_kernel_launch_count(void) { return g_launches.load(); }

int fmm_device_status(int clear) { return device_status(clear != 0); }

long long fmm_set_workspace_limit(long long bytes) {
  return g_ws_limit.exchange(bytes > 0 ? bytes : kDefaultWorkspaceLimit);
}

long long fmm_last_workspace_bytes(void) { return t_last_ws; }

int fmm_debug_set(int what, long long value) {
  switch (what) {
    case FMM_DEBUG_WAIT_LIMIT_NS: {
      const unsigned long long v = value > 0 ? (unsigned long long)value : fmm::WAIT_LIMIT_NS;
      FMM_CUDA_TRY(cudaMemcpyToSymbol(fmm::g_wait_limit_ns, &v, sizeof(v)));
      return FMM_OK;
    }
    case FMM_DEBUG_TICKET_FILL:
      if (value < 0 || value > 255) return FMM_E_INVALID;
      g_ticket_fill = (int)value;
      return FMM_OK;
    case FMM_DEBUG_SPLIT_OPERANDS:
      if (value < 0 || value > 1) return FMM_E_INVALID;
      g_split_form = (int)value;
      return FMM_OK;
    case FMM_DEBUG_KSPLIT:
      if (value < 0 || value > 8) return FMM_E_INVALID;
      g_force_ksplit = (int)value;
      return FMM_OK;
    case FMM_DEBUG_COMBINE_POSITIONS:
      if (value < 0 || value > 2) return FMM_E_INVALID;
      g_combine_positions = (int)value;
      return FMM_OK;
    default:
      return FMM_E_INVALID;
  }
}

int fmm_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof) {
    cudaEventDestroy(r.e0);
    cudaEventDestroy(r.e1);
  }
  g_prof.clear();
  g_prof_on = true;
  return FMM_OK;
}

int fmm_profile_end(double* ms_out, long long* count_out) {
  std::vector<ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = false;
    recs.swap(g_prof);
  }
  for (int k = 0; k < K_NUM; ++k) {
    if (ms_out) ms_out[k] = 0.0;
    if (count_out) count_out[k] = 0;
  }
  int rc = FMM_OK;
  for (auto& r : recs) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(r.e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.e0, r.e1);
    if (e != cudaSuccess) rc = cuda_status(e);
    if (ms_out) ms_out[r.kind] += ms;
    if (count_out) count_out[r.kind] += 1;
    cudaEventDestroy(r.e0);
    cudaEventDestroy(r.e1);
  }
  return rc;
}

int fmm_profile_num_kinds(void) { return K_NUM; }

const char* fmm_profile_kind_name(int kind) { return (kind >= 0 && kind < K_NUM) ? kKernelNames[kind] : ""; }

}  // extern "C"

// ------------------------------------------------------------------------------------
// No-allocation entry point.
//
// Some callers cannot allocate device memory when they call us: frameworks that own the
// whole device memory through their own arena or caching allocator and forbid foreign
// cudaMalloc calls (an allocation behind their back can fail or fragment their pool),
// and code on latency-critical paths where an allocation (or the synchronisation a
// cudaFree implies) is not acceptable.  fmm_dgemm_dev_noalloc() serves them: it runs the
// ABC FMM with the operand sums folded during staging (no pre-summed workspace), and
// keeps the only scratch the kernel needs -- per-tile tickets, a work-unit counter, the status word --
// and the plan tables in one statically allocated device array.
// ------------------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxTiles = 16384;   // tile positions (128 x 128) of one call
constexpr int kNoAllocMaxProds = 1024;    // products of a plan
constexpr int kNoAllocMaxTerms = 12288;   // A, B and C terms of a plan
constexpr size_t kNoAllocTicketsOff = 0;
constexpr size_t kNoAllocStatusOff = kNoAllocTicketsOff + sizeof(int) * kNoAllocMaxTiles;
constexpr size_t kNoAllocCounterOff = kNoAllocStatusOff + 128;  // a launch's work-unit counter
constexpr size_t kNoAllocProdsOff = kNoAllocStatusOff + 256;
constexpr size_t kNoAllocTermsOff = kNoAllocProdsOff + sizeof(fmm::Prod) * (kNoAllocMaxProds + 1);
constexpr size_t kNoAllocBytes = kNoAllocTermsOff + sizeof(fmm::Term) * (kNoAllocMaxTerms + 3);

}  // namespace

// Every GPU that loads this library holds this array (about 384 KB) until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices];  // device address of g_noalloc_scratch, per device
bool g_noalloc_ready[kMaxDevices];

// Once per device, with that device current: resolve the array's device address (in host
// code the symbol is only a host-side stand-in) and configure the kernels.  Nothing here
// allocates device memory.
int noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (g_noalloc_ready[dev]) return FMM_OK;
  void* p = nullptr;
  FMM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  if (p == nullptr) return FMM_E_CUDA;
  FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)fmm::smem_bytes(false)));
  FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)fmm::smem_bytes(true)));
  int nsm = 0;
  FMM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  {
    std::lock_guard<std::mutex> lk2(g_attr_mu);
    if (sm_count[dev] == 0) sm_count[dev] = nsm;
    if (!g_encode_tiled) {
      cudaDriverEntryPointQueryResult q;
      void* fn = nullptr;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
          q == cudaDriverEntryPointSuccess)
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
  }
  // The classical product used by the fringe strips never changes: its tables (product
  // index kNoAllocMaxProds, terms after the plan's) are written here once, and the status
  // word starts at zero.  Both copies are blocking, from memory that outlives them.
  static const fmm::Prod classic{kNoAllocMaxTerms, 1, kNoAllocMaxTerms + 1, 1, kNoAllocMaxTerms + 2, 1};
  static const fmm::Term classic_terms[3] = {{0, 0, 1.0, 0, 0}, {0, 0, 1.0, 0, 0}, {0, 0, 1.0, 0, 0}};
  unsigned char* base = static_cast<unsigned char*>(p);
  FMM_CUDA_TRY(cudaMemcpy(base + kNoAllocProdsOff + sizeof(fmm::Prod) * kNoAllocMaxProds, &classic, sizeof(classic),
                          cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemcpy(base + kNoAllocTermsOff + sizeof(fmm::Term) * kNoAllocMaxTerms, classic_terms,
                          sizeof(classic_terms), cudaMemcpyHostToDevice));
  FMM_CUDA_TRY(cudaMemset(base + kNoAllocStatusOff, 0, sizeof(unsigned)));
  g_noalloc_ptr[dev] = base;
  g_noalloc_ready[dev] = true;
  return FMM_OK;
}

int noalloc_status(int dev, bool clear) {
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ready[dev]) return FMM_OK;
    base = g_noalloc_ptr[dev];
  }
  unsigned v = 0;
  FMM_CUDA_TRY(cudaMemcpy(&v, base + kNoAllocStatusOff, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (clear && v) FMM_CUDA_TRY(cudaMemset(base + kNoAllocStatusOff, 0, sizeof(unsigned)));
  return v ? FMM_E_TIMEOUT : FMM_OK;
}

// One launch of fmm_gemm_kernel in MODE_ACCUM_C with caller-provided tables, tickets and
// status word (nothing allocated).
int noalloc_launch(const fmm::Prod* prods, const fmm::Term* terms, const int grid_dims[3], int nprod,
                   const double* A, long long lda, const double* B, long long ldb, double* C, long long ldc,
                   int ms, int ns, int ks, int* tickets, unsigned* status, int* counter, int nsm, cudaStream_t st) {
  if (ms <= 0 || ns <= 0 || ks <= 0 || nprod <= 0) return FMM_OK;
  fmm::GemmArgs a{};
  a.A = A;
  a.lda = lda;
  a.B = B;
  a.ldb = ldb;
  a.Aw = A;
  a.ldaw = lda;
  a.Bw = B;
  a.ldbw = ldb;
  a.C = C;
  a.ldc = ldc;
  a.ms = ms;
  a.ns = ns;
  a.ks = ks;
  a.prods = prods;
  a.terms = terms;
  a.nprod = nprod;
  a.tiles_m = (ms + fmm::BM - 1) / fmm::BM;
  a.tiles_n = (ns + fmm::BN - 1) / fmm::BN;
  a.mode = fmm::MODE_ACCUM_C;
  a.status = status;
  const int ntiles = a.tiles_m * a.tiles_n;
  a.chunks = choose_chunks(ntiles, nprod, nsm);
  a.tickets = tickets;
  if (a.chunks > 1 && ntiles > kNoAllocMaxTiles) return FMM_E_TOO_LARGE;  // tickets of one launch must fit
  if (a.chunks > 1) FMM_CUDA_TRY(cudaMemsetAsync(tickets, 0, sizeof(int) * ntiles, st));
  a.counter = counter;
  FMM_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), st));
  const long long units = (long long)ntiles * a.chunks;
  const unsigned grid = (unsigned)(units < nsm ? units : nsm);
  const long long am = (long long)grid_dims[0] * ms, ak = (long long)grid_dims[1] * ks,
                  bn = (long long)grid_dims[2] * ns;
  const bool tma = make_tensor_map(&a.tmA, A, am, ak, lda, fmm::BM, fmm::BK) &&
                   make_tensor_map(&a.tmB, B, ak, bn, ldb, fmm::BK, fmm::BN) &&
                   make_tensor_map(&a.tmB2, B, ak, bn, ldb, fmm::TB_K, fmm::BN);
  a.tmAw = a.tmA;
  a.tmBw = a.tmB;
  a.tmBw2 = a.tmB2;
  if (tma)
    fmm::fmm_gemm_kernel<true><<<grid, fmm::NTHREADS, fmm::smem_bytes(true), st>>>(a);
  else
    fmm::fmm_gemm_kernel<false><<<grid, fmm::NTHREADS, fmm::smem_bytes(false), st>>>(a);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cuda_status(cudaGetLastError());
}

}  // namespace

extern "C" int fmm_dgemm_dev_noalloc(const fmm_plan* plan, int m, int n, int k, const double* A, long lda,
                                     const double* B, long ldb, double* C, long ldc, void* stream, int sync) {
  if (!plan) return FMM_E_NOPLAN;
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK) return rc;
  if (m == 0 || n == 0 || k == 0) return FMM_OK;
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return FMM_E_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // size limits of the static scratch
  const int pm = plan->dims[0] * kMR, pk = plan->dims[1], pn = plan->dims[2] * kNR;
  const int md = m - m % pm, kd = k - k % pk, nd = n - n % pn;
  const int ms = md / plan->dims[0], ks = kd / plan->dims[1], ns = nd / plan->dims[2];
  const long long tiles_fmm = (long long)((ms + fmm::BM - 1) / fmm::BM) * ((ns + fmm::BN - 1) / fmm::BN);
  if ((int)plan->prods.size() > kNoAllocMaxProds || (int)plan->terms.size() > kNoAllocMaxTerms ||
      tiles_fmm > kNoAllocMaxTiles)
    return FMM_E_TOO_LARGE;
  rc = noalloc_setup(dev);
  if (rc != FMM_OK) return rc;
  unsigned char* base = g_noalloc_ptr[dev];
  int* tickets = reinterpret_cast<int*>(base + kNoAllocTicketsOff);
  unsigned* status = reinterpret_cast<unsigned*>(base + kNoAllocStatusOff);
  int* counter = reinterpret_cast<int*>(base + kNoAllocCounterOff);
  fmm::Prod* prods = reinterpret_cast<fmm::Prod*>(base + kNoAllocProdsOff);
  fmm::Term* terms = reinterpret_cast<fmm::Term*>(base + kNoAllocTermsOff);
  // the plan's tables (from the plan's own storage, which outlives the copy); the classical
  // product of the fringe strips was written at set-up
  FMM_CUDA_TRY(cudaMemcpyAsync(prods, plan->prods.data(), sizeof(fmm::Prod) * plan->prods.size(),
                               cudaMemcpyHostToDevice, st));
  FMM_CUDA_TRY(cudaMemcpyAsync(terms, plan->terms.data(), sizeof(fmm::Term) * plan->terms.size(),
                               cudaMemcpyHostToDevice, st));
  const int nsm = sm_count[dev] > 0 ? sm_count[dev] : 148;
  rc = noalloc_launch(prods, terms, plan->dims, plan->rank, A, lda, B, ldb, C, ldc, ms, ns, ks, tickets, status,
                      counter, nsm, st);
  // fringe GEMMs (same regions and order as the reference's dynamic peeling)
  const int mr = m - md, kr = k - kd, nr = n - nd;
  const fmm::Prod* cp = prods + kNoAllocMaxProds;
  if (rc == FMM_OK && kr > 0 && md > 0 && nd > 0)
    rc = noalloc_launch(cp, terms, kUnitGrid, 1, A + (long long)kd * lda, lda, B + kd, ldb, C, ldc, md, nd, kr,
                        tickets, status, counter, nsm, st);
  if (rc == FMM_OK && nr > 0)
    rc = noalloc_launch(cp, terms, kUnitGrid, 1, A, lda, B + (long long)nd * ldb, ldb, C + (long long)nd * ldc, ldc, m,
                        nr, k, tickets, status, counter, nsm, st);
  if (rc == FMM_OK && mr > 0 && nd > 0)
    rc = noalloc_launch(cp, terms, kUnitGrid, 1, A + md, lda, B, ldb, C + md, ldc, mr, nd, k, tickets, status,
                        counter, nsm, st);
  // The status word is not cleared per call: a timeout recorded by a sync = 0 call stays
  // until a sync = 1 call or fmm_device_status() reports (and clears) it.
  if (rc == FMM_OK && sync) {
    unsigned v = 0;
    FMM_CUDA_TRY(cudaMemcpyAsync(&v, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (v) {
      FMM_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned), st));
      FMM_CUDA_TRY(cudaStreamSynchronize(st));
      rc = FMM_E_TIMEOUT;
    }
  }
  return rc;
}

// ---------------------------------------------------------------------------------------
// Split-BF16 FMM (tcgen05 tensor cores): FP32 A and B, FP64 C.  Same partition, product
// order and fringe peeling as the FP64 path; every GEMM (FMM core and fringe strips) runs
// as bf16 plane products with FP64 accumulation across 64-deep k chunks.
// ---------------------------------------------------------------------------------------
namespace {

bool split_configured[kMaxDevices];

int split_configure(int* dev_out) {
  int rc = configure_kernel(dev_out);
  if (rc != FMM_OK) return rc;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (!split_configured[*dev_out]) {
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmms::fmm_split_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmms::SMEM_BYTES));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmms::fmm_split_all_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      100 * 1024));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmms::fmm_split_all_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      100 * 1024));
    split_configured[*dev_out] = true;
  }
  return g_encode_tiled ? FMM_OK : FMM_E_UNSUPPORTED;
}

// bf16 planes (rows x kpad, row-major, pitch kpad) as a tensor map with box 64 x 128 and
// the 128-byte swizzle the UMMA descriptors expect.
bool make_plane_map(CUtensorMap* map, const __nv_bfloat16* base, long long rows, long long kpad) {
  if (rows <= 0 || rows >= (1LL << 32) || kpad % fmms::KPAD != 0) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kpad * sizeof(__nv_bfloat16)};
  cuuint32_t box[2] = {(cuuint32_t)fmms::BK, (cuuint32_t)fmms::BM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode_tiled(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims,
                              strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// One split-BF16 launch pair over sub-blocks ms x ks x ns of a plan (R products):
// operand planes into a stream-ordered workspace, then the persistent tcgen05 GEMM.
int split_core(const fmm_plan* plan, const DevTables& d, const float* A, long long lda, const float* B,
               long long ldb, double* C, long long ldc, int ms, int ns, int ks, cudaStream_t st) {
  if (ms <= 0 || ns <= 0 || ks <= 0) return FMM_OK;
  const int R = plan->rank;
  // several products: store each M_r, then one combine pass applies W (no C loads in the
  // tensor-core kernel's epilogue); a single product goes straight into C
  const bool use_m = R > 1 && combine_fits(plan);
  int dev = 0;
  int rc = split_configure(&dev);
  if (rc != FMM_OK) return rc;
  static_assert(fmms::BM == fmms::BN, "one box shape for both plane maps");
  const long long kpad = ((long long)ks + fmms::KPAD - 1) / fmms::KPAD * fmms::KPAD;
  const long long rows_a = 3LL * R * ms, rows_b = 3LL * R * ns;
  const int tiles_m = (ms + fmms::BM - 1) / fmms::BM, tiles_n = (ns + fmms::BN - 1) / fmms::BN;
  const long long ntiles = (long long)tiles_m * tiles_n;
  if (ntiles * R > INT32_MAX || (ms + fmms::SPLIT_ROWS - 1) / fmms::SPLIT_ROWS > 65535 ||
      (ns + fmms::SPLIT_ROWS - 1) / fmms::SPLIT_ROWS > 65535 || kpad / fmms::SPLIT_K > 65535)
    return FMM_E_UNSUPPORTED;
  const size_t bytes_a = sizeof(__nv_bfloat16) * (size_t)(rows_a * kpad);
  const size_t bytes_b = sizeof(__nv_bfloat16) * (size_t)(rows_b * kpad);
  const size_t bytes_m = use_m ? sizeof(double) * (size_t)R * ms * ns : 0;
  const size_t bytes_t = (R > 1 && !use_m) ? sizeof(int) * (size_t)ntiles : 0;
  char* ws = nullptr;
  // planes, product tiles, then the work-unit counter and the tickets
  FMM_CUDA_TRY(cudaMallocAsync((void**)&ws, bytes_a + bytes_b + bytes_m + sizeof(int) + bytes_t + 16, st));
  __nv_bfloat16* PA = reinterpret_cast<__nv_bfloat16*>(ws);
  __nv_bfloat16* PB = reinterpret_cast<__nv_bfloat16*>(ws + bytes_a);
  double* Mws = use_m ? reinterpret_cast<double*>(ws + bytes_a + bytes_b) : nullptr;
  int* counter = reinterpret_cast<int*>(ws + bytes_a + bytes_b + bytes_m);
  int* tickets = bytes_t ? counter + 1 : nullptr;
  rc = cuda_status(cudaMemsetAsync(counter, 0, sizeof(int) + bytes_t, st));

  fmms::SplitArgs sa{};
  sa.X = A;
  sa.ldx = lda;
  sa.rows = ms;
  sa.ks = ks;
  sa.kpad = (int)kpad;
  sa.blk_row_stride = ms;
  sa.blk_col_stride = ks;
  sa.out = PA;
  sa.prods = d.prods;
  sa.terms = d.terms;
  sa.side = 0;
  fmms::SplitArgs sb = sa;
  sb.X = B;
  sb.ldx = ldb;
  sb.rows = ns;
  sb.blk_row_stride = ks;
  sb.blk_col_stride = ns;
  sb.out = PB;
  sb.side = 1;
  // every product's sums from one read of each operand, where the staged tiles fit
  int nta = 0, ntb = 0;
  for (const auto& pr : plan->prods) nta += pr.na, ntb += pr.nb;
  const int nblk_a = plan->dims[0] * plan->dims[1], nblk_b = plan->dims[1] * plan->dims[2];
  const size_t sm_a = fmms::split_all_smem_bytes(0, nblk_a, R, nta), sm_b = fmms::split_all_smem_bytes(1, nblk_b, R, ntb);
  const bool all_form = g_split_form.load() == 0 && sm_a <= 100 * 1024 && sm_b <= 100 * 1024 && kpad % 64 == 0;
  if (rc == FMM_OK && all_form) {
    fmms::SplitAllArgs ga{sa, nblk_a, plan->dims[1], R, nta};
    fmms::SplitAllArgs gb{sb, nblk_b, plan->dims[2], R, ntb};
    ProfScope pf(K_SPLIT_OPERANDS, st);
    fmms::fmm_split_all_kernel<0><<<dim3((unsigned)(kpad / 32), (unsigned)((ms + 15) / 16)), 256, sm_a, st>>>(ga);
    fmms::fmm_split_all_kernel<1><<<dim3((unsigned)(kpad / 64), (unsigned)((ns + 7) / 8)), 256, sm_b, st>>>(gb);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    rc = cuda_status(cudaGetLastError());
  } else if (rc == FMM_OK) {
    ProfScope pf(K_SPLIT_OPERANDS, st);
    const dim3 blk(32, 8);
    const unsigned kt = (unsigned)(kpad / fmms::SPLIT_K);
    fmms::fmm_split_operands_kernel<<<dim3((unsigned)R, kt, (unsigned)((ms + fmms::SPLIT_ROWS - 1) / fmms::SPLIT_ROWS)),
                                      blk, 0, st>>>(sa);
    fmms::fmm_split_operands_kernel<<<dim3((unsigned)R, kt, (unsigned)((ns + fmms::SPLIT_ROWS - 1) / fmms::SPLIT_ROWS)),
                                      blk, 0, st>>>(sb);
    g_launches.fetch_add(2, std::memory_order_relaxed);
    rc = cuda_status(cudaGetLastError());
  }
  fmms::SplitGemmArgs g{};
  if (rc == FMM_OK && (!make_plane_map(&g.tmA, PA, rows_a, kpad) || !make_plane_map(&g.tmB, PB, rows_b, kpad)))
    rc = FMM_E_UNSUPPORTED;
  if (rc == FMM_OK) {
    g.C = C;
    g.ldc = ldc;
    g.ms = ms;
    g.ns = ns;
    g.kpad = (int)kpad;
    g.prods = d.prods;
    g.terms = d.terms;
    g.nprod = R;
    g.tiles_m = tiles_m;
    g.tiles_n = tiles_n;
    g.tickets = tickets;
    g.counter = counter;
    g.M = Mws;
    g.ldm = ms;
    g.m_stride = (long long)ms * ns;
    g.status = dev_status[dev];
    const long long units = ntiles * R;
    const unsigned grid = (unsigned)(units < sm_count[dev] ? units : sm_count[dev]);
    {
      ProfScope pf(K_GEMM_SPLIT, st);
      fmms::fmm_split_gemm_kernel<<<grid, fmms::NTHREADS, fmms::SMEM_BYTES, st>>>(g);
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    rc = cuda_status(cudaGetLastError());
  }
  if (rc == FMM_OK && use_m) rc = launch_combine(plan, d, C, ldc, ms, ns, Mws, ms, (long long)ms * ns, st);
  cudaError_t fe = cudaFreeAsync(ws, st);
  if (rc == FMM_OK) rc = cuda_status(fe);
  return rc;
}

int split_plain(int m, int n, int k, const float* A, long long lda, const float* B, long long ldb, double* C,
                long long ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0 || k <= 0) return FMM_OK;
  DevTables* d = nullptr;
  int rc = device_tables(classical_plan(), &d);
  if (rc != FMM_OK) return rc;
  return split_core(classical_plan(), *d, A, lda, B, ldb, C, ldc, m, n, k, st);
}

int run_split(const fmm_plan* plan, int m, int n, int k, const float* A, long long lda, const float* B,
              long long ldb, double* C, long long ldc, cudaStream_t st) {
  int rc = check_args(m, n, k, A, lda, B, ldb, C, ldc);
  if (rc != FMM_OK || m == 0 || n == 0 || k == 0) return rc;
  if (!plan) return split_plain(m, n, k, A, lda, B, ldb, C, ldc, st);
  const int pm = plan->dims[0] * kMR, pk = plan->dims[1], pn = plan->dims[2] * kNR;
  const int mr = m % pm, kr = k % pk, nr = n % pn;
  const int md = m - mr, kd = k - kr, nd = n - nr;
  if (md > 0 && nd > 0 && kd > 0) {
    DevTables* d = nullptr;
    rc = device_tables(plan, &d);
    if (rc != FMM_OK) return rc;
    rc = split_core(plan, *d, A, lda, B, ldb, C, ldc, md / plan->dims[0], nd / plan->dims[2], kd / plan->dims[1],
                    st);
    if (rc != FMM_OK) return rc;
  }
  // fringe strips: the same regions, in the same order, as the FP64 path's peeling
  if (kr > 0 && md > 0 && nd > 0) {
    rc = split_plain(md, nd, kr, A + (long long)kd * lda, lda, B + kd, ldb, C, ldc, st);
    if (rc != FMM_OK) return rc;
  }
  if (nr > 0) {
    rc = split_plain(m, nr, k, A, lda, B + (long long)nd * ldb, ldb, C + (long long)nd * ldc, ldc, st);
    if (rc != FMM_OK) return rc;
  }
  if (mr > 0 && nd > 0) rc = split_plain(mr, nd, k, A + md, lda, B, ldb, C + md, ldc, st);
  return rc;
}

}  // namespace

extern "C" int fmm_split_gemm_dev(const fmm_plan* plan, int m, int n, int k, const float* A, long lda,
                                  const float* B, long ldb, double* C, long ldc, void* stream) {
  return run_split(plan, m, n, k, A, lda, B, ldb, C, ldc, static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------------------
// Batches: many independent FP64 problems, each with its own plan (or classical), in one
// persistent launch.  The reference runs one generated entry point per call
// (meta/abc_gen_mix.py:448-472); a batch is the GPU form of calling it for many shapes.
// ---------------------------------------------------------------------------------------
struct fmm_batch {
  struct Job {
    int prob;                      // problem index
    const fmm_plan* plan;          // tables to run (the classical plan for strips)
    int grid[3];                   // plan dims (1,1,1 for classical)
    int ms, ns, ks;                // sub-block sizes
    int a_r, a_c, b_r, b_c, c_r, c_c;  // operand offsets (row, column) inside the problem
    bool presum;
    int kk;                        // k extent of the products: ks, or ks rounded up to the k step
                                   // when every product reads a zero-padded slot (ks % 8 != 0)
    int nA, nB;                    // pre-summed operand slots
    size_t ws_off;                 // byte offset of S (then T) in the workspace
    long long ldT;
    int chunks, tiles_m, tiles_n, units;
    int bm;                        // tile height: fmm::BM, or BM / 2 (direct phases only)
    int S;                         // k split of the job's products (the one a single call chooses)
    const fmm::Prod* vprods;       // its k-split tables when S > 1
    const fmm::Term* vterms;
    size_t ticket_off;             // int offset into the ticket array
    double cost;                   // estimated k steps per unit (scheduling order)
  };
  int count = 0;
  int dev = 0;
  std::vector<int> m, n, k;
  std::vector<const fmm_plan*> plans;
  std::vector<Job> jobs[2];        // phase 0: FMM cores and disjoint strips; phase 1: k strips
  bool direct[2] = {true, true};   // every job of the phase can run the direct variant
  std::vector<int> unit_start[2];
  int max_slots = 0;
  unsigned max_lincomb_chunks = 1;
  int n_lincomb = 0;
  size_t n_tickets = 0, ws_bytes = 0;
  fmm::GemmArgs* d_jobs[2] = {nullptr, nullptr};
  int* d_start[2] = {nullptr, nullptr};
  fmm::GemmArgs* h_jobs[2] = {nullptr, nullptr};  // pinned staging of the job tables
  fmm::LincombTask* d_lc = nullptr;
  fmm::LincombTask* h_lc = nullptr;
  int* d_tickets = nullptr;        // kBatchCounters work-unit counters (one per phase), then the tickets
  char* d_ws = nullptr;
  // Even-pitch copies of A / B for problems whose row count is odd (a dense operand then
  // has an odd leading dimension, which tensor copies cannot stage): byte offsets into
  // d_pitch, or SIZE_MAX when the operand needs none.
  std::vector<size_t> pitch_a, pitch_b;
  size_t pitch_bytes = 0;
  char* d_pitch = nullptr;
  fmm::PitchCopy* d_pc = nullptr;
  fmm::PitchCopy* h_pc = nullptr;
  cudaEvent_t staged = nullptr;    // the staging buffers' last copies are done
};

namespace {

bool batch_configured[kMaxDevices];

int batch_configure(int* dev) {
  int rc = configure_kernel(dev);
  if (rc != FMM_OK) return rc;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (!batch_configured[*dev]) {
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmm::smem_bytes(true)));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_batch_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fmm::smem_bytes(false)));
    FMM_CUDA_TRY(cudaFuncSetAttribute(fmm::fmm_gemm_direct_batch_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fmm::SMEM_BYTES_DIRECT));
    batch_configured[*dev] = true;
  }
  return FMM_OK;
}

// Products per unit: units of about the work of a 128 x 128 x 4096 classical tile, so the
// persistent grid balances across problems of very different sizes.
int batch_chunks(int nprod, int ks) {
  const long long ksteps = (long long)nprod * ((ks + fmm::BK - 1) / fmm::BK);
  long long c = (ksteps + 511) / 512;
  if (c < 1) c = 1;
  if (c > nprod) c = nprod;
  return (int)c;
}

void batch_add_job(fmm_batch* b, int phase, int prob, const fmm_plan* plan, int ms, int ns, int ks, int a_r, int a_c,
                   int b_r, int b_c, int c_r, int c_c, int bm) {
  if (ms <= 0 || ns <= 0 || ks <= 0) return;
  fmm_batch::Job j{};
  j.prob = prob;
  j.bm = bm;
  j.plan = plan;
  std::memcpy(j.grid, plan->dims, sizeof(j.grid));
  j.ms = ms;
  j.ns = ns;
  j.ks = ks;
  j.a_r = a_r;
  j.a_c = a_c;
  j.b_r = b_r;
  j.b_c = b_c;
  j.c_r = c_r;
  j.c_c = c_c;
  j.presum = plan->rank > 1 && use_presum(plan, ms, ns, ks);
  j.kk = ks;
  if (j.presum) {
    // as in run_fmm: with ks not a multiple of the k step every product gets its own slot,
    // zero-padded to whole k steps, so the phase keeps the direct variant
    const bool padded = ks % fmm::BK != 0;
    j.kk = padded ? (ks + fmm::BK - 1) / fmm::BK * fmm::BK : ks;
    j.nA = padded ? plan->rank : (int)plan->plistA.size();
    j.nB = padded ? plan->rank : (int)plan->plistB.size();
    j.ldT = padded ? j.kk : ks + (ks & 1);
    j.ws_off = b->ws_bytes;
    b->ws_bytes += sizeof(double) * ((size_t)ms * j.kk * j.nA + (size_t)j.ldT * ns * j.nB);
    b->ws_bytes = (b->ws_bytes + 255) & ~(size_t)255;
    b->max_slots = std::max(b->max_slots, std::max(j.nA, j.nB));
    b->max_lincomb_chunks = std::max({b->max_lincomb_chunks, lincomb_chunks((long long)(ms + 1) / 2 * ks),
                                      lincomb_chunks((long long)(ks + 1) / 2 * ns)});
    b->n_lincomb += (j.nA > 0) + (j.nB > 0);
  }
  j.tiles_n = (ns + fmm::BN - 1) / fmm::BN;
  // the k split a single call gives these products, so a batch computes each problem with the
  // same arithmetic as a call of its own
  j.S = call_ksplit(plan, ms, ns, ks, j.presum, j.kk, sm_count[b->dev]);
  j.chunks = batch_chunks(plan->rank * j.S, j.kk / j.S);
  // direct staging: operands are single unit-coefficient blocks (pre-summed or classical)
  // and every k step stays inside them
  if (!((j.presum || plan->rank == 1) && whole_k_steps(j.grid, j.kk))) b->direct[phase] = false;
  b->jobs[phase].push_back(j);
}

void batch_free(fmm_batch* b) {
  for (int ph = 0; ph < 2; ++ph) {
    if (b->d_jobs[ph]) cudaFree(b->d_jobs[ph]);
    if (b->d_start[ph]) cudaFree(b->d_start[ph]);
    if (b->h_jobs[ph]) cudaFreeHost(b->h_jobs[ph]);
  }
  if (b->d_lc) cudaFree(b->d_lc);
  if (b->h_lc) cudaFreeHost(b->h_lc);
  if (b->d_tickets) cudaFree(b->d_tickets);
  if (b->d_ws) cudaFree(b->d_ws);
  if (b->d_pitch) cudaFree(b->d_pitch);
  if (b->d_pc) cudaFree(b->d_pc);
  if (b->h_pc) cudaFreeHost(b->h_pc);
  if (b->staged) cudaEventDestroy(b->staged);
  delete b;
}

// The host side of a batch: jobs per phase in scheduling order, unit ranges, and the sizes
// of the tickets and workspaces.  Allocates no device memory (the plans' tables are
// uploaded on first use by device_tables).
int batch_build(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k, fmm_batch** out,
                const int* tile_m = nullptr) {
  if (!out || count <= 0 || !m || !n || !k) return FMM_E_INVALID;
  for (int i = 0; i < count; ++i) {
    if (m[i] < 0 || n[i] < 0 || k[i] < 0) return FMM_E_INVALID;
    if (tile_m && tile_m[i] != 0 && tile_m[i] != fmm::BM && tile_m[i] != fmm::BM / 2) return FMM_E_INVALID;
  }
  int dev = 0;
  int rc = batch_configure(&dev);
  if (rc != FMM_OK) return rc;
  fmm_batch* b = new (std::nothrow) fmm_batch();
  if (!b) return FMM_E_NOMEM;
  b->count = count;
  b->dev = dev;
  b->m.assign(m, m + count);
  b->n.assign(n, n + count);
  b->k.assign(k, k + count);
  const fmm_plan* cls = classical_plan();
  for (int i = 0; i < count; ++i) {
    const fmm_plan* p = (plans && plans[i]) ? plans[i] : nullptr;
    b->plans.push_back(p);
    const bool live = m[i] > 0 && n[i] > 0 && k[i] > 0;
    const int bm = (tile_m && tile_m[i] != 0) ? tile_m[i] : fmm::BM;
    auto reserve = [&](int rows, int cols) {
      const size_t off = b->pitch_bytes;
      b->pitch_bytes += (sizeof(double) * (size_t)(rows + 1) * cols + 255) & ~(size_t)255;
      return off;
    };
    b->pitch_a.push_back(live && (m[i] & 1) ? reserve(m[i], k[i]) : SIZE_MAX);
    b->pitch_b.push_back(live && (k[i] & 1) ? reserve(k[i], n[i]) : SIZE_MAX);
    if (!live) continue;
    if (!p) {
      batch_add_job(b, 0, i, cls, m[i], n[i], k[i], 0, 0, 0, 0, 0, 0, bm);
      continue;
    }
    // same partition and fringe regions as the single-problem path (run_fmm + peel)
    const int pm = p->dims[0] * kMR, pk = p->dims[1], pn = p->dims[2] * kNR;
    const int mr = m[i] % pm, kr = k[i] % pk, nr = n[i] % pn;
    const int md = m[i] - mr, kd = k[i] - kr, nd = n[i] - nr;
    if (md > 0 && nd > 0 && kd > 0)
      batch_add_job(b, 0, i, p, md / p->dims[0], nd / p->dims[2], kd / p->dims[1], 0, 0, 0, 0, 0, 0, bm);
    if (kr > 0 && md > 0 && nd > 0) batch_add_job(b, 1, i, cls, md, nd, kr, 0, kd, kd, 0, 0, 0, bm);
    if (nr > 0) batch_add_job(b, 0, i, cls, m[i], nr, k[i], 0, 0, 0, nd, 0, nd, bm);
    if (mr > 0 && nd > 0) batch_add_job(b, 0, i, cls, mr, nd, k[i], md, 0, 0, 0, md, 0, bm);
  }
  // Tile heights (64-row tiles only where the whole phase runs the direct variant), then
  // each job's units and tickets.
  for (int ph = 0; ph < 2; ++ph)
    for (auto& j : b->jobs[ph]) {
      if (!b->direct[ph]) j.bm = fmm::BM;
      j.tiles_m = (j.ms + j.bm - 1) / j.bm;
      j.units = j.tiles_m * j.tiles_n * j.chunks;
      j.ticket_off = b->n_tickets;
      if (j.chunks > 1) b->n_tickets += (size_t)j.tiles_m * j.tiles_n;
      j.cost = (double)j.plan->rank / j.chunks * ((j.kk + fmm::BK - 1) / fmm::BK) * j.bm / fmm::BM;
    }
  // Longest units first: the persistent grid takes units in order, so the short ones
  // fill in at the end.
  for (int ph = 0; ph < 2; ++ph) {
    std::stable_sort(b->jobs[ph].begin(), b->jobs[ph].end(),
                     [](const fmm_batch::Job& x, const fmm_batch::Job& y) { return x.cost > y.cost; });
    long long acc = 0;
    for (auto& j : b->jobs[ph]) {
      b->unit_start[ph].push_back((int)acc);
      acc += j.units;
    }
    if (acc > INT32_MAX) {
      batch_free(b);
      return FMM_E_UNSUPPORTED;
    }
    b->unit_start[ph].push_back((int)acc);
    for (auto& j : b->jobs[ph]) {
      DevTables* d = nullptr;
      rc = device_tables(j.plan, &d);
      if (rc == FMM_OK && j.S > 1)
        rc = ksplit_tables(j.plan, j.plan->rank == 1 ? BASE_ORIG : (j.kk != j.ks ? BASE_ALL : BASE_PS), j.S,
                           &j.vprods, &j.vterms);
      if (rc != FMM_OK) {
        batch_free(b);
        return rc;
      }
    }
  }
  *out = b;
  return FMM_OK;
}

int batch_create(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k, fmm_batch** out,
                 const int* tile_m = nullptr) {
  fmm_batch* b = nullptr;
  int rc = batch_build(count, plans, m, n, k, &b, tile_m);
  if (rc != FMM_OK) return rc;
  auto fail = [&](cudaError_t e) {
    batch_free(b);
    return cuda_status(e);
  };
  cudaError_t e = cudaSuccess;
  for (int ph = 0; ph < 2 && e == cudaSuccess; ++ph) {
    const size_t nj = b->jobs[ph].size();
    if (nj == 0) continue;
    e = cudaMalloc((void**)&b->d_jobs[ph], sizeof(fmm::GemmArgs) * nj);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_start[ph], sizeof(int) * (nj + 1));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_jobs[ph], sizeof(fmm::GemmArgs) * nj);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->d_start[ph], b->unit_start[ph].data(), sizeof(int) * (nj + 1), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && b->n_lincomb > 0) {
    e = cudaMalloc((void**)&b->d_lc, sizeof(fmm::LincombTask) * b->n_lincomb);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_lc, sizeof(fmm::LincombTask) * b->n_lincomb);
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_tickets, sizeof(int) * (kBatchCounters + b->n_tickets));
  if (e == cudaSuccess && b->ws_bytes > 0) e = cudaMalloc((void**)&b->d_ws, b->ws_bytes);
  if (e == cudaSuccess && b->pitch_bytes > 0) {
    e = cudaMalloc((void**)&b->d_pitch, b->pitch_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_pc, sizeof(fmm::PitchCopy) * 2 * count);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_pc, sizeof(fmm::PitchCopy) * 2 * count);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
  if (e != cudaSuccess) return fail(e);
  *out = b;
  return FMM_OK;
}

// Fill the job table of one phase for this call's operands; false if a problem cannot
// use TMA staging (the phase then runs with cp.async staging).
bool batch_fill(fmm_batch* b, int ph, const double* const* A, const long* lda, const double* const* B,
                const long* ldb, double* const* C, const long* ldc, int* n_lc) {
  bool tma = true;
  for (size_t q = 0; q < b->jobs[ph].size(); ++q) {
    const fmm_batch::Job& j = b->jobs[ph][q];
    const DevTables& d = j.plan->dev[b->dev];
    fmm::GemmArgs a{};
    const long long la = lda[j.prob], lb = ldb[j.prob], lc = ldc[j.prob];
    a.A = A[j.prob] + j.a_r + (long long)j.a_c * la;
    a.lda = la;
    a.B = B[j.prob] + j.b_r + (long long)j.b_c * lb;
    a.ldb = lb;
    a.C = C[j.prob] + j.c_r + (long long)j.c_c * lc;
    a.ldc = lc;
    a.ms = j.ms;
    a.ns = j.ns;
    a.ks = j.ks;
    a.nprod = j.plan->rank;
    a.tiles_m = j.tiles_m;
    a.bm = j.bm;
    a.tiles_n = j.tiles_n;
    a.chunks = j.chunks;
    a.mode = fmm::MODE_ACCUM_C;
    a.tickets = j.chunks > 1 ? b->d_tickets + kBatchCounters + j.ticket_off : nullptr;
    a.status = dev_status[b->dev];
    const long long am = (long long)j.grid[0] * j.ms, ak = (long long)j.grid[1] * j.ks,
                    bn = (long long)j.grid[2] * j.ns;
    if (j.presum) {
      const bool padded = j.kk != j.ks;
      const double* S = reinterpret_cast<const double*>(b->d_ws + j.ws_off);
      const double* T = S + (size_t)j.ms * j.kk * j.nA;
      a.ks = j.kk;
      a.prods = padded ? d.prods_all : d.prods_ps;
      a.terms = padded ? d.terms_all : d.terms_ps;
      a.Aw = S;
      a.ldaw = j.ms;
      a.Bw = T;
      a.ldbw = j.ldT;
      for (int side = 0; side < 2; ++side) {
        const int ns = side == 0 ? j.nA : j.nB;
        if (ns == 0) continue;
        fmm::LincombTask& t = b->h_lc[(*n_lc)++];
        t = fmm::LincombTask{};
        t.nout = ns;
        fmm::LincombArgs& l = t.a;
        l.X = side == 0 ? a.A : a.B;
        l.ldx = side == 0 ? la : lb;
        l.rows = side == 0 ? j.ms : j.ks;
        l.cols = side == 0 ? j.ks : j.ns;
        l.blk_row_stride = l.rows;
        l.blk_col_stride = l.cols;
        l.out = const_cast<double*>(side == 0 ? S : T);
        l.ldo = side == 0 ? j.ms : j.ldT;
        l.out_stride = l.ldo * (side == 0 ? j.kk : l.cols);
        l.prods = d.prods;
        l.terms = d.terms;
        l.plist = padded ? d.plist_all : side == 0 ? d.plistA : d.plistB;
        l.side = side;
      }
    } else {
      a.prods = d.prods;
      a.terms = d.terms;
      a.Aw = a.A;
      a.ldaw = la;
      a.Bw = a.B;
      a.ldbw = lb;
    }
    bool ok = make_tensor_map(&a.tmA, a.A, am, ak, la, fmm::BM, fmm::BK) &&
              make_tensor_map(&a.tmA64, a.A, am, ak, la, fmm::BM / 2, fmm::BK) &&
              make_tensor_map(&a.tmB, a.B, ak, bn, lb, fmm::BK, fmm::BN) &&
              make_tensor_map(&a.tmB2, a.B, ak, bn, lb, fmm::TB_K, fmm::BN);
    if (ok && j.presum && j.nA > 0)
      ok = make_tensor_map(&a.tmAw, a.Aw, j.ms, (long long)j.nA * j.kk, j.ms, fmm::BM, fmm::BK) &&
           make_tensor_map(&a.tmAw64, a.Aw, j.ms, (long long)j.nA * j.kk, j.ms, fmm::BM / 2, fmm::BK);
    else
      a.tmAw = a.tmA, a.tmAw64 = a.tmA64;
    if (ok && j.presum && j.nB > 0)
      ok = make_tensor_map(&a.tmBw, a.Bw, j.kk, (long long)j.nB * j.ns, j.ldT, fmm::BK, fmm::BN) &&
           make_tensor_map(&a.tmBw2, a.Bw, j.kk, (long long)j.nB * j.ns, j.ldT, fmm::TB_K, fmm::BN);
    else
      a.tmBw = a.tmB, a.tmBw2 = a.tmB2;
    if (j.S > 1) {  // the k-split tables (part depth kk / S); the tensor maps keep the full depth
      a.ks /= j.S;
      a.nprod *= j.S;
      a.prods = j.vprods;
      a.terms = j.vterms;
    }
    tma = tma && ok;
    b->h_jobs[ph][q] = a;
  }
  return tma;
}

void batch_prepare(fmm_batch* b, const double* const* A, const long* lda, const double* const* B, const long* ldb,
                   double* const* C, const long* ldc, int* n_lc_out, int* n_pc_out, bool tma[2]);
int batch_launch(fmm_batch* b, cudaStream_t st, int n_lc, int n_pc, const bool tma[2]);

int batch_run(fmm_batch* b, const double* const* A, const long* lda, const double* const* B, const long* ldb,
              double* const* C, const long* ldc, cudaStream_t st) {
  if (!b || !A || !lda || !B || !ldb || !C || !ldc) return FMM_E_INVALID;
  int dev = 0;
  FMM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev != b->dev) return FMM_E_INVALID;
  for (int i = 0; i < b->count; ++i) {
    int rc = check_args(b->m[i], b->n[i], b->k[i], A[i], lda[i], B[i], ldb[i], C[i], ldc[i]);
    if (rc != FMM_OK) return rc;
  }
  // The staging buffers are reused: the previous call's copies out of them must be done.
  // Inside a stream capture the copies become graph nodes that read the staging buffers
  // at every replay, so a graph replays with the most recent call's operands.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  FMM_CUDA_TRY(cudaStreamIsCapturing(st, &cap));
  if (cap == cudaStreamCaptureStatusNone) FMM_CUDA_TRY(cudaEventSynchronize(b->staged));
  int n_lc = 0, n_pc = 0;
  bool tma[2] = {true, true};
  batch_prepare(b, A, lda, B, ldb, C, ldc, &n_lc, &n_pc, tma);
  for (int ph = 0; ph < 2; ++ph)
    if (!b->jobs[ph].empty())
      FMM_CUDA_TRY(cudaMemcpyAsync(b->d_jobs[ph], b->h_jobs[ph], sizeof(fmm::GemmArgs) * b->jobs[ph].size(),
                                   cudaMemcpyHostToDevice, st));
  if (n_lc > 0)
    FMM_CUDA_TRY(cudaMemcpyAsync(b->d_lc, b->h_lc, sizeof(fmm::LincombTask) * n_lc, cudaMemcpyHostToDevice, st));
  if (n_pc > 0)
    FMM_CUDA_TRY(cudaMemcpyAsync(b->d_pc, b->h_pc, sizeof(fmm::PitchCopy) * n_pc, cudaMemcpyHostToDevice, st));
  if (cap == cudaStreamCaptureStatusNone) FMM_CUDA_TRY(cudaEventRecord(b->staged, st));
  return batch_launch(b, st, n_lc, n_pc, tma);
}

// This call's job tables (host staging): even-pitch copies for odd leading dimensions,
// per-job arguments and tensor maps, pre-sum tasks.
void batch_prepare(fmm_batch* b, const double* const* A, const long* lda, const double* const* B, const long* ldb,
                   double* const* C, const long* ldc, int* n_lc_out, int* n_pc_out, bool tma[2]) {
  // Operands with an odd leading dimension and a reserved even-pitch copy are staged
  // through it (rows + 1 pitch); the others are used in place.
  std::vector<const double*> eA(A, A + b->count), eB(B, B + b->count);
  std::vector<long> elda(lda, lda + b->count), eldb(ldb, ldb + b->count);
  int n_pc = 0;
  for (int i = 0; i < b->count; ++i) {
    if ((lda[i] & 1) && b->pitch_a[i] != SIZE_MAX) {
      double* dst = reinterpret_cast<double*>(b->d_pitch + b->pitch_a[i]);
      b->h_pc[n_pc++] = fmm::PitchCopy{A[i], lda[i], dst, b->m[i] + 1LL, b->m[i], b->k[i]};
      eA[i] = dst;
      elda[i] = b->m[i] + 1;
    }
    if ((ldb[i] & 1) && b->pitch_b[i] != SIZE_MAX) {
      double* dst = reinterpret_cast<double*>(b->d_pitch + b->pitch_b[i]);
      b->h_pc[n_pc++] = fmm::PitchCopy{B[i], ldb[i], dst, b->k[i] + 1LL, b->k[i], b->n[i]};
      eB[i] = dst;
      eldb[i] = b->k[i] + 1;
    }
  }
  int n_lc = 0;
  for (int ph = 0; ph < 2; ++ph)
    if (!b->jobs[ph].empty())
      tma[ph] = batch_fill(b, ph, eA.data(), elda.data(), eB.data(), eldb.data(), C, ldc, &n_lc);
  *n_lc_out = n_lc;
  *n_pc_out = n_pc;
}

// Enqueue the launches of a prepared batch whose tables are (being) copied to the device.
int batch_launch(fmm_batch* b, cudaStream_t st, int n_lc, int n_pc, const bool tma[2]) {
  // the phases' work-unit counters and every ticket start at zero
  FMM_CUDA_TRY(cudaMemsetAsync(b->d_tickets, 0, sizeof(int) * (kBatchCounters + b->n_tickets), st));
  if (n_pc > 0) {
    ProfScope pf(K_PITCH_COPY, st);
    fmm::fmm_pitch_copy_kernel<<<dim3(256, (unsigned)n_pc), 256, 0, st>>>(b->d_pc);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    FMM_CUDA_TRY(cudaGetLastError());
  }
  // zero padding of the padded slots (k columns [ks, kk) of every S slot, rows [ks, kk)
  // of every T slot column): the sums fill only [0, ks)
  for (int ph = 0; ph < 2; ++ph)
    for (const auto& j : b->jobs[ph]) {
      if (!j.presum || j.kk == j.ks) continue;
      char* S = b->d_ws + j.ws_off;
      char* T = S + sizeof(double) * (size_t)j.ms * j.kk * j.nA;
      FMM_CUDA_TRY(cudaMemset2DAsync(S + sizeof(double) * (size_t)j.ms * j.ks, sizeof(double) * (size_t)j.ms * j.kk, 0,
                                     sizeof(double) * (size_t)j.ms * (j.kk - j.ks), j.nA, st));
      FMM_CUDA_TRY(cudaMemset2DAsync(T + sizeof(double) * j.ks, sizeof(double) * (size_t)j.kk, 0,
                                     sizeof(double) * (j.kk - j.ks), (size_t)j.nB * j.ns, st));
    }
  if (n_lc > 0) {
    ProfScope pf(K_LINCOMB_BATCH, st);
    fmm::fmm_lincomb_batch_kernel<<<dim3((unsigned)b->max_slots, b->max_lincomb_chunks, (unsigned)n_lc), 256, 0, st>>>(
        b->d_lc);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    FMM_CUDA_TRY(cudaGetLastError());
  }
  for (int ph = 0; ph < 2; ++ph) {
    if (b->jobs[ph].empty()) continue;
    fmm::BatchArgs ba{};
    ba.jobs = b->d_jobs[ph];
    ba.unit_start = b->d_start[ph];
    ba.njobs = (int)b->jobs[ph].size();
    ba.units = b->unit_start[ph].back();
    ba.status = dev_status[b->dev];
    ba.counter = b->d_tickets + ph;
    const unsigned grid = (unsigned)std::min<long long>(ba.units, sm_count[b->dev]);
    {
      ProfScope pf(K_GEMM_BATCH, st);
      if (tma[ph] && b->direct[ph])
        fmm::fmm_gemm_direct_batch_kernel<<<grid, fmm::NTHREADS, fmm::SMEM_BYTES_DIRECT, st>>>(ba);
      else if (tma[ph])
        fmm::fmm_gemm_batch_kernel<true><<<grid, fmm::NTHREADS, fmm::smem_bytes(true), st>>>(ba);
      else
        fmm::fmm_gemm_batch_kernel<false><<<grid, fmm::NTHREADS, fmm::smem_bytes(false), st>>>(ba);
    }
    g_launches.fetch_add(1, std::memory_order_relaxed);
    FMM_CUDA_TRY(cudaGetLastError());
  }
  return FMM_OK;
}

}  // namespace

extern "C" {

int fmm_batch_create(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k,
                     fmm_batch** out) {
  return batch_create(count, plans, m, n, k, out);
}

int fmm_batch_create_tiled(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k,
                           const int* tile_m, fmm_batch** out) {
  return batch_create(count, plans, m, n, k, out, tile_m);
}

int fmm_batch_dgemm(fmm_batch* batch, const double* const* A, const long* lda, const double* const* B,
                    const long* ldb, double* const* C, const long* ldc, void* stream) {
  return batch_run(batch, A, lda, B, ldb, C, ldc, static_cast<cudaStream_t>(stream));
}

int fmm_batch_units(const fmm_batch* batch, int phase) {
  if (!batch || phase < 0 || phase > 1) return FMM_E_INVALID;
  return batch->unit_start[phase].empty() ? 0 : batch->unit_start[phase].back();
}

int fmm_batch_destroy(fmm_batch* batch) {
  if (!batch) return FMM_E_INVALID;
  cudaEventSynchronize(batch->staged);
  batch_free(batch);
  return FMM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// One-shot batches for request loops: the batch is formed, run and released per call with
// no cudaMalloc / cudaFree (those synchronise the device, which would stop the requests
// of a serving loop from overlapping).  Device buffers come from the stream-ordered pool;
// the job tables go through a ring of pinned host buffers, each reused only after the
// copy out of it has completed.
// ---------------------------------------------------------------------------------------
namespace {

struct PinnedRing {
  static constexpr int N = 8;
  char* buf[N] = {};
  size_t cap[N] = {};
  cudaEvent_t ev[N] = {};
  int next = 0;
  std::mutex mu;
};
PinnedRing g_ring[kMaxDevices];

int ring_acquire(int dev, size_t bytes, char** buf, cudaEvent_t* ev) {
  PinnedRing& r = g_ring[dev];
  std::lock_guard<std::mutex> lk(r.mu);
  const int s = r.next;
  r.next = (s + 1) % PinnedRing::N;
  if (!r.ev[s]) FMM_CUDA_TRY(cudaEventCreateWithFlags(&r.ev[s], cudaEventDisableTiming));
  FMM_CUDA_TRY(cudaEventSynchronize(r.ev[s]));  // the slot's previous copy is done
  if (r.cap[s] < bytes) {
    if (r.buf[s]) cudaFreeHost(r.buf[s]);
    r.buf[s] = nullptr;
    r.cap[s] = 0;
    const size_t cap = std::max<size_t>(bytes + bytes / 2, (size_t)1 << 20);
    FMM_CUDA_TRY(cudaMallocHost((void**)&r.buf[s], cap));
    r.cap[s] = cap;
  }
  *buf = r.buf[s];
  *ev = r.ev[s];
  return FMM_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int batch_submit(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k,
                 const double* const* A, const long* lda, const double* const* B, const long* ldb, double* const* C,
                 const long* ldc, cudaStream_t st) {
  if (!A || !lda || !B || !ldb || !C || !ldc) return FMM_E_INVALID;
  for (int i = 0; i < count; ++i) {
    int rc = check_args(m[i], n[i], k[i], A[i], lda[i], B[i], ldb[i], C[i], ldc[i]);
    if (rc != FMM_OK) return rc;
  }
  fmm_batch* b = nullptr;
  int rc = batch_build(count, plans, m, n, k, &b);
  if (rc != FMM_OK) return rc;
  // table block (identical layout in pinned staging and on the device)
  size_t off = 0, o_jobs[2], o_start[2];
  for (int ph = 0; ph < 2; ++ph) {
    off = align_up(off, 64);
    o_jobs[ph] = off;
    off += sizeof(fmm::GemmArgs) * b->jobs[ph].size();
  }
  for (int ph = 0; ph < 2; ++ph) {
    off = align_up(off, 16);
    o_start[ph] = off;
    off += sizeof(int) * b->unit_start[ph].size();
  }
  off = align_up(off, 64);
  const size_t o_lc = off;
  off += sizeof(fmm::LincombTask) * b->n_lincomb;
  off = align_up(off, 64);
  const size_t o_pc = off;
  off += sizeof(fmm::PitchCopy) * 2 * count;
  const size_t table_bytes = align_up(off, 256);
  const size_t o_tk = table_bytes;
  const size_t o_ws = align_up(o_tk + sizeof(int) * (kBatchCounters + b->n_tickets), 256);
  const size_t o_pt = align_up(o_ws + b->ws_bytes, 256);
  const size_t dev_bytes = o_pt + b->pitch_bytes;
  char* stage = nullptr;
  cudaEvent_t stage_ev = nullptr;
  rc = ring_acquire(b->dev, table_bytes, &stage, &stage_ev);
  char* blk = nullptr;
  if (rc == FMM_OK) rc = cuda_status(cudaMallocAsync((void**)&blk, dev_bytes, st));
  if (rc != FMM_OK) {
    batch_free(b);
    return rc;
  }
  for (int ph = 0; ph < 2; ++ph) {
    b->h_jobs[ph] = reinterpret_cast<fmm::GemmArgs*>(stage + o_jobs[ph]);
    b->d_jobs[ph] = reinterpret_cast<fmm::GemmArgs*>(blk + o_jobs[ph]);
    b->d_start[ph] = reinterpret_cast<int*>(blk + o_start[ph]);
    if (!b->unit_start[ph].empty())
      std::memcpy(stage + o_start[ph], b->unit_start[ph].data(), sizeof(int) * b->unit_start[ph].size());
  }
  b->h_lc = reinterpret_cast<fmm::LincombTask*>(stage + o_lc);
  b->d_lc = reinterpret_cast<fmm::LincombTask*>(blk + o_lc);
  b->h_pc = reinterpret_cast<fmm::PitchCopy*>(stage + o_pc);
  b->d_pc = reinterpret_cast<fmm::PitchCopy*>(blk + o_pc);
  b->d_tickets = reinterpret_cast<int*>(blk + o_tk);
  b->d_ws = b->ws_bytes ? blk + o_ws : nullptr;
  b->d_pitch = b->pitch_bytes ? blk + o_pt : nullptr;
  int n_lc = 0, n_pc = 0;
  bool tma[2] = {true, true};
  batch_prepare(b, A, lda, B, ldb, C, ldc, &n_lc, &n_pc, tma);
  rc = cuda_status(cudaMemcpyAsync(blk, stage, table_bytes, cudaMemcpyHostToDevice, st));
  if (rc == FMM_OK) rc = cuda_status(cudaEventRecord(stage_ev, st));
  if (rc == FMM_OK) rc = batch_launch(b, st, n_lc, n_pc, tma);
  cudaError_t fe = cudaFreeAsync(blk, st);
  if (rc == FMM_OK) rc = cuda_status(fe);
  // the buffers belong to the pool and the ring: detach them before freeing the host side
  for (int ph = 0; ph < 2; ++ph) b->h_jobs[ph] = nullptr, b->d_jobs[ph] = nullptr, b->d_start[ph] = nullptr;
  b->h_lc = nullptr, b->d_lc = nullptr, b->h_pc = nullptr, b->d_pc = nullptr;
  b->d_tickets = nullptr, b->d_ws = nullptr, b->d_pitch = nullptr;
  batch_free(b);
  return rc;
}

}  // namespace

extern "C" int fmm_batch_submit(int count, const fmm_plan* const* plans, const int* m, const int* n, const int* k,
                                const double* const* A, const long* lda, const double* const* B, const long* ldb,
                                double* const* C, const long* ldc, void* stream) {
  return batch_submit(count, plans, m, n, k, A, lda, B, ldb, C, ldc, static_cast<cudaStream_t>(stream));
}
