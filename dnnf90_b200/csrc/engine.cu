// engine.cu - batched forward / seed / adjoint on the device.
//
// Kernels, in the order one training step launches them (per chunk):
//   k_layer2       first hidden layer, analytic: its input T is x and the
//                  unit vectors (lib/train_module.f90:253-257), so
//                  S^alpha is b+Wx, W e_i or 0 and T^alpha = sigma^(|a|) W^a
//   k_gemm<FWD>    S_l = W_l T_{l-1} (+ bias on the alpha = 0 rows)
//                  (lib/train_module.f90:267-278)
//   k_bell_fwd     Faa di Bruno / partial Bell step (:283-325)
//   k_output_fwd   identity read-out, residual, seed and loss
//                  (:326-328; app/pinn_module.f90:32-65)
//   k_output_adj   Tb_{L-1} = W_L^T seed and dW_L (:382, :409-444)
//   k_bell_adj     Bell adjoint (:381-403)
//   k_gemm<DW>     dW_l += Sb_l T_{l-1}^T (:409-422), split over rows
//   k_gemm<DT>     Tb_{l-1} = W_l^T Sb_l (:430-444)
//   k_bell_adj_l2  Bell adjoint of the first hidden layer fused with its
//                  weight gradient (only Sb^0 and Sb^{e_i} are needed)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "engine.hpp"
#include "gemm_f64.hpp"
#include "gemm_tc.hpp"
#include "kernels.cuh"

namespace dnnf90 {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;
const char *last_error() { return g_err.c_str(); }
void set_error(const std::string &m) { g_err = m; }

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ---------------------------------------------------------------- profiler
namespace {
struct ProfRec {
  const char *name;
  cudaEvent_t a, b;
};
std::mutex g_pmu;
bool g_prof = false;
std::vector<ProfRec> g_recs;
std::vector<cudaEvent_t> g_evpool;
cudaEvent_t prof_event() {
  if (!g_evpool.empty()) {
    cudaEvent_t e = g_evpool.back();
    g_evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

void profile_enable(bool on) {
  std::lock_guard<std::mutex> lk(g_pmu);
  g_prof = on;
}

int prof_begin(const char *name, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(g_pmu);
  if (!g_prof) return -1;
  ProfRec r{name, prof_event(), prof_event()};
  cudaEventRecord(r.a, st);
  g_recs.push_back(r);
  return (int)g_recs.size() - 1;
}

void prof_end(int idx, cudaStream_t st) {
  if (idx < 0) return;
  std::lock_guard<std::mutex> lk(g_pmu);
  if (idx < (int)g_recs.size()) cudaEventRecord(g_recs[idx].b, st);
}

// "name count total_ms" lines, one per kernel name; clears the records
std::string profile_read() {
  std::lock_guard<std::mutex> lk(g_pmu);
  std::vector<std::pair<std::string, std::pair<long, double>>> agg;
  for (ProfRec &r : g_recs) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    bool found = false;
    for (auto &e : agg)
      if (e.first == r.name) {
        e.second.first++;
        e.second.second += ms;
        found = true;
        break;
      }
    if (!found) agg.push_back({r.name, {1, (double)ms}});
    g_evpool.push_back(r.a);
    g_evpool.push_back(r.b);
  }
  g_recs.clear();
  std::string out;
  char buf[256];
  for (auto &e : agg) {
    std::snprintf(buf, sizeof buf, "%s %ld %.6f\n", e.first.c_str(), e.second.first,
                  e.second.second);
    out += buf;
  }
  return out;
}

#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) {                                            \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));    \
      return e_ == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;    \
    }                                                                   \
  } while (0)

int device_ready() {
  static int state = 0;  // 0 unknown, 1 ok, -1 none
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (state == 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n < 1) {
      set_error("no CUDA device: the dnnf90 device path needs a B200");
      state = -1;
    } else {
      state = 1;
    }
  }
  if (state < 0) {
    set_error("no CUDA device: the dnnf90 device path needs a B200");
    return RC_DEVICE;
  }
  return RC_OK;
}

// ------------------------------------------------------------ device copies
template <typename T>
static int dalloc(T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc((void **)p, n * sizeof(T)));
  return RC_OK;
}
template <typename T>
static int dput(T **p, const T *h, size_t n) {
  int rc = dalloc(p, n);
  if (rc) return rc;
  if (n) CK(cudaMemcpy(*p, h, n * sizeof(T), cudaMemcpyHostToDevice));
  return RC_OK;
}

void DevTables::release() {
  void *ps[] = {deg, alpha, ind_e1, seg, fq_pk, fq_c64, fq_c32, pseg, pair_pk,
                pair_c64, pair_c32, tpc, l2par, l2up};
  for (void *p : ps)
    if (p) cudaFree(p);
  bp.release();
  *this = DevTables();
}

int upload_tables(const TableSet &t, DevTables &d) {
  int rc = device_ready();
  if (rc) return rc;
  d.release();
  d.d0 = t.d0;
  d.k = t.k;
  d.na = t.na;
  d.nslot = t.nslot;
  d.iact = t.iact;
  const int na = t.na, k = t.k;
  std::vector<int> seg((size_t)na * (k + 1) * 3, 0);
  std::vector<uint32_t> fq_pk(t.fq_ib.size());
  std::vector<float> fq32(t.fq_c.size());
  for (int ia = 1; ia < na; ++ia)
    for (int q = 2; q <= t.deg[ia]; ++q) {
      int st = t.fq_at(ia, q), nn = t.fq_len(ia, q);
      int *s = &seg[((size_t)ia * (k + 1) + q) * 3];
      s[0] = st;
      s[1] = nn;
      s[2] = t.bslot[(size_t)ia * (k + 1) + q];
      for (int it = st; it < st + nn; ++it) {
        int op;
        if (q == 2) {
          op = t.fq_id[it];  // B_{id,1} = S_id
        } else {
          op = t.bslot[(size_t)t.fq_id[it] * (k + 1) + (q - 1)];
          if (op < 0) {
            set_error("table program: a Bell operand has no state slot");
            return RC_BAD_ARG;
          }
        }
        if (t.fq_ib[it] > 0xffff || op > 0xffff) {
          set_error("carried set too large for the device tables");
          return RC_UNSUPPORTED;
        }
        fq_pk[it] = (uint32_t)t.fq_ib[it] | ((uint32_t)op << 16);
        fq32[it] = (float)t.fq_c[it];
      }
    }
  std::vector<int> pseg((size_t)na * 2, 0);
  std::vector<uint32_t> pair_pk(t.pair_ia.size());
  std::vector<float> pair32(t.pair_binom.size());
  for (int ib = 0; ib < na; ++ib) {
    pseg[ib * 2] = t.pair_start[ib];
    pseg[ib * 2 + 1] = t.pair_num[ib];
  }
  for (size_t i = 0; i < t.pair_ia.size(); ++i) {
    pair_pk[i] = (uint32_t)t.pair_ia[i] | ((uint32_t)t.pair_id[i] << 16);
    pair32[i] = (float)t.pair_binom[i];
  }
  std::vector<int> ie1(t.ind_e1);
  d.nfq = (int)t.fq_ib.size();
  d.npair = (int)t.pair_ia.size();
  if ((rc = dput(&d.deg, t.deg.data(), t.deg.size()))) return rc;
  if ((rc = dput(&d.alpha, t.alpha.data(), t.alpha.size()))) return rc;
  if ((rc = dput(&d.ind_e1, ie1.data(), ie1.size()))) return rc;
  if ((rc = dput(&d.seg, seg.data(), seg.size()))) return rc;
  if ((rc = dput(&d.fq_pk, fq_pk.data(), fq_pk.size()))) return rc;
  if ((rc = dput(&d.fq_c64, t.fq_c.data(), t.fq_c.size()))) return rc;
  if ((rc = dput(&d.fq_c32, fq32.data(), fq32.size()))) return rc;
  if ((rc = dput(&d.pseg, pseg.data(), pseg.size()))) return rc;
  if ((rc = dput(&d.pair_pk, pair_pk.data(), pair_pk.size()))) return rc;
  if ((rc = dput(&d.pair_c64, t.pair_binom.data(), t.pair_binom.size()))) return rc;
  if ((rc = dput(&d.pair_c32, pair32.data(), pair32.size()))) return rc;
  if ((rc = dput(&d.tpc, t.tpc.data(), t.tpc.size()))) return rc;
  {
    // parent / child slots along unit steps (downward closure keeps a - e_i)
    const int d0 = t.d0;
    std::vector<int> par(na, 0), up((size_t)na * d0, -1);
    std::vector<int> b(d0);
    for (int ia = 1; ia < na; ++ia) {
      const int *al = &t.alpha[(size_t)ia * d0];
      int i0 = 0;
      while (i0 < d0 && al[i0] == 0) ++i0;
      for (int i = 0; i < d0; ++i) b[i] = al[i];
      b[i0] -= 1;
      const int ps = t.find(b.data());
      if (ps < 0) {
        set_error("table program: the carried set is not downward closed");
        return RC_BAD_ARG;
      }
      par[ia] = ps | (i0 << 16);
    }
    for (int ia = 0; ia < na; ++ia)
      for (int i = 0; i < d0; ++i) {
        for (int c = 0; c < d0; ++c) b[c] = t.alpha[(size_t)ia * d0 + c];
        b[i] += 1;
        const int u = t.find(b.data());
        if (u >= 0) up[(size_t)ia * d0 + i] = u | (b[i] << 16);
      }
    d.graded = true;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] < t.deg[ia - 1]) d.graded = false;
    d.dstart.assign(k + 2, na);
    for (int ia = na - 1; ia >= 0; --ia) d.dstart[t.deg[ia]] = ia;
    for (int p = k; p >= 0; --p) d.dstart[p] = std::min(d.dstart[p], d.dstart[p + 1]);
    if ((rc = dput(&d.l2par, par.data(), par.size()))) return rc;
    if ((rc = dput(&d.l2up, up.data(), up.size()))) return rc;
  }
  if ((rc = upload_bell_plan(t, d.bp))) return rc;
  return RC_OK;
}

void DevNet::release() {
  if (w64) cudaFree(w64);
  if (wpk) cudaFree(wpk);
  wpk = nullptr;
  if (w32) cudaFree(w32);
  gemm_tc_release_weights(this);
  w64 = nullptr;
  w32 = nullptr;
  uploaded = 0;
}

void DevRule::release() {
  void *ps[] = {coeff, ind, nonlin, sys, sfac, wres};
  for (void *p : ps)
    if (p) cudaFree(p);
  coeff = nullptr;
  ind = nullptr;
  nonlin = nullptr;
  sys = sfac = nullptr;
  wres = nullptr;
}

int upload_rule(const SeedRuleHost &r, DevRule &d) {
  int rc = device_ready();
  if (rc) return rc;
  d.release();
  d.kind = r.kind;
  d.nterm = (int)r.coeff.size();
  d.fac = r.fac;
  if ((rc = dput(&d.coeff, r.coeff.data(), r.coeff.size()))) return rc;
  if ((rc = dput(&d.ind, r.ind.data(), r.ind.size()))) return rc;
  if ((rc = dput(&d.nonlin, r.nonlin.data(), r.nonlin.size()))) return rc;
  d.nres = r.nres;
  if (r.kind == SEED_SYS) {
    if ((rc = dput(&d.sys, r.sys.data(), r.sys.size()))) return rc;
    if ((rc = dput(&d.sfac, r.sfac.data(), r.sfac.size()))) return rc;
    if ((rc = dput(&d.wres, r.wres.data(), r.wres.size()))) return rc;
  }
  return RC_OK;
}

void Planes::release() {
  if (base) cudaFree(base);
  if (scratch) cudaFree(scratch);
  *this = Planes();
}

// ------------------------------------------------------------- kernel args
struct L2Args {
  int n, na, d0, k, iact, npts;
  const int *alpha, *deg;
  const double *tpc;
  const double *X;       // [P][d0]
  const double *W;       // layer-2 weights [n][d0+1]
  void *T, *h;           // [P][na][n]
};

// First hidden layer.  Its pre-activation is linear in x, so every mixed
// partial of the pre-activation of order >= 2 vanishes and the Faa di Bruno
// sum collapses to one term: T^alpha = sigma^(|alpha|)(a) prod_i W_i^alpha_i,
// h^alpha = sigma^(|alpha|+1)(a) prod_i W_i^alpha_i.  The reference reaches
// the same values through the general recurrence, whose other terms all
// multiply an exact zero.
template <typename R, bool TRAIN>
__global__ void __launch_bounds__(128) k_layer2(L2Args a) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  const int d0 = a.d0;
  double wj[D0MAX];
  const double *wr = a.W + (size_t)j * (d0 + 1);
  for (int i = 0; i < d0; ++i) wj[i] = wr[1 + i];
  double d[KMAX + 2];
  const size_t plane = (size_t)a.na * a.n;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const double *x = a.X + (size_t)pt * d0;
    double s = wr[0];
    for (int i = 0; i < d0; ++i) s = s + wj[i] * x[i];
    sigma_derivs(a.iact, a.tpc, a.k, s, d);
    R *T = (R *)a.T + pt * plane + j;
    R *H = TRAIN ? (R *)a.h + pt * plane + j : nullptr;
    T[0] = (R)d[0];
    if (TRAIN) H[0] = (R)d[1];
    for (int ia = 1; ia < a.na; ++ia) {
      const int *al = a.alpha + (size_t)ia * d0;
      double m = 1.0;
      for (int i = 0; i < d0; ++i) {
        int e = __ldg(al + i);
        for (int r = 0; r < e; ++r) m *= wj[i];
      }
      const int p = __ldg(a.deg + ia);
      T[(size_t)ia * a.n] = (R)(d[p] * m);
      if (TRAIN) H[(size_t)ia * a.n] = (R)(d[p + 1] * m);
    }
  }
}

struct BellArgs {
  int n, na, k, nslot, npts, iact;
  const int *deg, *seg;
  const uint32_t *fq_pk;
  const void *fq_c;
  const double *tpc;
  const void *S;
  void *T, *h;
  void *scratch;  // per-CTA state when it does not fit shared memory
};

// Bell forward of one hidden layer.  One thread per (point, neuron), the
// neuron index in the lanes so that every plane access is one coalesced
// line and every table read is warp-uniform.  Multi-indices are visited in
// the reference order; B_{alpha,q} (q >= 2) of the multi-indices that later
// ones reread (deg < K) is kept in a per-thread state array in shared memory
// (or a global spill), indexed [slot][thread].
template <typename R, bool TRAIN>
__global__ void __launch_bounds__(128) k_bell_fwd(BellArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nthr = blockDim.x;
  const int j = blockIdx.y * nthr + threadIdx.x;
  const bool act = j < a.n;
  const int jc = act ? j : a.n - 1;
  const size_t plane = (size_t)a.na * a.n;
  const int n = a.n, k = a.k;
  R *B = a.scratch
             ? (R *)a.scratch + ((size_t)(blockIdx.y * gridDim.x + blockIdx.x) * a.nslot) * nthr
             : (R *)smem_raw;
  B += threadIdx.x;
  const R *coef = (const R *)a.fq_c;
  double dd[KMAX + 2];
  R dt[KMAX + 2];
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *S = (const R *)a.S + pt * plane + jc;
    R *T = (R *)a.T + pt * plane + jc;
    R *H = TRAIN ? (R *)a.h + pt * plane + jc : nullptr;
    sigma_derivs(a.iact, a.tpc, k, (double)S[0], dd);
    for (int q = 0; q <= k + 1; ++q) dt[q] = (R)dd[q];
    if (act) {
      T[0] = dt[0];
      if (TRAIN) H[0] = dt[1];
    }
    for (int ia = 1; ia < a.na; ++ia) {
      const int p = __ldg(a.deg + ia);
      const R sa = S[(size_t)ia * n];
      R tt = dt[1] * sa;
      R hh = dt[2] * sa;
      for (int q = 2; q <= p; ++q) {
        const int *sg = a.seg + ((size_t)ia * (k + 1) + q) * 3;
        const int st = __ldg(sg), nn = __ldg(sg + 1), slot = __ldg(sg + 2);
        R bs = (R)0;
        if (q == 2) {
          for (int it = st; it < st + nn; ++it) {
            const uint32_t pk = __ldg(a.fq_pk + it);
            bs = bs + __ldg(coef + it) * S[(size_t)(pk & 0xffffu) * n] * S[(size_t)(pk >> 16) * n];
          }
        } else {
          for (int it = st; it < st + nn; ++it) {
            const uint32_t pk = __ldg(a.fq_pk + it);
            bs = bs + __ldg(coef + it) * S[(size_t)(pk & 0xffffu) * n] * B[(size_t)(pk >> 16) * nthr];
          }
        }
        if (slot >= 0) B[(size_t)slot * nthr] = bs;
        tt = tt + dt[q] * bs;
        hh = hh + dt[q + 1] * bs;
      }
      if (act) {
        T[(size_t)ia * n] = tt;
        if (TRAIN) H[(size_t)ia * n] = hh;
      }
    }
  }
}

struct AdjArgs {
  int n, na, npts;
  const int *pseg;
  const uint32_t *pair_pk;
  const void *pair_c;
  const void *Tb, *h;
  void *Sb;
  double *gbias;   // bias column of dW_l (stride m+1), accumulated
  int gstride;
};

// Bell adjoint of one hidden layer (l >= 3):
//   Sb^0 = sum_alpha Tb^alpha h^alpha,
//   Sb^beta = sum_{alpha >= beta} C(alpha,beta) Tb^alpha h^{alpha-beta}.
template <typename R>
__global__ void __launch_bounds__(128) k_bell_adj(AdjArgs a) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  const size_t plane = (size_t)a.na * a.n;
  const int n = a.n;
  const R *coef = (const R *)a.pair_c;
  double gb = 0.0;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *Tb = (const R *)a.Tb + pt * plane + j;
    const R *H = (const R *)a.h + pt * plane + j;
    R *Sb = (R *)a.Sb + pt * plane + j;
    R bs = Tb[0] * H[0];
    for (int ia = 1; ia < a.na; ++ia) bs = bs + Tb[(size_t)ia * n] * H[(size_t)ia * n];
    Sb[0] = bs;
    gb += (double)bs;
    for (int ib = 1; ib < a.na; ++ib) {
      const int st = __ldg(a.pseg + 2 * ib), nn = __ldg(a.pseg + 2 * ib + 1);
      R s = (R)0;
      for (int ip = st; ip < st + nn; ++ip) {
        const uint32_t pk = __ldg(a.pair_pk + ip);
        s = s + __ldg(coef + ip) * Tb[(size_t)(pk & 0xffffu) * n] * H[(size_t)(pk >> 16) * n];
      }
      Sb[(size_t)ib * n] = s;
    }
  }
  if (a.gbias) atomicAdd(a.gbias + (size_t)j * a.gstride, gb);
}

struct AdjL2Args {
  int n, na, d0, npts;
  const int *pseg, *ind_e1;
  const uint32_t *pair_pk;
  const void *pair_c;
  const void *Tb, *h;
  const double *X;
  double *g;      // dW_2 [n][d0+1], accumulated (null in row mode)
  double *rows;   // [P][nw] with the layer-2 block at woff (row mode)
  size_t nw, woff;
};

// Bell adjoint of the first hidden layer fused with its weight gradient.
// Its input plane is x and the unit vectors, so dW_2[j][0] = Sb^0 and
// dW_2[j][i] = Sb^0 x_i + Sb^{e_i} (lib/train_module.f90:409-422 with the
// analytic T of layer 1): only Sb^0 and the Sb^{e_i} are formed.
template <typename R>
__global__ void __launch_bounds__(128) k_bell_adj_l2(AdjL2Args a) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  const size_t plane = (size_t)a.na * a.n;
  const int n = a.n, d0 = a.d0;
  const R *coef = (const R *)a.pair_c;
  double acc[D0MAX + 1];
  for (int i = 0; i <= d0; ++i) acc[i] = 0.0;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *Tb = (const R *)a.Tb + pt * plane + j;
    const R *H = (const R *)a.h + pt * plane + j;
    R b0 = Tb[0] * H[0];
    for (int ia = 1; ia < a.na; ++ia) b0 = b0 + Tb[(size_t)ia * n] * H[(size_t)ia * n];
    const double *x = a.X + (size_t)pt * d0;
    double *row = a.rows ? a.rows + pt * a.nw + a.woff + (size_t)j * (d0 + 1) : nullptr;
    if (row) row[0] = (double)b0; else acc[0] += (double)b0;
    for (int i = 0; i < d0; ++i) {
      const int e = __ldg(a.ind_e1 + i);
      double v = (double)b0 * x[i];
      if (e >= 0) {
        const int st = __ldg(a.pseg + 2 * e), nn = __ldg(a.pseg + 2 * e + 1);
        R s = (R)0;
        for (int ip = st; ip < st + nn; ++ip) {
          const uint32_t pk = __ldg(a.pair_pk + ip);
          s = s + __ldg(coef + ip) * Tb[(size_t)(pk & 0xffffu) * n] * H[(size_t)(pk >> 16) * n];
        }
        v = v + (double)s;
      }
      if (row) row[1 + i] = v; else acc[1 + i] += v;
    }
  }
  if (a.g)
    for (int i = 0; i <= d0; ++i) atomicAdd(a.g + (size_t)j * (d0 + 1) + i, acc[i]);
}

struct OutArgs {
  int nout, m, na, npts, kind, nterm;
  const void *Tm;        // T_{L-1} [P][na][m]
  const double *W;       // W_L [nout][m+1]
  double *out;           // [P][na][nout] (may be null)
  double *seed;          // [P][nout][na] written by the rule (may be null)
  const double *coeff;
  const int *ind, *nonlin;
  double fac;
  double *loss;
  int nres;              // SEED_SYS
  const int *sys, *sfac;
  const double *wres;
  const double *src;     // [P][nres] sources (may be null)
};

// Residuals of a system rule at one point and the seed they imply
// (calc_sys_residual / set_sys_seed, app/pinn_module.f90:86-162), in the
// reference's order of operations; tl[nout][na] the point's outputs, sd
// (zeroed) receives the seed.  Returns the point's loss fac/2 sum_r w_r R_r^2.
__device__ double sys_seed(const OutArgs &a, const double *tl, double *sd, long pt) {
  const int na = a.na;
  double R[SYS_MAXRES];
  for (int r = 0; r < a.nres; ++r) R[r] = a.src ? -a.src[pt * a.nres + r] : 0.0;
  for (int k = 0; k < a.nterm; ++k) {
    const int r = a.sys[3 * k], nf = a.sys[3 * k + 1], f0 = a.sys[3 * k + 2];
    double prod = a.coeff[k];
    for (int m = 0; m < nf; ++m) prod = prod * tl[a.sfac[2 * (f0 + m)] * na + a.sfac[2 * (f0 + m) + 1]];
    R[r] = R[r] + prod;
  }
  double l = 0.0;
  for (int r = 0; r < a.nres; ++r) l += a.wres[r] * R[r] * R[r];
  for (int k = 0; k < a.nterm; ++k) {
    const int r = a.sys[3 * k], nf = a.sys[3 * k + 1], f0 = a.sys[3 * k + 2];
    for (int m = 0; m < nf; ++m) {
      double other = a.fac * a.wres[r] * R[r] * a.coeff[k];
      for (int mm = 0; mm < nf; ++mm) {
        if (mm == m) continue;
        other = other * tl[a.sfac[2 * (f0 + mm)] * na + a.sfac[2 * (f0 + mm) + 1]];
      }
      const int at = a.sfac[2 * (f0 + m)] * na + a.sfac[2 * (f0 + m) + 1];
      sd[at] = sd[at] + other;
    }
  }
  return 0.5 * a.fac * l;
}

// Output layer (identity read-out, lib/train_module.f90:326-328) and the
// seed of the loss at every point (app/pinn_module.f90:32-65).  One block
// per point; shared memory tl[nout][na] and sd[nout][na] (double).
template <typename R>
__global__ void __launch_bounds__(256) k_output_fwd(OutArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *tl = (double *)smem_raw;
  double *sd = tl + (size_t)a.nout * a.na;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int m = a.m, na = a.na, nout = a.nout;
  const size_t plane = (size_t)na * m;
  double lsum = 0.0;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *Tm = (const R *)a.Tm + pt * plane;
    for (int pr = warp; pr < na * nout; pr += nwarp) {
      const int ia = pr / nout, o = pr - ia * nout;
      const double *w = a.W + (size_t)o * (m + 1);
      double acc = 0.0;
      for (int i = lane; i < m; i += 32) acc += w[1 + i] * (double)Tm[(size_t)ia * m + i];
      acc = warp_sum(acc);
      if (lane == 0) {
        double v = (ia == 0 ? w[0] : 0.0) + acc;
        tl[o * na + ia] = v;
        if (a.out) a.out[(pt * (size_t)na + ia) * nout + o] = v;
      }
    }
    __syncthreads();
    if (a.seed && threadIdx.x == 0) {
      for (int i = 0; i < nout * na; ++i) sd[i] = 0.0;
      if (a.kind == SEED_HALFSQ) {
        double l = 0.0;
        for (int ia = 0; ia < na; ++ia) { sd[ia] = tl[ia]; l += tl[ia] * tl[ia]; }
        lsum += 0.5 * l;
      } else if (a.kind == SEED_SYS) {
        lsum += sys_seed(a, tl, sd, pt);
      } else {
        double R0 = 0.0;
        for (int t = 0; t < a.nterm; ++t) {
          const int ind = a.ind[t];
          if (a.nonlin[t]) R0 = R0 + a.coeff[t] * tl[0] * tl[ind];
          else R0 = R0 + a.coeff[t] * tl[ind];
        }
        double Rs = R0, fac = a.fac;
        if (a.kind == SEED_JROW) { Rs = 1.0; fac = 1.0; }
        else lsum += 0.5 * a.fac * R0 * R0;
        for (int t = 0; t < a.nterm; ++t) {
          const int ind = a.ind[t];
          if (a.nonlin[t]) {
            sd[ind] = sd[ind] + fac * Rs * a.coeff[t] * tl[0];
            sd[0] = sd[0] + fac * Rs * a.coeff[t] * tl[ind];
          } else {
            sd[ind] = sd[ind] + fac * Rs * a.coeff[t];
          }
        }
      }
      double *dst = a.seed + pt * (size_t)nout * na;
      for (int i = 0; i < nout * na; ++i) dst[i] = sd[i];
    }
    __syncthreads();
  }
  if (a.loss && threadIdx.x == 0 && lsum != 0.0) atomicAdd(a.loss, lsum);
}

struct OutAdjArgs {
  int nout, m, na, npts;
  const void *Tm;        // T_{L-1} [P][na][m]
  const double *W;       // W_L [nout][m+1]
  const double *seed;    // [P][nout][na]
  void *Tb;              // [P][na][m]
  double *g;             // dW_L [nout][m+1], accumulated
  double *rows;          // row mode
  size_t nw, woff;
};

// Adjoint of the output layer: Tb_{L-1} = W_L^T seed (:430-444) and
// dW_L += seed T_{L-1}^T (:409-422).  Gradient partials stay in registers
// across the block's points and are added once.
template <typename R>
__global__ void __launch_bounds__(256) k_output_adj(OutAdjArgs a) {
  const int m = a.m, na = a.na, nout = a.nout;
  const size_t plane = (size_t)na * m;
  constexpr int MAXO = 4, MAXI = 4;
  double acc[MAXO][MAXI + 1];
  for (int o = 0; o < MAXO; ++o)
    for (int r = 0; r <= MAXI; ++r) acc[o][r] = 0.0;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *Tm = (const R *)a.Tm + pt * plane;
    const double *sd = a.seed + pt * (size_t)nout * na;
    int r = 0;
    for (int i = threadIdx.x; i < m; i += blockDim.x, ++r) {
      R *Tb = (R *)a.Tb + pt * plane + i;
      for (int ia = 0; ia < na; ++ia) {
        double tb = 0.0;
        for (int o = 0; o < nout; ++o) tb += a.W[(size_t)o * (m + 1) + 1 + i] * sd[o * na + ia];
        Tb[(size_t)ia * m] = (R)tb;
      }
      for (int o = 0; o < nout; ++o) {
        double gi = 0.0;
        for (int ia = 0; ia < na; ++ia) gi += sd[o * na + ia] * (double)Tm[(size_t)ia * m + i];
        if (a.rows) a.rows[pt * a.nw + a.woff + (size_t)o * (m + 1) + 1 + i] = gi;
        else acc[o][1 + r] += gi;
      }
    }
    if (threadIdx.x < nout) {
      const int o = threadIdx.x;
      if (a.rows) a.rows[pt * a.nw + a.woff + (size_t)o * (m + 1)] = sd[o * na];
      else acc[o][0] += sd[o * na];
    }
  }
  if (a.rows || !a.g) return;
  int r = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x, ++r)
    for (int o = 0; o < nout; ++o) atomicAdd(a.g + (size_t)o * (m + 1) + 1 + i, acc[o][1 + r]);
  if (threadIdx.x < nout) atomicAdd(a.g + (size_t)threadIdx.x * (m + 1), acc[threadIdx.x][0]);
}


// ------------------------------------------------- streaming layer kernels
// One warp per point, the lane index the neuron of a 32-neuron tile
// (blockIdx.y): every plane row a warp touches is one coalesced line.

struct L2vArgs {
  int n, na, d0, npts;
  int ds[KMAX + 2];        // slots of degree p: [ds[p], ds[p + 1])
  int iact;
  const int *par;          // [na]
  const double *tpc;
  const double *X;         // [P][d0]
  const double *W;         // [n][d0 + 1]
  void *T, *h;             // [P][na][n]
  void *sig;               // [P][KK + 2][n]: s^(q)(S^0) (null: not kept)
};

// First hidden layer, analytic (see k_layer2): T^a = s^(|a|) W^a with the
// monomial W^a = prod_i W_i^{a_i} of each neuron built once per block in
// shared memory along unit steps, M[a] = M[a - e_i] W_i.  The slots are
// graded, so each degree is one contiguous run sharing s^(p).
template <typename R, int KK, bool TRAIN>
__global__ void __launch_bounds__(256) k_layer2v(L2vArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *M = (R *)smem_raw;  // [na][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int j = blockIdx.y * 32 + lane;
  const bool act = j < a.n;
  const double *wr = a.W + (size_t)(act ? j : a.n - 1) * (a.d0 + 1);
  if (warp == 0) {
    M[lane] = (R)1;
    for (int ia = 1; ia < a.na; ++ia) {
      const int pk = __ldg(a.par + ia);
      M[ia * 32 + lane] = (R)((double)M[(pk & 0xffff) * 32 + lane] * wr[1 + (pk >> 16)]);
    }
  }
  __syncthreads();
  const size_t plane = (size_t)a.na * a.n;
  for (long pt = (long)blockIdx.x * nw + warp; pt < a.npts; pt += (long)gridDim.x * nw) {
    const double *x = a.X + pt * a.d0;
    double s = wr[0];
    for (int i = 0; i < a.d0; ++i) s = s + wr[1 + i] * x[i];
    double d[KK + 2];
    sigma_derivs(a.iact, a.tpc, KK, s, d);
    R *T = (R *)a.T + pt * plane + j;
    R *H = TRAIN ? (R *)a.h + pt * plane + j : nullptr;
    if (a.sig && act) {
      R *G = (R *)a.sig + (size_t)pt * (KK + 2) * a.n + j;
#pragma unroll
      for (int q = 0; q <= KK + 1; ++q) G[(size_t)q * a.n] = (R)d[q];
    }
#pragma unroll
    for (int p = 0; p <= KK; ++p) {
      const R dp = (R)d[p], dq = (R)d[p + 1];
      const int e = a.ds[p + 1];
#pragma unroll 4
      for (int ia = a.ds[p]; ia < e; ++ia) {
        const R m = M[ia * 32 + lane];
        if (act) {
          T[(size_t)ia * a.n] = dp * m;
          if (TRAIN) H[(size_t)ia * a.n] = dq * m;
        }
      }
    }
  }
}

struct AdjL2vArgs {
  int n, na, npts;
  const int *up;           // [na][D0]
  const void *Tb, *h;
  const double *X;
  double *g;               // dW_2 [n][D0 + 1], accumulated (null in row mode)
  double *rows;            // [P][nw] (row mode)
  size_t nw, woff;
};

// Bell adjoint of the first hidden layer fused with dW_2 (see k_bell_adj_l2):
//   Sb^0 = sum_g Tb^g h^g,  Sb^{e_i} = sum_g (g_i + 1) Tb^{g + e_i} h^g,
//   dW_2[j][0] += Sb^0,  dW_2[j][1 + i] += Sb^0 x_i + Sb^{e_i}.
template <typename R, int D0>
__global__ void __launch_bounds__(256) k_adj_l2v(AdjL2vArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int *up = (int *)smem_raw;  // [na][D0], copied once per block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int j = blockIdx.y * 32 + lane;
  const bool act = j < a.n;
  const int jc = act ? j : a.n - 1;
  const size_t plane = (size_t)a.na * a.n;
  for (int e = threadIdx.x; e < a.na * D0; e += blockDim.x) up[e] = __ldg(a.up + e);
  __syncthreads();
  double acc[D0 + 1];
#pragma unroll
  for (int i = 0; i <= D0; ++i) acc[i] = 0.0;
  for (long pt = (long)blockIdx.x * nw + warp; pt < a.npts; pt += (long)gridDim.x * nw) {
    const R *Tb = (const R *)a.Tb + pt * plane + jc;
    const R *H = (const R *)a.h + pt * plane + jc;
    R s[D0 + 1];
#pragma unroll
    for (int i = 0; i <= D0; ++i) s[i] = (R)0;
    // four multi-indices per step: their loads are independent and issue
    // together; a missing child (u < 0) reads row 0 with weight 0
    int g = 0;
    for (; g + 4 <= a.na; g += 4) {
      R hv[4], tv[4], cv[4][D0], wv[4][D0];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        hv[q] = H[(size_t)(g + q) * a.n];
        tv[q] = Tb[(size_t)(g + q) * a.n];
#pragma unroll
        for (int i = 0; i < D0; ++i) {
          const int u = up[(g + q) * D0 + i];
          wv[q][i] = u >= 0 ? (R)(u >> 16) : (R)0;
          cv[q][i] = Tb[(size_t)(u >= 0 ? (u & 0xffff) : 0) * a.n];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        s[0] += tv[q] * hv[q];
#pragma unroll
        for (int i = 0; i < D0; ++i) s[1 + i] += wv[q][i] * cv[q][i] * hv[q];
      }
    }
    for (; g < a.na; ++g) {
      const R hg = H[(size_t)g * a.n];
      s[0] += Tb[(size_t)g * a.n] * hg;
#pragma unroll
      for (int i = 0; i < D0; ++i) {
        const int u = up[g * D0 + i];
        if (u >= 0) s[1 + i] += (R)(u >> 16) * Tb[(size_t)(u & 0xffff) * a.n] * hg;
      }
    }
    const double *x = a.X + pt * D0;
    const double v0 = (double)s[0];
    if (a.rows) {
      if (act) {
        double *row = a.rows + pt * a.nw + a.woff + (size_t)j * (D0 + 1);
        row[0] = v0;
#pragma unroll
        for (int i = 0; i < D0; ++i) row[1 + i] = v0 * x[i] + (double)s[1 + i];
      }
    } else {
      acc[0] += v0;
#pragma unroll
      for (int i = 0; i < D0; ++i) acc[1 + i] += v0 * x[i] + (double)s[1 + i];
    }
  }
  if (a.g && act)
#pragma unroll
    for (int i = 0; i <= D0; ++i) atomicAdd(a.g + (size_t)j * (D0 + 1) + i, acc[i]);
}

// Sum of 8 values over the 32 lanes of a warp with 9 shuffles (not 40):
// each level hands half of the still-open rows to the partner lane.  On
// return, lanes 4r .. 4r + 3 hold the total of row r.
__device__ __forceinline__ double warp_sum8(double (&p)[8]) {
  const int lane = threadIdx.x & 31;
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  double q[4], r[2];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    q[k] = (b4 ? p[k + 4] : p[k]) + __shfl_xor_sync(0xffffffffu, b4 ? p[k] : p[k + 4], 16);
#pragma unroll
  for (int k = 0; k < 2; ++k)
    r[k] = (b3 ? q[k + 2] : q[k]) + __shfl_xor_sync(0xffffffffu, b3 ? q[k] : q[k + 2], 8);
  double v = (b2 ? r[1] : r[0]) + __shfl_xor_sync(0xffffffffu, b2 ? r[0] : r[1], 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v + __shfl_xor_sync(0xffffffffu, v, 1);
}

// Output layer and seed, one warp per point (see k_output_fwd for the
// formulas).  Shared memory per warp: tl[nout][na], sd[nout][na] (double).
// VEC (rows a whole number of 16-byte pieces): 8 rows per pass, each lane
// reading 16-byte pieces of every row, so that 8 loads per lane are in
// flight, one 8-row reduction (warp_sum8) per pass, and few enough
// registers for three blocks per SM.
template <typename R, bool VEC>
__global__ void __launch_bounds__(256, VEC ? 3 : 1) k_output_fwdv(OutArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int m = a.m, na = a.na, nout = a.nout;
  double *tl = (double *)smem_raw + (size_t)warp * 2 * nout * na;
  double *sd = tl + (size_t)nout * na;
  const size_t plane = (size_t)na * m;
  double lsum = 0.0;
  for (long pt = (long)blockIdx.x * nw + warp; pt < a.npts; pt += (long)gridDim.x * nw) {
    const R *Tm = (const R *)a.Tm + pt * plane;
    if constexpr (VEC) {
      constexpr int V = 16 / sizeof(R);  // values per 16-byte piece
      using VT = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
      for (int o = 0; o < nout; ++o) {
        const double *w = a.W + (size_t)o * (m + 1) + 1;
        for (int ia0 = 0; ia0 < na; ia0 += 8) {
          double p[8];
#pragma unroll
          for (int r = 0; r < 8; ++r) p[r] = 0.0;
          for (int c0 = lane * V; c0 < m; c0 += 32 * V) {
            double wv[V];
#pragma unroll
            for (int v = 0; v < V; ++v) wv[v] = __ldg(w + c0 + v);
            VT t[8];
#pragma unroll
            for (int r = 0; r < 8; ++r)
              if (ia0 + r < na) t[r] = __ldg((const VT *)(Tm + (size_t)(ia0 + r) * m + c0));
#pragma unroll
            for (int r = 0; r < 8; ++r)
              if (ia0 + r < na) {
                if constexpr (V == 4)
                  p[r] += wv[0] * (double)t[r].x + wv[1] * (double)t[r].y +
                          wv[2] * (double)t[r].z + wv[3] * (double)t[r].w;
                else
                  p[r] += wv[0] * (double)t[r].x + wv[1] * (double)t[r].y;
              }
          }
          const double tot = warp_sum8(p);
          const int ia = ia0 + (lane >> 2);
          if (!(lane & 3) && ia < na) {
            const double v = (ia == 0 ? a.W[(size_t)o * (m + 1)] : 0.0) + tot;
            tl[o * na + ia] = v;
            if (a.out) a.out[(pt * (size_t)na + ia) * nout + o] = v;
          }
        }
      }
    } else
    for (int o = 0; o < nout; ++o) {
      const double *w = a.W + (size_t)o * (m + 1) + 1;
      // four multi-indices per step, independent loads and reductions
      for (int ia0 = 0; ia0 < na; ia0 += 4) {
        double part[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = lane; i < m; i += 32) {
          const double wi = __ldg(w + i);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (ia0 + q < na) part[q] += wi * (double)Tm[(size_t)(ia0 + q) * m + i];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) part[q] = warp_sum(part[q]);
        if (lane < 4 && ia0 + lane < na) {
          const int ia = ia0 + lane;
          const double pv = lane == 0 ? part[0] : lane == 1 ? part[1] : lane == 2 ? part[2] : part[3];
          const double v = (ia == 0 ? a.W[(size_t)o * (m + 1)] : 0.0) + pv;
          tl[o * na + ia] = v;
          if (a.out) a.out[(pt * (size_t)na + ia) * nout + o] = v;
        }
      }
    }
    __syncwarp();
    if (a.seed) {
      for (int i = lane; i < nout * na; i += 32) sd[i] = 0.0;
      __syncwarp();
      if (lane == 0) {
        if (a.kind == SEED_HALFSQ) {
          double l = 0.0;
          for (int ia = 0; ia < na; ++ia) { sd[ia] = tl[ia]; l += tl[ia] * tl[ia]; }
          lsum += 0.5 * l;
        } else if (a.kind == SEED_SYS) {
          lsum += sys_seed(a, tl, sd, pt);
        } else {
          double R0 = 0.0;
          for (int t = 0; t < a.nterm; ++t) {
            const int ind = a.ind[t];
            if (a.nonlin[t]) R0 = R0 + a.coeff[t] * tl[0] * tl[ind];
            else R0 = R0 + a.coeff[t] * tl[ind];
          }
          double Rs = R0, fac = a.fac;
          if (a.kind == SEED_JROW) { Rs = 1.0; fac = 1.0; }
          else lsum += 0.5 * a.fac * R0 * R0;
          for (int t = 0; t < a.nterm; ++t) {
            const int ind = a.ind[t];
            if (a.nonlin[t]) {
              sd[ind] = sd[ind] + fac * Rs * a.coeff[t] * tl[0];
              sd[0] = sd[0] + fac * Rs * a.coeff[t] * tl[ind];
            } else {
              sd[ind] = sd[ind] + fac * Rs * a.coeff[t];
            }
          }
        }
      }
      __syncwarp();
      double *dst = a.seed + pt * (size_t)nout * na;
      for (int i = lane; i < nout * na; i += 32) dst[i] = sd[i];
    }
    __syncwarp();
  }
  if (a.loss && lane == 0 && lsum != 0.0) atomicAdd(a.loss, lsum);
}

// Adjoint of the output layer, one warp per point (see k_output_adj):
// Tb_{L-1}^a[i] = sum_o W_L[o][1+i] seed[o][a], dW_L[o][1+i] += sum_a
// seed[o][a] T_{L-1}^a[i].  Lane i + 32 t holds neuron i + 32 t, t < NT.
template <typename R, int MAXO, int NT>
__global__ void __launch_bounds__(256) k_output_adjv(OutAdjArgs a) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int m = a.m, na = a.na, nout = a.nout;
  const size_t plane = (size_t)na * m;
  double acc[MAXO][NT], acc0[MAXO];
  double w[MAXO][NT];
#pragma unroll
  for (int o = 0; o < MAXO; ++o) {
    acc0[o] = 0.0;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = lane + 32 * t;
      acc[o][t] = 0.0;
      w[o][t] = (o < nout && i < m) ? a.W[(size_t)o * (m + 1) + 1 + i] : 0.0;
    }
  }
  for (long pt = (long)blockIdx.x * nw + warp; pt < a.npts; pt += (long)gridDim.x * nw) {
    const R *Tm = (const R *)a.Tm + pt * plane;
    R *Tb = (R *)a.Tb + pt * plane;
    const double *sd = a.seed + pt * (size_t)nout * na;
    double pg[MAXO][NT];
#pragma unroll
    for (int o = 0; o < MAXO; ++o)
#pragma unroll
      for (int t = 0; t < NT; ++t) pg[o][t] = 0.0;
#pragma unroll 2
    for (int ia = 0; ia < na; ++ia) {
      double so[MAXO];
#pragma unroll
      for (int o = 0; o < MAXO; ++o) so[o] = o < nout ? __ldg(sd + o * na + ia) : 0.0;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int i = lane + 32 * t;
        if (i < m) {
          double tb = 0.0;
#pragma unroll
          for (int o = 0; o < MAXO; ++o) tb += w[o][t] * so[o];
          Tb[(size_t)ia * m + i] = (R)tb;
          const double tv = (double)Tm[(size_t)ia * m + i];
#pragma unroll
          for (int o = 0; o < MAXO; ++o) pg[o][t] += so[o] * tv;
        }
      }
    }
    if (a.rows) {
      double *row = a.rows + pt * a.nw + a.woff;
#pragma unroll
      for (int o = 0; o < MAXO; ++o)
        if (o < nout) {
#pragma unroll
          for (int t = 0; t < NT; ++t)
            if (lane + 32 * t < m) row[(size_t)o * (m + 1) + 1 + lane + 32 * t] = pg[o][t];
          if (lane == 0) row[(size_t)o * (m + 1)] = sd[o * na];
        }
    } else {
#pragma unroll
      for (int o = 0; o < MAXO; ++o) {
        acc0[o] += sd[o * na];
#pragma unroll
        for (int t = 0; t < NT; ++t) acc[o][t] += pg[o][t];
      }
    }
  }
  if (a.rows || !a.g) return;
#pragma unroll
  for (int o = 0; o < MAXO; ++o)
    if (o < nout) {
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (lane + 32 * t < m) atomicAdd(a.g + (size_t)o * (m + 1) + 1 + lane + 32 * t, acc[o][t]);
      if (lane == 0) atomicAdd(a.g + (size_t)o * (m + 1), acc0[o]);
    }
}

// --------------------------------------------------------- CUDA-core GEMM
// Tiled GEMM for the FP64 path (and the split path where the tensor-core
// kernel does not apply).  Three forms:
//   FWD: C[r][c] = sum_k A[r][k] B[c][1+k] (+ B[c][0] on rows r % na == 0)
//   DT : C[r][c] = sum_k A[r][k] B[k][1+c]
//   DW : G[c1][1+c2] += sum_r A[r][c1] X[r][c2]  (split over r, atomics)
enum { G_FWD = 0, G_DT = 1, G_DW = 2 };
struct GemmArgs {
  int M, N, K, na;
  const void *A, *B;
  int lda, ldb;
  void *C;
  int ldc;
  double *G;     // DW target
  int gld;
  int kchunk;    // DW rows per block
};

template <typename R, int MODE>
__global__ void __launch_bounds__(256) k_gemm(GemmArgs g) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ R As[BK][BM + 1];
  __shared__ R Bs[BK][BN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;  // M tiles on x (no 65535 cap)
  const R *A = (const R *)g.A;
  const R *B = (const R *)g.B;
  R acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj] = (R)0;
  int kbeg = 0, kend = g.K;
  if (MODE == G_DW) {
    kbeg = blockIdx.z * g.kchunk;
    kend = min(g.K, kbeg + g.kchunk);
  }
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += 256) {
      int kk, mm;
      R v = (R)0;
      if (MODE == G_DW) {
        kk = e / BM; mm = e - kk * BM;  // A[r][c1], c1 fastest
        int r = k0 + kk, c = m0 + mm;
        if (r < kend && c < g.M) v = A[(size_t)r * g.lda + c];
      } else {
        mm = e / BK; kk = e - mm * BK;  // A[r][k], k fastest
        int r = m0 + mm, c = k0 + kk;
        if (r < g.M && c < kend) v = A[(size_t)r * g.lda + c];
      }
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < BN * BK; e += 256) {
      int kk, nn;
      R v = (R)0;
      if (MODE == G_FWD) {
        nn = e / BK; kk = e - nn * BK;
        int c = n0 + nn, kx = k0 + kk;
        if (c < g.N && kx < kend) v = B[(size_t)c * g.ldb + 1 + kx];
      } else if (MODE == G_DT) {
        kk = e / BN; nn = e - kk * BN;
        int kx = k0 + kk, c = n0 + nn;
        if (kx < kend && c < g.N) v = B[(size_t)kx * g.ldb + 1 + c];
      } else {
        kk = e / BN; nn = e - kk * BN;
        int r = k0 + kk, c = n0 + nn;
        if (r < kend && c < g.N) v = B[(size_t)r * g.ldb + c];
      }
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      R av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) bv[jj] = Bs[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[i][jj] += av[i] * bv[jj];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = m0 + ty + 16 * i;
    if (r >= g.M) continue;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int c = n0 + tx + 16 * jj;
      if (c >= g.N) continue;
      if (MODE == G_FWD) {
        R v = acc[i][jj];
        if (r % g.na == 0) v = B[(size_t)c * g.ldb] + v;
        ((R *)g.C)[(size_t)r * g.ldc + c] = v;
      } else if (MODE == G_DT) {
        ((R *)g.C)[(size_t)r * g.ldc + c] = acc[i][jj];
      } else {
        atomicAdd(g.G + (size_t)r * g.gld + 1 + c, (double)acc[i][jj]);
      }
    }
  }
}

// Per-point weight gradient rows of a hidden layer l >= 3 (Jacobian rows of
// a residual, app/lib_net_module.f90:314-330): one block per point.
template <typename R>
__global__ void k_dw_rows(int n, int m, int na, int npts, const void *Sbv,
                          const void *Tmv, double *rows, size_t nw, size_t woff) {
  for (int pt = blockIdx.x; pt < npts; pt += gridDim.x) {
    const R *Sb = (const R *)Sbv + (size_t)pt * na * n;
    const R *Tm = (const R *)Tmv + (size_t)pt * na * m;
    double *row = rows + pt * nw + woff;
    for (int e = threadIdx.x; e < n * (m + 1); e += blockDim.x) {
      const int j = e / (m + 1), i = e - j * (m + 1);
      double v = 0.0;
      if (i == 0) {
        v = (double)Sb[j];
      } else {
        for (int ia = 0; ia < na; ++ia)
          v += (double)Sb[(size_t)ia * n + j] * (double)Tm[(size_t)ia * m + i - 1];
      }
      row[(size_t)j * (m + 1) + i] = v;
    }
  }
}

__global__ void k_to_f32(const double *a, float *b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// --------------------------------------------------------------- planes
static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Threads per block of the Bell forward kernel and whether its state fits
// in shared memory.
static void bell_shape(int nslot, size_t rsz, int n, int *nthr, size_t *smem) {
  const size_t budget = 200 * 1024;
  int t = std::min(128, (n + 31) / 32 * 32);
  while (t > 32 && (size_t)nslot * t * rsz > budget) t -= 32;
  *nthr = t;
  *smem = (size_t)nslot * t * rsz;
}

int ensure_planes(const DevTables &t, const DevNet &net, int prec, int cap_pts,
                  Planes &p) {
  if (p.base && p.cap_pts >= cap_pts && p.prec == prec) return RC_OK;
  p.release();
  const size_t rsz = prec == PREC_F64 ? 8 : 4;
  const int L = net.nlayer;
  int nmax = 0;
  for (int l = 1; l < L; ++l) nmax = std::max(nmax, net.dims[l]);
  nmax = std::max(nmax, net.dims[0]);
  const size_t na = t.na, P = cap_pts;
  std::vector<size_t> off;
  size_t cur = 0;
  auto take = [&](size_t bytes) {
    size_t o = cur;
    cur = align_up(cur + bytes, 256);
    return o;
  };
  std::vector<size_t> oT(L, 0), oH(L, 0);
  for (int l = 2; l < L; ++l) {  // hidden layers 2..L-1 (1-based)
    oT[l - 1] = take(P * na * net.dims[l - 1] * rsz);
    oH[l - 1] = take(P * na * net.dims[l - 1] * rsz);
  }
  size_t oS = take(P * na * nmax * rsz);
  size_t oSb = take(P * na * nmax * rsz);
  size_t oTb = take(P * na * nmax * rsz);
  size_t oSeed = take(P * na * net.dims[L - 1] * sizeof(double));
  size_t oSig = take(P * (size_t)(t.k + 2) * net.dims[1] * rsz);
  size_t oX = take(P * t.d0 * sizeof(double));
  size_t oOut = take(P * na * net.dims[L - 1] * sizeof(double));
  size_t oLoss = take(sizeof(double) * 4);
  void *base = nullptr;
  CK(cudaMalloc(&base, cur));
  p.base = base;
  p.bytes = cur;
  p.cap_pts = cap_pts;
  p.prec = prec;
  char *b = (char *)base;
  p.T.assign(L, nullptr);
  p.h.assign(L, nullptr);
  for (int l = 2; l < L; ++l) {
    p.T[l - 1] = b + oT[l - 1];
    p.h[l - 1] = b + oH[l - 1];
  }
  p.S = b + oS;
  p.Sb = b + oSb;
  p.Tb = b + oTb;
  p.seed = b + oSeed;
  p.sig = b + oSig;
  p.X = (double *)(b + oX);
  p.out = (double *)(b + oOut);
  p.loss = (double *)(b + oLoss);
  // Bell state spill when a block of 32 threads cannot hold it in smem
  int nthr;
  size_t smem;
  bell_shape(t.nslot, rsz, nmax, &nthr, &smem);
  if (smem > 200 * 1024) {
    size_t bytes = (size_t)sm_count() * 4 * ((nmax + nthr - 1) / nthr) * t.nslot * nthr * rsz;
    CK(cudaMalloc(&p.scratch, bytes));
    p.scratch_bytes = bytes;
  }
  return RC_OK;
}

// ------------------------------------------------------------- launchers
template <typename R>
static int launch_bell_fwd(const DevTables &t, int n, int npts, const void *S,
                           void *T, void *h, bool train, Planes &p,
                           cudaStream_t st) {
  {
    int rc2 = bell_fwd2(t.bp, t, n, npts, S, T, h, train,
                        sizeof(R) == 8 ? PREC_F64 : PREC_SPLIT, st);
    if (rc2 != RC_UNSUPPORTED) return rc2;
  }
  int nthr;
  size_t smem;
  bell_shape(t.nslot, sizeof(R), n, &nthr, &smem);
  BellArgs a;
  a.n = n; a.na = t.na; a.k = t.k; a.nslot = t.nslot; a.npts = npts;
  a.iact = t.iact; a.deg = t.deg; a.seg = t.seg; a.fq_pk = t.fq_pk;
  a.fq_c = sizeof(R) == 8 ? (const void *)t.fq_c64 : (const void *)t.fq_c32;
  a.tpc = t.tpc; a.S = S; a.T = T; a.h = h; a.scratch = nullptr;
  const int gy = (n + nthr - 1) / nthr;
  int gx = npts;
  if (smem > 200 * 1024) {
    if (!p.scratch) { set_error("Bell state spill missing"); return RC_DEVICE; }
    a.scratch = p.scratch;
    gx = std::min(npts, grid_sms() * 4);
    smem = 0;
  }
  dim3 grid(gx, gy);
  if (train) {
    auto kfn = k_bell_fwd<R, true>;
    CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 0)));
    LAUNCH("k_bell_fwd", st, kfn<<<grid, nthr, smem, st>>>(a));
  } else {
    auto kfn = k_bell_fwd<R, false>;
    CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 0)));
    LAUNCH("k_bell_fwd", st, kfn<<<grid, nthr, smem, st>>>(a));
  }
  CK(cudaGetLastError());
  return RC_OK;
}

template <typename R>
static int launch_gemm_cc(int mode, int M, int N, int K, int na, const void *A,
                          int lda, const void *B, int ldb, void *C, int ldc,
                          double *G, int gld, cudaStream_t st, double *pack = nullptr) {
  if (sizeof(R) == 8) {
    // FP64 tensor cores (gemm_f64.cu); the CUDA-core tiles below take the
    // shapes it refuses (odd widths)
    const int rc = gemm_f64(mode, M, N, K, na, (const double *)A, lda, (const double *)B, ldb,
                            (double *)C, ldc, G, gld, st, pack);
    if (rc != RC_UNSUPPORTED) return rc;
  }
  GemmArgs g;
  g.M = M; g.N = N; g.K = K; g.na = na; g.A = A; g.B = B; g.lda = lda;
  g.ldb = ldb; g.C = C; g.ldc = ldc; g.G = G; g.gld = gld; g.kchunk = 0;
  if (mode == G_FWD) {
    dim3 grid((M + 63) / 64, (N + 63) / 64);
    LAUNCH("k_gemm", st, k_gemm<R, G_FWD><<<grid, 256, 0, st>>>(g));
  } else if (mode == G_DT) {
    dim3 grid((M + 63) / 64, (N + 63) / 64);
    LAUNCH("k_gemm", st, k_gemm<R, G_DT><<<grid, 256, 0, st>>>(g));
  } else {
    int tiles = ((N + 63) / 64) * ((M + 63) / 64);
    int splits = std::max(1, std::min((K + 255) / 256, grid_sms() * 8 / std::max(1, tiles)));
    g.kchunk = ((K + splits - 1) / splits + 15) / 16 * 16;
    // FP32 partial sums stay short: the reduction across blocks is FP64
    if (sizeof(R) == 4) g.kchunk = std::min(g.kchunk, 4096);
    splits = (K + g.kchunk - 1) / g.kchunk;
    dim3 grid((M + 63) / 64, (N + 63) / 64, splits);
    LAUNCH("k_gemm", st, k_gemm<R, G_DW><<<grid, 256, 0, st>>>(g));
  }
  CK(cudaGetLastError());
  return RC_OK;
}


static thread_local int g_grid_cap = 0;
int grid_sms() { return g_grid_cap > 0 ? std::min(g_grid_cap, sm_count()) : sm_count(); }
void set_grid_cap(int sms) { g_grid_cap = sms; }

// blocks of k resident at once on the SMs a launch may fill
static int occ_grid(const void *k, int threads, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return grid_sms() * per_sm;
}

template <typename R, int KK>
static int layer2v_k(const L2vArgs &a, bool train, cudaStream_t st) {
  const size_t smem = (size_t)a.na * 32 * sizeof(R);
  const void *k = train ? (const void *)k_layer2v<R, KK, true> : (const void *)k_layer2v<R, KK, false>;
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int gy = (a.n + 31) / 32;
  const int gx = std::max(1, std::min((a.npts + 7) / 8, occ_grid(k, 256, smem) / gy));
  dim3 grid(gx, gy);
  if (train) { LAUNCH("k_layer2", st, (k_layer2v<R, KK, true><<<grid, 256, smem, st>>>(a))); }
  else { LAUNCH("k_layer2", st, (k_layer2v<R, KK, false><<<grid, 256, smem, st>>>(a))); }
  CK(cudaGetLastError());
  return RC_OK;
}

// whether the first hidden layer runs analytically in both directions:
// k_layer2v forms T (and h would be s^(|g|+1) W^g), and the first-layer
// adjoint forms h itself, so a training forward writes no h plane for it.
// The forward and every adjoint of the same table set and width agree.
template <typename R>
static bool l2_analytic(const DevTables &t, int n) {
  return t.graded && t.k >= 1 && t.k <= 8 && (size_t)t.na * 32 * sizeof(R) <= 200 * 1024 &&
         (int)t.dstart.size() >= t.k + 2 &&
         bell_adj_l2s_analytic(t.d0, t.na, n, sizeof(R) == 8 ? PREC_F64 : PREC_SPLIT);
}

// streaming first hidden layer; RC_UNSUPPORTED when the shape is outside it
template <typename R>
static int launch_layer2v(const DevTables &t, int n, int npts, const double *X, const double *W,
                          void *T, void *h, bool train, cudaStream_t st, void *sig = nullptr) {
  if (!t.graded || t.k > 8 || (size_t)t.na * 32 * sizeof(R) > 200 * 1024) return RC_UNSUPPORTED;
  L2vArgs a;
  a.n = n; a.na = t.na; a.d0 = t.d0; a.npts = npts; a.iact = t.iact;
  for (int p = 0; p < KMAX + 2; ++p) a.ds[p] = p <= t.k + 1 ? t.dstart[std::min(p, t.k + 1)] : t.na;
  a.par = t.l2par; a.tpc = t.tpc; a.X = X; a.W = W; a.T = T; a.h = h; a.sig = sig;
  switch (t.k) {
    case 1: return layer2v_k<R, 1>(a, train, st);
    case 2: return layer2v_k<R, 2>(a, train, st);
    case 3: return layer2v_k<R, 3>(a, train, st);
    case 4: return layer2v_k<R, 4>(a, train, st);
    case 5: return layer2v_k<R, 5>(a, train, st);
    case 6: return layer2v_k<R, 6>(a, train, st);
    case 7: return layer2v_k<R, 7>(a, train, st);
    case 8: return layer2v_k<R, 8>(a, train, st);
    default: return RC_UNSUPPORTED;
  }
}

template <typename R, int D0>
static int adjl2v_k(const AdjL2vArgs &a, cudaStream_t st) {
  const void *k = (const void *)k_adj_l2v<R, D0>;
  const size_t smem = (size_t)a.na * D0 * sizeof(int);
  if (smem > 96 * 1024) return RC_UNSUPPORTED;
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int gy = (a.n + 31) / 32;
  const int gx = std::max(1, std::min((a.npts + 7) / 8, occ_grid(k, 256, smem) / gy));
  LAUNCH("k_bell_adj_l2", st, (k_adj_l2v<R, D0><<<dim3(gx, gy), 256, smem, st>>>(a)));
  CK(cudaGetLastError());
  return RC_OK;
}

template <typename R>
static int launch_adj_l2v(const DevTables &t, const AdjL2vArgs &a, cudaStream_t st) {
  switch (t.d0) {
    case 1: return adjl2v_k<R, 1>(a, st);
    case 2: return adjl2v_k<R, 2>(a, st);
    case 3: return adjl2v_k<R, 3>(a, st);
    case 4: return adjl2v_k<R, 4>(a, st);
    case 5: return adjl2v_k<R, 5>(a, st);
    case 6: return adjl2v_k<R, 6>(a, st);
    case 7: return adjl2v_k<R, 7>(a, st);
    case 8: return adjl2v_k<R, 8>(a, st);
    default: return RC_UNSUPPORTED;
  }
}

template <typename R>
static int launch_output_fwdv(const OutArgs &o, cudaStream_t st) {
  const size_t per_warp = (size_t)2 * o.nout * o.na * sizeof(double);
  const int wpb = (int)std::min<size_t>(8, (200 * 1024) / std::max<size_t>(per_warp, 1));
  if (wpb < 1) return RC_UNSUPPORTED;
  const size_t smem = per_warp * wpb;
  const bool vec = o.m % (16 / (int)sizeof(R)) == 0;
  const void *k = vec ? (const void *)k_output_fwdv<R, true> : (const void *)k_output_fwdv<R, false>;
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = std::max(1, std::min((o.npts + wpb - 1) / wpb, occ_grid(k, 32 * wpb, smem)));
  if (vec)
    LAUNCH("k_output_fwd", st, (k_output_fwdv<R, true><<<grid, 32 * wpb, smem, st>>>(o)));
  else
    LAUNCH("k_output_fwd", st, (k_output_fwdv<R, false><<<grid, 32 * wpb, smem, st>>>(o)));
  CK(cudaGetLastError());
  return RC_OK;
}

template <typename R, int NO, int NT>
static int outadjv_k(const OutAdjArgs &o, cudaStream_t st) {
  const void *k = (const void *)k_output_adjv<R, NO, NT>;
  const int grid = std::max(1, std::min((o.npts + 7) / 8, occ_grid(k, 256, 0)));
  LAUNCH("k_output_adj", st, (k_output_adjv<R, NO, NT><<<grid, 256, 0, st>>>(o)));
  CK(cudaGetLastError());
  return RC_OK;
}

template <typename R, int NO>
static int outadjv_nt(const OutAdjArgs &o, cudaStream_t st) {
  const int nt = (o.m + 31) / 32;
  if (nt <= 1) return outadjv_k<R, NO, 1>(o, st);
  if (nt <= 2) return outadjv_k<R, NO, 2>(o, st);
  if (nt <= 4) return outadjv_k<R, NO, 4>(o, st);
  if (nt <= 8) return outadjv_k<R, NO, 8>(o, st);
  return RC_UNSUPPORTED;
}

template <typename R>
static int launch_output_adjv(const OutAdjArgs &o, cudaStream_t st) {
  if (o.nout == 1) return outadjv_nt<R, 1>(o, st);
  if (o.nout == 2) return outadjv_nt<R, 2>(o, st);
  if (o.nout <= 4) return outadjv_nt<R, 4>(o, st);
  return RC_UNSUPPORTED;
}

// ------------------------------------------------------------- the driver
template <typename R>
struct Chunk {
  const DevTables &t;
  const DevNet &net;
  Planes &p;
  int c0, np;
  cudaStream_t st;
  bool split() const { return sizeof(R) == 4; }
  const double *W64(int l) const { return net.w64 + net.woff[l - 1]; }
  const void *W(int l) const {
    return split() ? (const void *)(net.w32 + net.woff[l - 1]) : (const void *)W64(l);
  }
  // the plain path's packed operands of layer l (null on the split path)
  double *pack(int l) const { return split() || !net.wpk ? nullptr : net.wpk + 2 * net.woff[l - 1]; }
};

// Forward of one chunk: hidden layers, read-out, and (seed != null) the
// rule's seed and loss.  train keeps the h planes for the adjoint.
template <typename R>
static int fwd_chunk(Chunk<R> &c, const DevRule *rule, const double *X,
                     double *out, double *seed, double *loss, bool train,
                     const double *src = nullptr) {
  const DevTables &t = c.t;
  const DevNet &net = c.net;
  Planes &p = c.p;
  const int L = net.nlayer, na = t.na, np = c.np, smc = grid_sms();
  int rc;
  {
    L2Args l2;
    l2.n = net.dims[1]; l2.na = na; l2.d0 = t.d0; l2.k = t.k; l2.iact = t.iact;
    l2.npts = np; l2.alpha = t.alpha; l2.deg = t.deg; l2.tpc = t.tpc; l2.X = X;
    l2.W = c.W64(2); l2.T = p.T[1]; l2.h = p.h[1];
    // the analytic adjoint forms the first layer's h itself from s^(q),
    // which the forward keeps instead of the h plane
    const bool an = train && l2_analytic<R>(t, l2.n);
    rc = launch_layer2v<R>(t, l2.n, np, X, l2.W, l2.T, l2.h, train && !an, c.st,
                           an ? p.sig : nullptr);
    if (rc == RC_UNSUPPORTED) {
      dim3 grid(std::min(np, smc * 8), (l2.n + 127) / 128);
      if (train) { LAUNCH("k_layer2", c.st, k_layer2<R, true><<<grid, 128, 0, c.st>>>(l2)); }
      else { LAUNCH("k_layer2", c.st, k_layer2<R, false><<<grid, 128, 0, c.st>>>(l2)); }
      CK(cudaGetLastError());
    } else if (rc) {
      return rc;
    }
  }
  for (int l = 3; l < L; ++l) {
    const int n = net.dims[l - 1], m = net.dims[l - 2];
    const int M = np * na;
    rc = c.split() && gemm_tc_available()
             ? gemm_tc_fwd(&net, l, M, n, m, na, p.T[l - 2], p.S, c.st)
             : RC_UNSUPPORTED;
    if (rc == RC_UNSUPPORTED)
      rc = launch_gemm_cc<R>(G_FWD, M, n, m, na, p.T[l - 2], m, c.W(l), m + 1, p.S, n,
                             nullptr, 0, c.st, c.pack(l));
    if (rc) return rc;
    rc = launch_bell_fwd<R>(t, n, np, p.S, p.T[l - 1], p.h[l - 1], train, p, c.st);
    if (rc) return rc;
  }
  OutArgs o;
  o.nout = net.dims[L - 1]; o.m = net.dims[L - 2]; o.na = na; o.npts = np;
  o.kind = rule ? rule->kind : SEED_HALFSQ;
  o.nterm = rule ? rule->nterm : 0;
  o.Tm = p.T[L - 2]; o.W = c.W64(L); o.out = out; o.seed = seed;
  o.coeff = rule ? rule->coeff : nullptr;
  o.ind = rule ? rule->ind : nullptr;
  o.nonlin = rule ? rule->nonlin : nullptr;
  o.fac = rule ? rule->fac : 1.0;
  o.loss = loss;
  o.nres = rule ? rule->nres : 0;
  o.sys = rule ? rule->sys : nullptr;
  o.sfac = rule ? rule->sfac : nullptr;
  o.wres = rule ? rule->wres : nullptr;
  o.src = src;
  size_t smem = (size_t)2 * o.nout * na * sizeof(double);
  if (smem > 200 * 1024) { set_error("output layer too wide"); return RC_UNSUPPORTED; }
  rc = launch_output_fwdv<R>(o, c.st);
  if (rc != RC_UNSUPPORTED) return rc;
  CK(cudaFuncSetAttribute(k_output_fwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  LAUNCH("k_output_fwd", c.st, k_output_fwd<R><<<std::min(np, smc * 8), 256, smem, c.st>>>(o));
  CK(cudaGetLastError());
  return RC_OK;
}

// Adjoint of one chunk from seed [np][nout][na] (the forward's planes must
// be in place): output layer, hidden layers, first hidden layer.  Either
// accumulates into grad or writes per-point rows.
template <typename R>
static int adj_chunk(Chunk<R> &c, const double *X, const double *seed,
                     double *grad, double *rows) {
  const DevTables &t = c.t;
  const DevNet &net = c.net;
  Planes &p = c.p;
  const int L = net.nlayer, na = t.na, np = c.np, smc = grid_sms();
  const bool split = c.split();
  int rc;
  {
    OutAdjArgs o;
    o.nout = net.dims[L - 1]; o.m = net.dims[L - 2]; o.na = na; o.npts = np;
    o.Tm = p.T[L - 2]; o.W = c.W64(L); o.seed = seed; o.Tb = p.Tb;
    o.g = grad ? grad + net.woff[L - 1] : nullptr;
    o.rows = rows; o.nw = net.nw; o.woff = net.woff[L - 1];
    if (o.nout > 4 || o.m > 4 * 256) {
      set_error("output layer shape outside the device path (nout <= 4, width <= 1024)");
      return RC_UNSUPPORTED;
    }
    rc = launch_output_adjv<R>(o, c.st);
    if (rc == RC_UNSUPPORTED) {
      LAUNCH("k_output_adj", c.st, k_output_adj<R><<<std::min(np, smc * 8), 256, 0, c.st>>>(o));
      CK(cudaGetLastError());
    } else if (rc) {
      return rc;
    }
  }
  for (int l = L - 1; l >= 3; --l) {
    const int n = net.dims[l - 1], m = net.dims[l - 2];
    AdjArgs aj;
    aj.n = n; aj.na = na; aj.npts = np; aj.pseg = t.pseg; aj.pair_pk = t.pair_pk;
    aj.pair_c = split ? (const void *)t.pair_c32 : (const void *)t.pair_c64;
    aj.Tb = p.Tb; aj.h = p.h[l - 1]; aj.Sb = p.Sb;
    aj.gbias = rows || !grad ? nullptr : grad + net.woff[l - 1];
    aj.gstride = m + 1;
    rc = bell_adj2(t.bp, t, n, np, p.Tb, p.h[l - 1], p.Sb, aj.gbias, aj.gstride,
                   split ? PREC_SPLIT : PREC_F64, c.st);
    if (rc == RC_UNSUPPORTED) {
      dim3 grid(std::min(np, smc * 8), (n + 127) / 128);
      LAUNCH("k_bell_adj", c.st, k_bell_adj<R><<<grid, 128, 0, c.st>>>(aj));
      CK(cudaGetLastError());
    } else if (rc) {
      return rc;
    }
    const int M = np * na;
    if (rows) {
      LAUNCH("k_dw_rows", c.st, k_dw_rows<R><<<std::min(np, smc * 8), 256, 0, c.st>>>(n, m, na, np, p.Sb, p.T[l - 2],
                                                             rows, net.nw, net.woff[l - 1]));
      CK(cudaGetLastError());
    } else if (grad) {
      rc = split && gemm_tc_available()
               ? gemm_tc_dw(&net, l, M, n, m, p.Sb, p.T[l - 2], grad + net.woff[l - 1], c.st)
               : RC_UNSUPPORTED;
      if (rc == RC_UNSUPPORTED)
        rc = launch_gemm_cc<R>(G_DW, n, m, M, na, p.Sb, n, p.T[l - 2], m, nullptr, 0,
                               grad + net.woff[l - 1], m + 1, c.st);
      if (rc) return rc;
    }
    rc = split && gemm_tc_available() ? gemm_tc_dt(&net, l, M, n, m, p.Sb, p.Tb, c.st)
                                      : RC_UNSUPPORTED;
    if (rc == RC_UNSUPPORTED)
      rc = launch_gemm_cc<R>(G_DT, M, m, n, na, p.Sb, n, c.W(l), m + 1, p.Tb, m, nullptr,
                             0, c.st, c.pack(l) ? c.pack(l) + (size_t)n * m : nullptr);
    if (rc) return rc;
  }
  AdjL2Args a2;
  a2.n = net.dims[1]; a2.na = na; a2.d0 = t.d0; a2.npts = np; a2.pseg = t.pseg;
  a2.ind_e1 = t.ind_e1; a2.pair_pk = t.pair_pk;
  a2.pair_c = split ? (const void *)t.pair_c32 : (const void *)t.pair_c64;
  a2.Tb = p.Tb; a2.h = p.h[1]; a2.X = X;
  a2.g = rows || !grad ? nullptr : grad + net.woff[1];
  a2.rows = rows; a2.nw = net.nw; a2.woff = net.woff[1];
  L2Analytic an{c.W64(2), p.sig, t.l2par, t.k, t.dstart.data()};
  rc = bell_adj_l2s(t.d0, a2.n, na, np, t.l2up, p.Tb, p.h[1], X, a2.g, rows, net.nw,
                    net.woff[1], split ? PREC_SPLIT : PREC_F64, c.st,
                    l2_analytic<R>(t, a2.n) ? &an : nullptr);
  if (rc == RC_UNSUPPORTED && l2_analytic<R>(t, a2.n)) {
    // the forward wrote no h plane for this layer, so no other kernel may run
    set_error("first-layer adjoint: the analytic kernel refused a shape it was chosen for");
    return RC_DEVICE;
  }
  if (rc != RC_UNSUPPORTED) return rc;
  {
    AdjL2vArgs v;
    v.n = a2.n; v.na = na; v.npts = np; v.up = t.l2up; v.Tb = p.Tb; v.h = p.h[1]; v.X = X;
    v.g = a2.g; v.rows = rows; v.nw = net.nw; v.woff = net.woff[1];
    rc = launch_adj_l2v<R>(t, v, c.st);
    if (rc != RC_UNSUPPORTED) return rc;
  }
  dim3 grid(std::min(np, smc * 8), (a2.n + 127) / 128);
  LAUNCH("k_bell_adj_l2", c.st, k_bell_adj_l2<R><<<grid, 128, 0, c.st>>>(a2));
  CK(cudaGetLastError());
  return RC_OK;
}

template <typename R>
static int run_all(const DevTables &t, const DevNet &net, const DevRule &rule,
                   Planes &p, const BatchArgs &a, cudaStream_t st) {
  const int na = t.na, nout = net.dims[net.nlayer - 1];
  for (int c0 = 0; c0 < a.npts; c0 += p.cap_pts) {
    Chunk<R> c{t, net, p, c0, std::min(p.cap_pts, a.npts - c0), st};
    const double *X = a.X + (size_t)c0 * t.d0;
    double *out = a.out ? a.out + (size_t)c0 * na * nout : nullptr;
    const bool given = rule.kind == SEED_GIVEN;
    double *seed = (a.train && !given) ? (double *)p.seed : nullptr;
    int rc = fwd_chunk<R>(c, a.train && !given ? &rule : nullptr, X, out, seed, a.loss,
                          a.train, a.src ? a.src + (size_t)c0 * rule.nres : nullptr);
    if (rc) return rc;
    if (!a.train) continue;
    const double *sd = given ? a.seeds + (size_t)c0 * nout * na : seed;
    double *rows = rule.kind == SEED_JROW ? a.rows + (size_t)c0 * net.nw : nullptr;
    rc = adj_chunk<R>(c, X, sd, rows ? nullptr : a.grad, rows);
    if (rc) return rc;
  }
  return RC_OK;
}

int run_batch(const DevTables &t, const DevNet &net, const DevRule &rule,
              Planes &p, const BatchArgs &a, cudaStream_t st) {
  if (a.npts <= 0) return RC_OK;
  if (t.d0 > D0MAX) {
    set_error("input width above the device limit");
    return RC_UNSUPPORTED;
  }
  if (net.nlayer < 3) {
    set_error("networks without a hidden layer are not on the device path");
    return RC_UNSUPPORTED;
  }
  if (p.prec != a.prec || p.cap_pts < 1) {
    set_error("work space not prepared for this precision");
    return RC_BAD_ARG;
  }
  if (a.prec == PREC_SPLIT && !net.w32) {
    set_error("split-precision weights not uploaded");
    return RC_BAD_ARG;
  }
  if (a.train && rule.kind == SEED_JROW && !a.rows) {
    set_error("Jacobian rows requested without a row buffer");
    return RC_BAD_ARG;
  }
  return a.prec == PREC_F64 ? run_all<double>(t, net, rule, p, a, st)
                            : run_all<float>(t, net, rule, p, a, st);
}

// Forward of npts <= cap points keeping every plane (for a later
// adjoint_kept), and the adjoint from a caller seed on those planes.
int forward_keep(const DevTables &t, const DevNet &net, Planes &p, int prec,
                 int npts, const double *X, double *out, cudaStream_t st) {
  if (npts > p.cap_pts || p.prec != prec) {
    set_error("kept forward needs a work space of at least npts points");
    return RC_BAD_ARG;
  }
  if (prec == PREC_F64) {
    Chunk<double> c{t, net, p, 0, npts, st};
    return fwd_chunk<double>(c, nullptr, X, out, nullptr, nullptr, true);
  }
  Chunk<float> c{t, net, p, 0, npts, st};
  return fwd_chunk<float>(c, nullptr, X, out, nullptr, nullptr, true);
}

int adjoint_kept(const DevTables &t, const DevNet &net, Planes &p, int prec,
                 int npts, const double *X, const double *seed, double *grad,
                 cudaStream_t st) {
  if (npts > p.cap_pts || p.prec != prec) {
    set_error("kept adjoint needs the work space of its forward");
    return RC_BAD_ARG;
  }
  if (prec == PREC_F64) {
    Chunk<double> c{t, net, p, 0, npts, st};
    return adj_chunk<double>(c, X, seed, grad, nullptr);
  }
  Chunk<float> c{t, net, p, 0, npts, st};
  return adj_chunk<float>(c, X, seed, grad, nullptr);
}

// --------------------------------------------------------------- Adam
__global__ void k_adam(double *w, const double *g, double *m, double *v, int nw,
                       double eta, double b1, double b2, double eps, double nb,
                       double bc1, double bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    double gv = g[i] / nb;
    double mi = b1 * m[i] + (1.0 - b1) * gv;
    double vi = b2 * v[i] + (1.0 - b2) * (gv * gv);
    m[i] = mi;
    v[i] = vi;
    w[i] = w[i] - eta * (mi / bc1) / (sqrt(vi / bc2) + eps);
  }
}

int adam_device(double *w, const double *g, double *m, double *v, int nw,
                double eta, double b1, double b2, double eps, int nbatch,
                int istep, cudaStream_t st) {
  int s = istep > 1 ? istep : 1;
  double p1 = 1.0, p2 = 1.0, x1 = b1, x2 = b2;
  for (unsigned u = (unsigned)s;;) {
    if (u & 1u) { p1 *= x1; p2 *= x2; }
    u >>= 1;
    if (!u) break;
    x1 *= x1;
    x2 *= x2;
  }
  LAUNCH("k_adam", st, k_adam<<<std::max(1, std::min((nw + 255) / 256, 1024)), 256, 0, st>>>(
      w, g, m, v, nw, eta, b1, b2, eps, (double)nbatch, 1.0 - p1, 1.0 - p2));
  CK(cudaGetLastError());
  return RC_OK;
}

int weights_to_f32(const double *w, float *w32, size_t n, cudaStream_t st) {
  LAUNCH("k_to_f32", st, k_to_f32<<<std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 1024)), 256, 0, st>>>(w, w32, n));
  CK(cudaGetLastError());
  return RC_OK;
}

}  // namespace dnnf90
