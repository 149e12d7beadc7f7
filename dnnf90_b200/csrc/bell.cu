// bell.cu - warp-cooperative Bell forward and adjoint kernels.
//
// One block owns one point and NPB neurons (32 in FP32, 16 in FP64) and
// keeps, in shared memory, that point's pre-activation series S [na][NPB],
// the kept Bell values B_{a,q} [nslot][NPB] and sigma^(q) [K+2][NPB].  The
// lane index is the neuron, so every shared-memory access of a warp is one
// row of NPB consecutive words (conflict-free) and every table read is
// warp-uniform.  The warps of the block share the state and split the
// multi-indices of each degree between them (work lists of bell_plan.cpp);
// a barrier separates the degrees, since degree p reads only degrees < p.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "bell.hpp"
#include "engine.hpp"
#include "kernels.cuh"

namespace dnnf90 {

#define CKB(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));   \
      return e_ == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;   \
    }                                                                  \
  } while (0)

// the tanh series forward (v9), off by default: it carries 2.7x fewer
// multiply-adds than the Bell recurrence but loads 8 bytes of shared memory
// per multiply-add against about 4 for the v8 bands, and measured slower
// (C3: 24.9 against 20.0 ms per FP32 launch).  dnnf90_tune_force(2, 1)
// switches it on.
static std::atomic<bool> g_series_fwd{false};

void DevBellPlan::release() {
  {
    void *q[] = {f8.list, f8.hdr, f8.cpdst, f8.rec, f9.list, f9.hdr, f9.rec, f9.sdeg64,
                 f9.sdeg32};
    for (void *p : q)
      if (p) cudaFree(p);
  }
  for (auto &D : a7) {
    void *q[] = {D.list, D.unit, D.out, D.fin, D.glist, D.rec};
    for (void *p : q)
      if (p) cudaFree(p);
  }
  void *ps[] = {fw_list, fw_arec, fw_grec, fw_gc64, fw_gc32, aj_list, aj_orec, aj_pair,
                aj_c64, aj_c32, f3_list, f3_arec, f3_grec, f3_gc64, f3_gc32, a3_orec,
                a3_pair, sc64, sc32, f4_grec, a4_pair, f5_list, f5_arec, f5_rec, f5_cpdst,
                a5_pair, f6_rec};
  for (void *p : ps)
    if (p) cudaFree(p);
  tile.release();
  *this = DevBellPlan();
}

template <typename T>
static int put(T **d, const std::vector<T> &h) {
  size_t n = std::max<size_t>(h.size(), 1);
  CKB(cudaMalloc((void **)d, n * sizeof(T)));
  if (!h.empty()) CKB(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return RC_OK;
}

int upload_bell_plan(const TableSet &t, DevBellPlan &d) {
  static std::atomic<uint64_t> next_id{1};
  d.release();
  d.id = next_id++;
  BellPlan P = build_bell_plan(t, BELL_WORKERS, ADJ_WORKERS);
  d.workers = P.workers;
  d.k = P.k;
  d.na = P.na;
  d.nslot = P.nslot;
  std::vector<float> gc32(P.fw_gc.begin(), P.fw_gc.end());
  std::vector<float> ac32(P.aj_c.begin(), P.aj_c.end());
  int rc;
  if ((rc = put(&d.fw_list, P.fw_list))) return rc;
  if ((rc = put(&d.fw_arec, P.fw_arec))) return rc;
  if ((rc = put(&d.fw_grec, P.fw_grec))) return rc;
  if ((rc = put(&d.fw_gc64, P.fw_gc))) return rc;
  if ((rc = put(&d.fw_gc32, gc32))) return rc;
  if ((rc = put(&d.aj_list, P.aj_list))) return rc;
  if ((rc = put(&d.aj_orec, P.aj_orec))) return rc;
  if ((rc = put(&d.aj_pair, P.aj_pair))) return rc;
  if ((rc = put(&d.aj_c64, P.aj_c))) return rc;
  if ((rc = put(&d.aj_c32, ac32))) return rc;
  std::vector<float> g3(P.f3_gc.begin(), P.f3_gc.end());
  if ((rc = put(&d.f3_list, P.f3_list))) return rc;
  if ((rc = put(&d.f3_arec, P.f3_arec))) return rc;
  if ((rc = put(&d.f3_grec, P.f3_grec))) return rc;
  if ((rc = put(&d.f3_gc64, P.f3_gc))) return rc;
  if ((rc = put(&d.f3_gc32, g3))) return rc;
  if ((rc = put(&d.a3_orec, P.a3_orec))) return rc;
  if ((rc = put(&d.a3_pair, P.a3_pair))) return rc;
  if ((rc = put(&d.f4_grec, P.f4_grec))) return rc;
  std::vector<uint32_t> a4(P.a4_pair);
  for (int i = 0; i < 4; ++i) a4.push_back(0);
  if ((rc = put(&d.a4_pair, a4))) return rc;
  d.nuv = P.nuv;
  std::vector<double> sc(3 * (size_t)P.na);
  for (int i = 0; i < P.na; ++i) {
    sc[i] = P.fact[i];
    sc[P.na + i] = 1.0 / P.fact[i];
    sc[2 * P.na + i] = 1.0 / P.fact[i];
  }
  std::vector<float> sc32(sc.begin(), sc.end());
  if ((rc = put(&d.sc64, sc))) return rc;
  if ((rc = put(&d.sc32, sc32))) return rc;
  if ((rc = put(&d.f5_list, P.f5_list))) return rc;
  if ((rc = put(&d.f5_arec, P.f5_arec))) return rc;
  if ((rc = put(&d.f5_rec, P.f5_rec))) return rc;
  if ((rc = put(&d.f5_cpdst, P.f5_cpdst))) return rc;
  if ((rc = put(&d.f6_rec, P.f6_rec))) return rc;
  d.nrec32 = (int)P.f6_rec.size();
  d.norec = (int)P.a3_orec.size() / 4;
  {
    // adjoint pairs as (Tb row, h row) byte offsets; the kernel reads up to
    // three pairs past the last one of a list
    std::vector<uint32_t> a5(P.a3_pair.begin(), P.a3_pair.end());
    for (int i = 0; i < 8; ++i) a5.push_back(0);
    while (a5.size() % 4) a5.push_back(0);  // whole 16-byte pieces
    d.npair5 = (int)a5.size() / 2;
    if ((rc = put(&d.a5_pair, a5))) return rc;
  }
  for (int v = 0; v < 2; ++v) {
    const A7Plan &Q = v ? P.a7d : P.a7f;
    DevBellPlan::A7Dev &D = d.a7[v];
    if ((rc = put(&D.list, Q.list))) return rc;
    if ((rc = put(&D.unit, Q.unit))) return rc;
    if ((rc = put(&D.out, Q.out))) return rc;
    if ((rc = put(&D.glist, Q.glist))) return rc;
    if ((rc = put(&D.rec, Q.rec))) return rc;
    if ((rc = put(&D.fin, Q.fin))) return rc;
    D.nunit = (int)Q.unit.size() / 8;
    D.nout = (int)Q.out.size();
    D.nglist = (int)Q.glist.size();
    D.nrec = (int)Q.rec.size();
    D.nfin = (int)Q.fin.size() / 2;
    D.nscratch = Q.nscratch;
    D.ok = Q.ok;
  }
  {
    const F8Plan &F = P.f8;
    if ((rc = put(&d.f8.list, F.list))) return rc;
    if ((rc = put(&d.f8.hdr, F.hdr))) return rc;
    if ((rc = put(&d.f8.cpdst, F.cpdst))) return rc;
    if ((rc = put(&d.f8.rec, F.rec))) return rc;
    d.f8.nrec = (int)F.rec.size();
    d.f8.sbase1 = F.sbase1;
    d.f8.bbase = F.bbase;
    d.f8.uvbase = F.uvbase;
    d.f8.dtbase = F.dtbase;
    d.f8.recbase = F.recbase;
    d.f8.zuv = F.zuv;
    d.f8.smem = F.smem;
    d.f8.ok = F.ok;
  }
  {
    const F9Plan &F = P.f9;
    std::vector<float> s32(F.sdeg.begin(), F.sdeg.end());
    if ((rc = put(&d.f9.list, F.list))) return rc;
    if ((rc = put(&d.f9.hdr, F.hdr))) return rc;
    if ((rc = put(&d.f9.rec, F.rec))) return rc;
    if ((rc = put(&d.f9.sdeg64, F.sdeg))) return rc;
    if ((rc = put(&d.f9.sdeg32, s32))) return rc;
    d.f9.pbase = F.pbase;
    d.f9.qbase = F.qbase;
    d.f9.smem = F.smem;
    d.f9.ok = F.ok;
  }
  d.f5_ok = P.f5_ok;
  d.nrows5 = P.nrows5;
  d.zuv5 = P.zuv5;
  d.dt_off5 = P.dt_off5;
  d.f3_ok = P.f3_ok;
  d.nrows = P.nrows;
  d.dt_off = P.dt_off;
  if ((rc = upload_tile_plan(t, d.tile))) return rc;
  d.ready = true;
  return RC_OK;
}

struct Fwd2Args {
  int n, na, nslot, npts, iact, workers;
  const double *tpc;
  const int *list;
  const int4 *arec, *grec;
  const void *gc;
  const void *S;
  void *T, *h;
};

template <typename R, int KK, int NPB, bool TRAIN>
__global__ void __launch_bounds__(BELL_WORKERS * 32) k_bell_fwd2(Fwd2Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R *sS = (R *)smem_raw;
  R *sB = sS + (size_t)a.na * NPB;
  R *sD = sB + (size_t)a.nslot * NPB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int j = blockIdx.y * NPB + ln;
  const bool act = lact && j < a.n;
  const int n = a.n;
  const size_t plane = (size_t)a.na * n;
  const R *gc = (const R *)a.gc;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *S = (const R *)a.S + pt * plane;
    R *T = (R *)a.T + pt * plane;
    R *H = TRAIN ? (R *)a.h + pt * plane : nullptr;
    for (int ia = warp; ia < a.na; ia += BELL_WORKERS)
      if (lact) sS[ia * NPB + lane] = act ? S[(size_t)ia * n + j] : (R)0;
    __syncthreads();
    if (warp == 0 && lact) {
      double d[KK + 2];
      sigma_derivs(a.iact, a.tpc, KK, (double)sS[lane], d);
#pragma unroll
      for (int q = 0; q <= KK + 1; ++q) sD[q * NPB + lane] = (R)d[q];
      if (act) {
        T[j] = (R)d[0];
        if (TRAIN) H[j] = (R)d[1];
      }
    }
    __syncthreads();
    R dt[KK + 2];
#pragma unroll
    for (int q = 0; q <= KK + 1; ++q) dt[q] = sD[q * NPB + ln];
    for (int p = 1; p <= KK; ++p) {
      const int rs = __ldg(a.list + (p * BELL_WORKERS + warp) * 2);
      const int rn = __ldg(a.list + (p * BELL_WORKERS + warp) * 2 + 1);
      for (int r = rs; r < rs + rn; ++r) {
        const int4 ar = __ldg(a.arec + r);
        const int ia = ar.x & 0xffff, bb = ar.w;
        R acc[KK + 1];
#pragma unroll
        for (int q = 0; q <= KK; ++q) acc[q] = (R)0;
        // the group records of four groups are fetched together, so their
        // latency is paid once per four groups, not on every group
        const int gend = ar.y + ar.z;
        for (int g0 = ar.y; g0 < gend; g0 += BELL_UNROLL) {
          int4 gr[BELL_UNROLL];
          R cv[BELL_UNROLL];
#pragma unroll
          for (int u = 0; u < BELL_UNROLL; ++u) {
            const int gi = min(g0 + u, gend - 1);
            gr[u] = __ldg(a.grec + gi);  // ib, g, gbase, qmax
            cv[u] = __ldg(gc + gi);
          }
#pragma unroll
          for (int u = 0; u < BELL_UNROLL; ++u) {
            if (g0 + u < gend) {
              const R x = cv[u] * sS[gr[u].x * NPB + ln];
              if (KK >= 2) acc[2] += x * sS[gr[u].y * NPB + ln];
#pragma unroll
              for (int q = 3; q <= KK; ++q)
                if (q <= gr[u].w) acc[q] += x * sB[(gr[u].z + q - 3) * NPB + ln];
            }
          }
        }
        const R sa = sS[ia * NPB + ln];
        R tt = dt[1] * sa, hh = dt[2] * sa;
#pragma unroll
        for (int q = 2; q <= KK; ++q) {
          if (q <= p) {
            const R b = acc[q] * (R)(1.0 / q);
            if (bb >= 0 && lact) sB[(bb + q - 2) * NPB + lane] = b;
            tt += dt[q] * b;
            hh += dt[q + 1] * b;
          }
        }
        if (act) {
          T[(size_t)ia * n + j] = tt;
          if (TRAIN) H[(size_t)ia * n + j] = hh;
        }
      }
      __syncthreads();
    }
  }
}

struct Adj2Args {
  int n, na, npts, gstride;
  const int *list;
  const int4 *orec;
  const int *pair;
  const void *c;
  const void *Tb, *h;
  void *Sb;
  double *gbias;
};

template <typename R, int NPB>
__global__ void __launch_bounds__(ADJ_WORKERS * 32) k_bell_adj2(Adj2Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R *sT = (R *)smem_raw;
  R *sH = sT + (size_t)a.na * NPB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int j = blockIdx.y * NPB + ln;
  const bool act = lact && j < a.n;
  const int n = a.n;
  const size_t plane = (size_t)a.na * n;
  const R *cc = (const R *)a.c;
  const int rs = __ldg(a.list + warp * 2), rn = __ldg(a.list + warp * 2 + 1);
  double gb = 0.0;
  for (int pt = blockIdx.x; pt < a.npts; pt += gridDim.x) {
    const R *Tb = (const R *)a.Tb + pt * plane;
    const R *Hh = (const R *)a.h + pt * plane;
    R *Sb = (R *)a.Sb + pt * plane;
    for (int ia = warp; ia < a.na; ia += ADJ_WORKERS)
      if (lact) {
        sT[ia * NPB + lane] = act ? Tb[(size_t)ia * n + j] : (R)0;
        sH[ia * NPB + lane] = act ? Hh[(size_t)ia * n + j] : (R)0;
      }
    __syncthreads();
    for (int r = rs; r < rs + rn; ++r) {
      const int4 o = __ldg(a.orec + r);  // ib, pstart, pcount
      R s0 = (R)0, s1 = (R)0;
      const int pe = o.y + o.z;
      for (int ip = o.y; ip < pe; ip += 2 * ADJ_UNROLL) {
        int kk[2 * ADJ_UNROLL];
        R cv[2 * ADJ_UNROLL];
#pragma unroll
        for (int u = 0; u < 2 * ADJ_UNROLL; ++u) {
          const int pi = min(ip + u, pe - 1);
          kk[u] = __ldg(a.pair + pi);
          cv[u] = __ldg(cc + pi);
        }
#pragma unroll
        for (int u = 0; u < 2 * ADJ_UNROLL; ++u) {
          if (ip + u < pe) {
            const R v = cv[u] * sT[(kk[u] & 0xffff) * NPB + ln] * sH[(kk[u] >> 16) * NPB + ln];
            if (u & 1) s1 += v;
            else s0 += v;
          }
        }
      }
      const R s = s0 + s1;
      if (act) Sb[(size_t)o.x * n + j] = s;
      if (o.x == 0) gb += (double)s;
    }
    __syncthreads();
  }
  if (a.gbias && act && gb != 0.0) atomicAdd(a.gbias + (size_t)j * a.gstride, gb);
}


// ---------------------------------------------------------------- v5
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// 16-byte asynchronous copy global -> shared; src_bytes < 16 zero-fills
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Rows [0, nr) of a [na][n] plane slice (neurons j0..j0+NPB-1, 128 bytes a
// row) copied into shared rows dst[r * 128]; columns at or beyond n fill
// with zeros.  n is a multiple of 4, so every 16-byte piece is either
// wholly inside the row or wholly outside it.
template <int NPB, typename R>
__device__ __forceinline__ void stage_rows(unsigned char *dst, const R *src, int nr, int n,
                                           int j0, int nthreads) {
  constexpr int PER = 16 / sizeof(R);  // values per 16-byte piece
  for (int c = threadIdx.x; c < nr * 8; c += nthreads) {
    const int r = c >> 3, piece = c & 7;
    const int col = j0 + piece * PER;
    const int ok = col < n ? 16 : 0;
    const R *g = src + (size_t)r * n + (ok ? col : 0);
    cp_async16(dst + r * 128 + piece * 16, g, ok);
  }
}

struct Fwd5Args {
  int n, na, npts, iact, dt_off, nrows, gy;
  int zuv;             // byte offset of the zero U/V pair
  int nrec32;          // 32-bit records copied to shared memory (SREC)
  const double *tpc;
  const int *list;     // [(K+1) * workers][2]
  const int4 *arec;    // [*][2]
  const uint2 *rec;    // flat records (byte offsets into the state)
  const uint32_t *rec32;  // the same records as row indices
  const int *cpdst;    // [na]
  const void *sc;      // [0, na): a!, [na, 2na): 1/a!
  const void *S;
  void *T, *h;
};

// shared-memory value at byte offset off of the dynamic shared area
template <typename R>
__device__ __forceinline__ R &srow(unsigned char *sm, uint32_t off) {
  return *(R *)(sm + off);
}

// Records of the forward: from global memory as two byte offsets, or from
// a copy in shared memory as two row indices (x row | z row << 16).
template <bool SREC>
struct RecSrc;
template <>
struct RecSrc<false> {
  const uint2 *p;
  __device__ __forceinline__ uint2 get(int i) const { return __ldg(p + i); }
};
template <>
struct RecSrc<true> {
  const uint32_t *p;  // shared memory
  __device__ __forceinline__ uint2 get(int i) const {
    const uint32_t r = p[i];
    return make_uint2((r & 0xffffu) << 7, (r >> 16) << 7);
  }
};

// one band of groups whose g has degree D: acc[q] += S~_b B~_{g,q-1},
// q = 2..D+1, B~_{g,1} = S~_g.  q0/q1 are the next two records.
template <typename R, int D, int KK, bool SREC>
__device__ __forceinline__ void fwd_band(unsigned char *sm, uint32_t los, uint32_t lo,
                                         const RecSrc<SREC> &src, int &ri, uint2 &q0, uint2 &q1,
                                         int cnt, R (&acc)[KK + 1]) {
#pragma unroll 2
  for (int e = 0; e < cnt; ++e) {
    const uint2 r = q0;
    q0 = q1;
    q1 = src.get(ri + 2);
    ++ri;
    const R x = srow<R>(sm, los + r.x);
    const uint32_t z = (D == 1 ? los : lo) + r.y;
#pragma unroll
    for (int l = 0; l < D; ++l) acc[2 + l] += x * srow<R>(sm, z + l * 128);
  }
}

// Bell forward over factorial-normalised state (S~_b = S_b/b!,
// B~_{a,q} = B_{a,q}/a!): for degree p < K
//   B~_{a,q} = (1/q) sum_{0<b<a} S~_b B~_{a-b,q-1},  B~_{a,1} = S~_a,
//   T_a = a! sum_q s^(q) B~_{a,q},  h_a = a! sum_q s^(q+1) B~_{a,q},
// and U~_a, V~_a (sums with s^(q+1)/(q+1), s^(q+2)/(q+1)) kept for the top
// degree, where
//   T_a = a! (s' S~_a + sum_{0<b<a} S~_b U~_{a-b}),  likewise h_a with s'', V~
// (lib/train_module.f90:297-325 regrouped by b; the q = 1 terms of U, V
// carry S~_g itself).
template <typename R, int KK, int NPB, bool TRAIN, bool SREC>
__global__ void __launch_bounds__(BELL_WORKERS * 32) k_bell_fwd5(Fwd5Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  RecSrc<SREC> src;
  if constexpr (SREC) {
    // the records follow the state; copied once, read by every item
    uint32_t *rs = (uint32_t *)(sm + (size_t)(a.nrows + a.na) * 128);
    for (int i = threadIdx.x; i < a.nrec32 / 4; i += blockDim.x)
      ((uint4 *)rs)[i] = __ldg((const uint4 *)a.rec32 + i);
    src.p = rs;
  } else {
    src.p = a.rec;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int n = a.n;
  const size_t plane = (size_t)a.na * n;
  const uint32_t lo = ln * sizeof(R);  // this lane's column in every row
  const R *sc = (const R *)a.sc;
  const uint32_t sbuf1 = a.nrows * 128;
  int buf = 0;
  if (threadIdx.x < 16)  // the zero U/V pair (read by the padding records)
    *(uint4 *)(sm + a.zuv + threadIdx.x * 16) = make_uint4(0, 0, 0, 0);
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  if (it0 < it1)
    stage_rows<NPB, R>(sm, (const R *)a.S + (it0 % a.npts) * plane, a.na, n,
                       (int)(it0 / a.npts) * NPB, BELL_WORKERS * 32);
  cp_async_commit();
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * NPB + ln;
    const bool act = lact && j < n;
    if (it + 1 < it1)
      stage_rows<NPB, R>(sm + (buf ? 0 : sbuf1), (const R *)a.S + ((it + 1) % a.npts) * plane,
                         a.na, n, (int)((it + 1) / a.npts) * NPB, BELL_WORKERS * 32);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const uint32_t los = lo + (buf ? sbuf1 : 0);  // this lane in the current S rows
    // normalise S_b -> S_b / b! (row 0 keeps S_0); copy level 1 of each B run
    for (int ia = warp; ia < a.na; ia += BELL_WORKERS) {
      const int cd = __ldg(a.cpdst + ia);
      if (lact) {
        const R v = srow<R>(sm, los + ia * 128) * __ldg(sc + a.na + ia);
        srow<R>(sm, los + ia * 128) = v;
        if (cd >= 0) srow<R>(sm, lo + cd) = v;
      }
    }
    __syncthreads();
    R *T = (R *)a.T + pt * plane;
    R *H = TRAIN ? (R *)a.h + pt * plane : nullptr;
    if (warp == 0 && lact) {
      double d[KK + 2];
      sigma_derivs(a.iact, a.tpc, KK, (double)srow<R>(sm, los), d);
#pragma unroll
      for (int q = 0; q <= KK + 1; ++q) srow<R>(sm, lo + a.dt_off + q * 128) = (R)d[q];
      if (act) {
        T[j] = (R)d[0];
        if (TRAIN) H[j] = (R)d[1];
      }
    }
    __syncthreads();
    R dt[KK + 2];
#pragma unroll
    for (int q = 0; q <= KK + 1; ++q) dt[q] = srow<R>(sm, lo + a.dt_off + q * 128);
    R uc[KK + 1], vc[KK + 1];
#pragma unroll
    for (int q = 1; q < KK; ++q) {
      uc[q] = dt[q + 1] * (R)(1.0 / (q + 1));
      vc[q] = dt[q + 2] * (R)(1.0 / (q + 1));
    }
    for (int p = 1; p <= KK; ++p) {
      const int rs = __ldg(a.list + (p * BELL_WORKERS + warp) * 2);
      const int rn = __ldg(a.list + (p * BELL_WORKERS + warp) * 2 + 1);
      for (int r = rs; r < rs + rn; ++r) {
        const int4 A0 = __ldg(a.arec + 2 * r), A1 = __ldg(a.arec + 2 * r + 1);
        const int ia = A0.x & 0xffff;
        const R sa = srow<R>(sm, los + ia * 128);
        const R fa = __ldg(sc + ia);
        int ri = A0.y;
        uint2 q0 = src.get(ri), q1 = src.get(ri + 1);
        if (p == KK) {
          R tt = dt[1] * sa, hh = dt[2] * sa;
          if constexpr (SREC) {
            // four records per 16-byte load (lists aligned and padded to 4)
            const uint4 *rq = (const uint4 *)(src.p + A0.y);
            uint4 q = rq[0];
            auto top = [&](uint32_t r) {
              const R x = srow<R>(sm, los + ((r & 0xffffu) << 7));
              const uint32_t u = lo + ((r >> 16) << 7);
              tt += x * srow<R>(sm, u);
              hh += x * srow<R>(sm, u + 128);
            };
            const int m = A0.z >> 2;
            for (int e = 0; e < m; ++e) {
              const uint4 g4 = q;
              q = rq[e + 1];
              top(g4.x);
              top(g4.y);
              top(g4.z);
              top(g4.w);
            }
          } else {
#pragma unroll 2
            for (int e = 0; e < A0.z; ++e) {
              const uint2 g = q0;
              q0 = q1;
              q1 = src.get(ri + 2);
              ++ri;
              const R x = srow<R>(sm, los + g.x);
              const uint32_t u = lo + g.y;
              tt += x * srow<R>(sm, u);
              hh += x * srow<R>(sm, u + 128);
            }
          }
          if (act) {
            T[(size_t)ia * n + j] = fa * tt;
            if (TRAIN) H[(size_t)ia * n + j] = fa * hh;
          }
          continue;
        }
        R acc[KK + 1];
#pragma unroll
        for (int q = 0; q <= KK; ++q) acc[q] = (R)0;
        const uint64_t bands = ((uint64_t)(uint32_t)A0.w << 32) | (uint32_t)A1.w;
#pragma unroll
        for (int d = KK - 2; d >= 1; --d) {
          if (d < p) {
            const int cnt = (int)((bands >> (8 * (d - 1))) & 0xffu);
            // d is a compile-time constant after unrolling
            switch (d) {
              case 1: if constexpr (1 <= KK - 2) fwd_band<R, 1, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              case 2: if constexpr (2 <= KK - 2) fwd_band<R, 2, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              case 3: if constexpr (3 <= KK - 2) fwd_band<R, 3, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              case 4: if constexpr (4 <= KK - 2) fwd_band<R, 4, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              case 5: if constexpr (5 <= KK - 2) fwd_band<R, 5, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              case 6: if constexpr (6 <= KK - 2) fwd_band<R, 6, KK, SREC>(sm, los, lo, src, ri, q0, q1, cnt, acc); break;
              default: break;
            }
          }
        }
        R tt = dt[1] * sa, hh = dt[2] * sa, uu = uc[1] * sa, vv = vc[1] * sa;
#pragma unroll
        for (int q = 2; q < KK; ++q) {
          if (q <= p) {
            const R b = acc[q] * (R)(1.0 / q);
            if (A1.x >= 0 && lact) srow<R>(sm, lo + A1.x + (q - 1) * 128) = b;
            tt += dt[q] * b;
            hh += dt[q + 1] * b;
            uu += uc[q] * b;
            vv += vc[q] * b;
          }
        }
        if (A1.y >= 0 && lact) {
          srow<R>(sm, lo + A1.y) = uu;
          srow<R>(sm, lo + A1.y + 128) = vv;
        }
        if (act) {
          T[(size_t)ia * n + j] = fa * tt;
          if (TRAIN) H[(size_t)ia * n + j] = fa * hh;
        }
      }
      __syncthreads();
    }
    buf ^= 1;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------- v8
struct Fwd8Args {
  int n, na, npts, iact, gy, nrec;
  uint32_t sbase1, bbase, uvbase, dtbase, recbase, zuv;
  const double *tpc;
  const int *list;     // [(K+1) * workers][2]
  const int4 *hdr;     // [*][2]
  const uint32_t *rec;
  const int *cpdst;    // [na]
  const void *sc;      // [0, na): a!, [na, 2na): 1/a!
  const void *S;
  void *T, *h;
};

// the (U, V) pair of one lane: two adjacent values of a 256-byte row
template <typename R>
struct Pair;
template <>
struct Pair<float> {
  using T = float2;
};
template <>
struct Pair<double> {
  using T = double2;
};

// (t, h) += x * (u, v) as one packed FP32 multiply-add; the register pairs
// are formed inside the asm so that no value is moved through integer ops
__device__ __forceinline__ void fma_pair(float2 &th, float x, float2 uv) {
  asm("{\n\t.reg .b64 acc, xx, u;\n\t"
      "mov.b64 acc, {%0, %1};\n\t"
      "mov.b64 xx, {%2, %2};\n\t"
      "mov.b64 u, {%3, %4};\n\t"
      "fma.rn.f32x2 acc, xx, u, acc;\n\t"
      "mov.b64 {%0, %1}, acc;\n\t}"
      : "+f"(th.x), "+f"(th.y)
      : "f"(x), "f"(uv.x), "f"(uv.y));
}
__device__ __forceinline__ void fma_pair(double2 &th, double x, double2 uv) {
  th.x += x * uv.x;
  th.y += x * uv.y;
}

// one band of records whose g has degree D: acc[q] += S~_b B~_{g,q-1},
// q = 2..D+1 (B~_{g,1} = S~_g).  lx: this lane in the S buffer; lz: this
// lane in the region of g's rows.
template <typename R, int D, int NA>
__device__ __forceinline__ void band8(unsigned char *sm, uint32_t lx, uint32_t lz,
                                      const uint32_t *rp, int cnt, R (&acc)[NA]) {
#pragma unroll 4
  for (int e = 0; e < cnt; ++e) {
    const uint32_t r = rp[e];
    const R x = srow<R>(sm, lx + (r >> 16));
    const uint32_t z = lz + (r & 0xffffu) * 4;
#pragma unroll
    for (int l = 0; l < D; ++l) acc[2 + l] += x * srow<R>(sm, z + l * 128);
  }
}

// the bands of one target, D = DD down to 1
template <typename R, int DD, int NA>
struct Bands8 {
  static __device__ __forceinline__ void run(unsigned char *sm, uint32_t lx, uint32_t lb,
                                             const uint32_t *rp, uint64_t bands, R (&acc)[NA]) {
    const int cnt = (int)((bands >> (8 * (DD - 1))) & 0xffu);
    band8<R, DD, NA>(sm, lx, DD == 1 ? lx : lb, rp, cnt, acc);
    Bands8<R, DD - 1, NA>::run(sm, lx, lb, rp + cnt, bands, acc);
  }
};
template <typename R, int NA>
struct Bands8<R, 0, NA> {
  static __device__ __forceinline__ void run(unsigned char *, uint32_t, uint32_t,
                                             const uint32_t *, uint64_t, R (&)[NA]) {}
};

// what the targets of one item share
template <typename R, int KK>
struct Item8 {
  unsigned char *sm;
  const uint32_t *rs;  // records in shared memory
  uint32_t lo, lx;     // this lane's column; the same in the current S buffer
  R *T, *H;            // this point's planes, offset by this lane's neuron
  uint32_t lp;         // this lane's (U, V) pair inside a 256-byte pair row
  bool act;
  R dt[KK + 2], uc[KK + 1], vc[KK + 1];
};

// the targets of degree P this warp owns
template <typename R, int KK, int P, int NPB, bool TRAIN>
__device__ __forceinline__ void fwd8_degree(const Fwd8Args &a, const Item8<R, KK> &c, int warp) {
  const int ts = __ldg(a.list + (P * BELL_WORKERS + warp) * 2);
  const int tn = __ldg(a.list + (P * BELL_WORKERS + warp) * 2 + 1);
  const R *sc = (const R *)a.sc;
  const bool wr = NPB == 32 || (threadIdx.x & 31) < NPB;  // lanes that own a column
  for (int t = ts; t < ts + tn; ++t) {
    const int4 h0 = __ldg(a.hdr + 2 * t), h1 = __ldg(a.hdr + 2 * t + 1);
    const int ia = h0.x;
    const R sa = srow<R>(c.sm, c.lx + ia * 128);
    const R fa = __ldg(sc + ia);
    R tt = c.dt[1] * sa, hh = c.dt[2] * sa;
    if constexpr (P == KK) {
      // T_a = a! (s' S~_a + sum_b S~_b U~_{a-b}), h_a likewise with s'', V~;
      // four records per 16-byte load, one load per (U, V) pair
      using PR = typename Pair<R>::T;
      const uint4 *rq = (const uint4 *)(c.rs + h0.y);
      const uint32_t lz = a.uvbase + c.lp;
      const int m = h0.z >> 2;
      PR th;
      th.x = tt;
      th.y = hh;
      auto top = [&](uint32_t r) {
        const R x = srow<R>(c.sm, c.lx + (r >> 16));
        fma_pair(th, x, srow<PR>(c.sm, lz + (r & 0xffffu) * 4));
      };
      for (int e = 0; e < m; ++e) {
        const uint4 g4 = rq[e];
        top(g4.x);
        top(g4.y);
        top(g4.z);
        top(g4.w);
      }
      tt = th.x;
      hh = th.y;
    } else {
      R uu = c.uc[1] * sa, vv = c.vc[1] * sa;
      if constexpr (P >= 2) {
        R acc[P + 1];
#pragma unroll
        for (int q = 0; q <= P; ++q) acc[q] = (R)0;
        const uint64_t bands = (uint64_t)(uint32_t)h1.z << 32 | (uint32_t)h1.y;
        Bands8<R, P - 1, P + 1>::run(c.sm, c.lx, a.bbase + c.lo, c.rs + h0.y, bands, acc);
#pragma unroll
        for (int q = 2; q <= P; ++q) {
          const R b = acc[q] * (R)(1.0 / q);
          if (P <= KK - 2 && wr) srow<R>(c.sm, a.bbase + c.lo + h0.w + (q - 1) * 128) = b;
          tt += c.dt[q] * b;
          hh += c.dt[q + 1] * b;
          uu += c.uc[q] * b;
          vv += c.vc[q] * b;
        }
      }
      if (wr) {
        typename Pair<R>::T p;
        p.x = uu;
        p.y = vv;
        srow<typename Pair<R>::T>(c.sm, a.uvbase + c.lp + h1.x) = p;
      }
    }
    if (c.act) {
      c.T[(size_t)ia * a.n] = fa * tt;
      if (TRAIN) c.H[(size_t)ia * a.n] = fa * hh;
    }
  }
}

// Bell forward v8: the v5 recurrences (see k_bell_fwd5) over the F8Plan
// layout.  Every degree is its own code path with its bands unrolled, the
// records are read from shared memory as they are used, and the sigma
// derivatives are formed while the other warps normalise S.
template <typename R, int KK, int NPB, bool TRAIN>
__global__ void __launch_bounds__(BELL_WORKERS * 32) k_bell_fwd8(Fwd8Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  {
    uint4 *rs = (uint4 *)(sm + a.recbase);
    for (int i = threadIdx.x; i < a.nrec / 4; i += blockDim.x) rs[i] = __ldg((const uint4 *)a.rec + i);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int n = a.n, na = a.na;
  const size_t plane = (size_t)na * n;
  const R *sc = (const R *)a.sc;
  // zero rows: row na of both S buffers and the zero U/V pair
  if (threadIdx.x < 8) {
    *(uint4 *)(sm + na * 128 + threadIdx.x * 16) = make_uint4(0, 0, 0, 0);
    *(uint4 *)(sm + a.sbase1 + na * 128 + threadIdx.x * 16) = make_uint4(0, 0, 0, 0);
  } else if (threadIdx.x < 24) {
    *(uint4 *)(sm + a.uvbase + a.zuv + (threadIdx.x - 8) * 16) = make_uint4(0, 0, 0, 0);
  }
  Item8<R, KK> c;
  c.sm = sm;
  c.rs = (const uint32_t *)(sm + a.recbase);
  c.lo = ln * sizeof(R);
  c.lp = ln * 2 * sizeof(R);
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  if (it0 < it1)
    stage_rows<NPB, R>(sm, (const R *)a.S + (it0 % a.npts) * plane, na, n,
                       (int)(it0 / a.npts) * NPB, BELL_WORKERS * 32);
  cp_async_commit();
  int buf = 0;
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * NPB + ln;
    c.act = lact && j < n;
    // FP32: the next item's rows are copied after the barrier, into the
    // buffer the last item used, so no barrier ends the top degree; FP64
    // (measured faster so) copies before it and keeps that barrier
    constexpr bool LATE = sizeof(R) == 4;
    if (!LATE && it + 1 < it1)
      stage_rows<NPB, R>(sm + (buf ? 0 : a.sbase1), (const R *)a.S + ((it + 1) % a.npts) * plane,
                         na, n, (int)((it + 1) / a.npts) * NPB, BELL_WORKERS * 32);
    if (!LATE) {
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();  // this item's S rows are in; every warp is done with the last item
    if (LATE) {
      if (it + 1 < it1)
        stage_rows<NPB, R>(sm + (buf ? 0 : a.sbase1), (const R *)a.S + ((it + 1) % a.npts) * plane,
                           na, n, (int)((it + 1) / a.npts) * NPB, BELL_WORKERS * 32);
      cp_async_commit();
    }
    c.lx = (buf ? a.sbase1 : 0) + c.lo;
    c.T = (R *)a.T + pt * plane + j;
    c.H = TRAIN ? (R *)a.h + pt * plane + j : nullptr;
    if (warp == 0 && lact) {
      // S_0 is its own scaled value (0! = 1): sigma^(q)(S_0) into the sigma rows
      double d[KK + 2];
      sigma_derivs(a.iact, a.tpc, KK, (double)srow<R>(sm, c.lx), d);
#pragma unroll
      for (int q = 0; q <= KK + 1; ++q) srow<R>(sm, a.dtbase + c.lo + q * 128) = (R)d[q];
      if (c.act) {
        c.T[0] = (R)d[0];
        if (TRAIN) c.H[0] = (R)d[1];
      }
    }
    // S_b -> S_b / b!, and the level-1 copy of each B run
    for (int ia = warp; ia < na; ia += BELL_WORKERS) {
      if (ia == 0) continue;
      const int cd = __ldg(a.cpdst + ia);
      if (lact) {
        const R v = srow<R>(sm, c.lx + ia * 128) * __ldg(sc + na + ia);
        srow<R>(sm, c.lx + ia * 128) = v;
        if (cd >= 0) srow<R>(sm, a.bbase + c.lo + cd) = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q <= KK + 1; ++q) c.dt[q] = srow<R>(sm, a.dtbase + c.lo + q * 128);
#pragma unroll
    for (int q = 1; q < KK; ++q) {
      c.uc[q] = c.dt[q + 1] * (R)(1.0 / (q + 1));
      c.vc[q] = c.dt[q + 2] * (R)(1.0 / (q + 1));
    }
#pragma unroll
    for (int p = 1; p <= 8; ++p) {
      if (p <= KK) {
        switch (p) {
          case 1: fwd8_degree<R, KK, 1, NPB, TRAIN>(a, c, warp); break;
          case 2: if constexpr (KK >= 2) fwd8_degree<R, KK, 2, NPB, TRAIN>(a, c, warp); break;
          case 3: if constexpr (KK >= 3) fwd8_degree<R, KK, 3, NPB, TRAIN>(a, c, warp); break;
          case 4: if constexpr (KK >= 4) fwd8_degree<R, KK, 4, NPB, TRAIN>(a, c, warp); break;
          case 5: if constexpr (KK >= 5) fwd8_degree<R, KK, 5, NPB, TRAIN>(a, c, warp); break;
          case 6: if constexpr (KK >= 6) fwd8_degree<R, KK, 6, NPB, TRAIN>(a, c, warp); break;
          case 7: if constexpr (KK >= 7) fwd8_degree<R, KK, 7, NPB, TRAIN>(a, c, warp); break;
          case 8: if constexpr (KK >= 8) fwd8_degree<R, KK, 8, NPB, TRAIN>(a, c, warp); break;
          default: break;
        }
        if (p < KK || !LATE) __syncthreads();  // FP32: the top degree ends at the next item's barrier
      }
    }
    buf ^= 1;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------- v9
// tanh forward by the series identity of tanh' = 1 - tanh^2 (F9Plan):
//   |a| t~_a = sum_{0<b<=a} |b| s~_b u~_{a-b},  u~_a = -sum_{b+c=a} t~_b t~_c,
// T_a = a! t~_a and h_a = a! u~_a (h = sigma'(S) = 1 - T^2 for tanh).  One
// record (b, c) adds (|b| s~_b, t~_b) * (u~_c, t~_c) to the pair (T sum,
// U sum); the b = a and b = 0 terms are added after the loop.
struct Fwd9Args {
  int n, na, npts, iact, gy, pbase, qbase;
  const double *tpc;
  const int *list;     // [(K+1) * workers][2]
  const int4 *hdr;     // ia, first record, records, 0
  const uint4 *rec;    // two records (P offset, Q offset) per 16 bytes
  const void *sc;      // [0, na): a!
  const void *sdeg;    // [na]: |a| / a!
  const void *S;
  void *T, *h;
};

// (t, u) += (x0, x1) * (y0, y1) elementwise, one packed FP32 multiply-add
__device__ __forceinline__ void fma_pp(float2 &acc, float2 x, float2 y) {
  asm("{\n\t.reg .b64 a, xx, yy;\n\t"
      "mov.b64 a, {%0, %1};\n\t"
      "mov.b64 xx, {%2, %3};\n\t"
      "mov.b64 yy, {%4, %5};\n\t"
      "fma.rn.f32x2 a, xx, yy, a;\n\t"
      "mov.b64 {%0, %1}, a;\n\t}"
      : "+f"(acc.x), "+f"(acc.y)
      : "f"(x.x), "f"(x.y), "f"(y.x), "f"(y.y));
}
__device__ __forceinline__ void fma_pp(double2 &acc, double2 x, double2 y) {
  acc.x += x.x * y.x;
  acc.y += x.y * y.y;
}

template <typename R, int P>
__device__ __forceinline__ void fwd9_degree(const Fwd9Args &a, unsigned char *sm, uint32_t lp,
                                            R t0, R u0, R *T, R *H, bool act, bool wr,
                                            bool train, int warp) {
  using PR = typename Pair<R>::T;
  const int ts = __ldg(a.list + (P * BELL_WORKERS + warp) * 2);
  const int tn = __ldg(a.list + (P * BELL_WORKERS + warp) * 2 + 1);
  const R *sc = (const R *)a.sc;
  for (int t = ts; t < ts + tn; ++t) {
    const int4 hd = __ldg(a.hdr + t);
    PR acc;
    acc.x = (R)0;
    acc.y = (R)0;
    if constexpr (P >= 2) {
      const uint4 *rq = a.rec + (hd.y >> 1);
      const int m = hd.z >> 1;
#pragma unroll 2
      for (int e = 0; e < m; ++e) {
        const uint4 r = __ldg(rq + e);
        fma_pp(acc, srow<PR>(sm, r.x + lp), srow<PR>(sm, r.y + lp));
        fma_pp(acc, srow<PR>(sm, r.z + lp), srow<PR>(sm, r.w + lp));
      }
    }
    const int ia = hd.x;
    const uint32_t pa = a.pbase + ia * 256 + lp;
    const R sa = srow<R>(sm, pa);  // |a| s~_a
    const R tt = (acc.x + sa * u0) * (R)(1.0 / P);
    const R uu = -(acc.y + (R)2 * t0 * tt);
    if (wr) {
      srow<R>(sm, pa + sizeof(R)) = tt;
      PR q;
      q.x = uu;
      q.y = tt;
      srow<PR>(sm, a.qbase + ia * 256 + lp) = q;
    }
    if (act) {
      const R fa = __ldg(sc + ia);
      T[(size_t)ia * a.n] = fa * tt;
      if (train) H[(size_t)ia * a.n] = fa * uu;
    }
  }
}

template <typename R, int KK, int NPB, bool TRAIN>
__global__ void __launch_bounds__(BELL_WORKERS * 32) k_tanh_fwd9(Fwd9Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  using PR = typename Pair<R>::T;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int n = a.n, na = a.na;
  const size_t plane = (size_t)na * n;
  const R *sdeg = (const R *)a.sdeg;
  const uint32_t lo = ln * sizeof(R), lp = ln * 2 * sizeof(R);
  // zero rows: S row na, and the P and Q rows na that pad the record lists
  if (threadIdx.x < 8) {
    *(uint4 *)(sm + na * 128 + threadIdx.x * 16) = make_uint4(0, 0, 0, 0);
  } else if (threadIdx.x < 24) {
    *(uint4 *)(sm + a.pbase + na * 256 + (threadIdx.x - 8) * 16) = make_uint4(0, 0, 0, 0);
  } else if (threadIdx.x < 40) {
    *(uint4 *)(sm + a.qbase + na * 256 + (threadIdx.x - 24) * 16) = make_uint4(0, 0, 0, 0);
  }
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  if (it0 < it1)
    stage_rows<NPB, R>(sm, (const R *)a.S + (it0 % a.npts) * plane, na, n,
                       (int)(it0 / a.npts) * NPB, BELL_WORKERS * 32);
  cp_async_commit();
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * NPB + ln;
    const bool act = lact && j < n;
    cp_async_wait<0>();
    __syncthreads();  // this item's S rows are in; every warp is done with the last item
    R *T = (R *)a.T + pt * plane + j;
    R *H = TRAIN ? (R *)a.h + pt * plane + j : nullptr;
    if (warp == 0 && lact) {
      double d[KK + 2];  // the table's polynomials are laid out for K
      sigma_derivs(a.iact, a.tpc, KK, (double)srow<R>(sm, lo), d);
      PR q;
      q.x = (R)d[1];
      q.y = (R)d[0];
      srow<PR>(sm, a.qbase + lp) = q;  // (u~_0, t~_0)
      if (act) {
        T[0] = (R)d[0];
        if (TRAIN) H[0] = (R)d[1];
      }
    }
    // P rows: |b| s~_b = |b| S_b / b!
    for (int ia = 1 + warp; ia < na; ia += BELL_WORKERS)
      if (lact) srow<R>(sm, a.pbase + ia * 256 + lp) = srow<R>(sm, lo + ia * 128) * __ldg(sdeg + ia);
    __syncthreads();  // S is read: the next item's rows may stream in
    if (it + 1 < it1)
      stage_rows<NPB, R>(sm, (const R *)a.S + ((it + 1) % a.npts) * plane, na, n,
                         (int)((it + 1) / a.npts) * NPB, BELL_WORKERS * 32);
    cp_async_commit();
    const PR q0 = srow<PR>(sm, a.qbase + lp);
    const R u0 = q0.x, t0 = q0.y;
#pragma unroll
    for (int p = 1; p <= 8; ++p) {
      if (p <= KK) {
        switch (p) {
          case 1: fwd9_degree<R, 1>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 2: if constexpr (KK >= 2) fwd9_degree<R, 2>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 3: if constexpr (KK >= 3) fwd9_degree<R, 3>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 4: if constexpr (KK >= 4) fwd9_degree<R, 4>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 5: if constexpr (KK >= 5) fwd9_degree<R, 5>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 6: if constexpr (KK >= 6) fwd9_degree<R, 6>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 7: if constexpr (KK >= 7) fwd9_degree<R, 7>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          case 8: if constexpr (KK >= 8) fwd9_degree<R, 8>(a, sm, lp, t0, u0, T, H, act, lact, TRAIN, warp); break;
          default: break;
        }
        if (p < KK) __syncthreads();  // the top degree ends at the next item's barrier
      }
    }
  }
  cp_async_wait<0>();
}

struct Adj5Args {
  int n, na, npts, gstride, gy;
  int norec, npair;    // counts copied to shared memory (SREC)
  const int *list;
  const int4 *orec;    // ib, pstart, pcount, 0
  const uint2 *pair;   // byte offsets of the Tb row and the h row in a buffer
  const void *sc;      // [3][na]
  const void *Tb, *h;
  void *Sb;
  double *gbias;
};

// Bell adjoint as a correlation: Sb_b b! = sum_{a >= b} (a! Tb_a)(h_{a-b}/(a-b)!)
// (lib/train_module.f90:381-403 with C(a,b) folded into row scales).
// Shared memory holds two buffers of [Tb rows | h rows]; the next item's
// rows stream into one while the other is scaled and read.
template <typename R, int NPB, bool SREC>
__global__ void __launch_bounds__(ADJ_WORKERS * 32) k_bell_adj5(Adj5Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int n = a.n, na = a.na;
  const size_t plane = (size_t)na * n;
  const uint32_t bufb = 2 * na * 128;  // bytes per buffer
  const int4 *orec = a.orec;
  const uint2 *pair = a.pair;
  if constexpr (SREC) {
    // output records and pairs follow the two buffers; copied once
    int4 *so = (int4 *)(sm + (size_t)2 * bufb);
    uint2 *sp = (uint2 *)(so + a.norec);
    for (int i = threadIdx.x; i < a.norec; i += blockDim.x) so[i] = __ldg(a.orec + i);
    for (int i = threadIdx.x; i < a.npair / 2; i += blockDim.x)
      ((uint4 *)sp)[i] = __ldg((const uint4 *)a.pair + i);
    orec = so;
    pair = sp;
  }
  const R *sc = (const R *)a.sc;
  const int rs = __ldg(a.list + warp * 2), rn = __ldg(a.list + warp * 2 + 1);
  double gb = 0.0;
  int gj = -1;
  int buf = 0;
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  if (it0 < it1) {
    const size_t o = (it0 % a.npts) * plane;
    const int j0 = (int)(it0 / a.npts) * NPB;
    stage_rows<NPB, R>(sm, (const R *)a.Tb + o, na, n, j0, ADJ_WORKERS * 32);
    stage_rows<NPB, R>(sm + na * 128, (const R *)a.h + o, na, n, j0, ADJ_WORKERS * 32);
  }
  cp_async_commit();
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * NPB + ln;
    const bool act = lact && j < n;
    if (j != gj) {
      if (a.gbias && gj >= 0 && gj < n && lact && gb != 0.0)
        atomicAdd(a.gbias + (size_t)gj * a.gstride, gb);
      gb = 0.0;
      gj = j;
    }
    if (it + 1 < it1) {
      unsigned char *oth = sm + (buf ^ 1) * bufb;
      const size_t o = ((it + 1) % a.npts) * plane;
      const int j0 = (int)((it + 1) / a.npts) * NPB;
      stage_rows<NPB, R>(oth, (const R *)a.Tb + o, na, n, j0, ADJ_WORKERS * 32);
      stage_rows<NPB, R>(oth + na * 128, (const R *)a.h + o, na, n, j0, ADJ_WORKERS * 32);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const uint32_t lc = buf * bufb + ln * sizeof(R);  // this lane in the current buffer
    // scale: row a of Tb by a!, row g of h by 1/g!
    for (int r = warp; r < 2 * na; r += ADJ_WORKERS)
      if (lact) srow<R>(sm, lc + r * 128) *= __ldg(sc + r);
    __syncthreads();
    R *Sb = (R *)a.Sb + pt * plane;
    for (int r = rs; r < rs + rn; ++r) {
      const int4 o = SREC ? orec[r] : __ldg(orec + r);  // ib, pstart, pcount
      const uint2 *pp = pair + o.y;
      uint2 q0 = SREC ? pp[0] : __ldg(pp), q1 = SREC ? pp[1] : __ldg(pp + 1);
      R s0 = (R)0, s1 = (R)0;
      int e = 0;
      for (; e + 2 <= o.z; e += 2) {
        const uint2 u0 = q0, u1 = q1;
        q0 = SREC ? pp[2] : __ldg(pp + 2);
        q1 = SREC ? pp[3] : __ldg(pp + 3);
        pp += 2;
        s0 += srow<R>(sm, lc + u0.x) * srow<R>(sm, lc + u0.y);
        s1 += srow<R>(sm, lc + u1.x) * srow<R>(sm, lc + u1.y);
      }
      if (e < o.z) s0 += srow<R>(sm, lc + q0.x) * srow<R>(sm, lc + q0.y);
      const R s = (s0 + s1) * __ldg(sc + 2 * na + o.x);
      if (act) Sb[(size_t)o.x * n + j] = s;
      if (o.x == 0) gb += (double)s;
    }
    __syncthreads();
    buf ^= 1;
  }
  cp_async_wait<0>();
  if (a.gbias && gj >= 0 && gj < n && lact && gb != 0.0)
    atomicAdd(a.gbias + (size_t)gj * a.gstride, gb);
}

// ---------------------------------------------------------------- v7
struct Adj7Args {
  int n, na, npts, gstride, gy;
  int nunit, nout, nglist, nrec, nfin, nscratch;
  const int *list;
  const int4 *unit;     // [nunit][2]
  const int *out;
  const uint32_t *glist, *rec;
  const int *fin;       // [nfin][2]
  const void *sc;       // [3][na]
  const void *Tb, *h;
  void *Sb;
  double *gbias;
};

// shared-memory layout of the v7 adjoint: two buffers of [Tb | h] rows, the
// scratch rows, then the tables (16-byte aligned pieces)
struct Adj7Layout {
  uint32_t scr, unit, out, gl, rec, fin, total;
  __host__ __device__ static uint32_t al16(uint32_t v) { return (v + 15u) & ~15u; }
  __host__ __device__ Adj7Layout(int na, int nscratch, int nunit, int nout, int nglist, int nrec,
                                 int nfin) {
    scr = 4u * na * 128u;
    unit = scr + (uint32_t)nscratch * 128u;
    out = unit + (uint32_t)nunit * 32u;
    gl = al16(out + (uint32_t)nout * 4u);
    rec = al16(gl + (uint32_t)nglist * 4u);
    fin = al16(rec + (uint32_t)nrec * 4u);
    total = al16(fin + (uint32_t)nfin * 8u);
  }
};

// 32-bit shared-window loads (the operands live in dynamic shared memory;
// volatile keeps them between the block's barriers)
__device__ __forceinline__ uint32_t ld_s32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ uint2 ld_s64(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ uint4 ld_s128(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(a));
  return v;
}
template <typename R>
__device__ __forceinline__ R ld_sr(uint32_t a);
template <>
__device__ __forceinline__ float ld_sr<float>(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
template <>
__device__ __forceinline__ double ld_sr<double>(uint32_t a) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

// one unit: acc[k] += (a! Tb)_{b_k + g} (h/g!)_g over its g range, then
// its nk outputs: scaled by 1/b! and stored (or added to the output's
// scratch row when its g list is split).  lcs is this lane's shared address
// in the current buffer; rec, gl shared addresses of the unit's tables.
template <typename R, int NK>
__device__ __forceinline__ void adj7_unit(uint32_t lcs, uint32_t rec, uint32_t gl, int ng,
                                          bool partial, const int *outs, unsigned char *scr,
                                          const R *scb, R *Sb, int n, int j, int ln, bool lact,
                                          bool act, double &gb) {
  constexpr int ST = NK <= 2 ? NK : (NK + 3) / 4 * 4;
  R acc[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) acc[k] = (R)0;
#pragma unroll 2
  for (int g = 0; g < ng; ++g) {
    const R hv = ld_sr<R>(lcs + ld_s32(gl + 4 * g));
    const uint32_t r = rec + 4 * ST * g;
    uint32_t o[ST];
    if constexpr (ST % 4 == 0) {
#pragma unroll
      for (int q = 0; q < ST / 4; ++q) {
        const uint4 v = ld_s128(r + 16 * q);
        o[4 * q] = v.x;
        o[4 * q + 1] = v.y;
        o[4 * q + 2] = v.z;
        o[4 * q + 3] = v.w;
      }
    } else if constexpr (ST == 2) {
      const uint2 v = ld_s64(r);
      o[0] = v.x;
      o[1] = v.y;
    } else {
      o[0] = ld_s32(r);
    }
#pragma unroll
    for (int k = 0; k < NK; ++k) acc[k] += ld_sr<R>(lcs + o[k]) * hv;
  }
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const int ob = outs[k];
    const int b = ob & 0xffff;
    if (partial) {
      if (lact) atomicAdd((R *)(scr + (ob >> 16) * 128) + ln, acc[k]);
    } else {
      const R v = acc[k] * __ldg(scb + b);
      if (act) Sb[(size_t)b * n + j] = v;
      if (b == 0) gb += (double)v;
    }
  }
}

// Bell adjoint v7, grouped correlation (bell_plan.hpp): units of up to 16
// outputs sharing each h_g load; split outputs summed in scratch rows.
template <typename R, int NPB>
__global__ void __launch_bounds__(ADJ_WORKERS * 32) k_bell_adj7(Adj7Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const int n = a.n, na = a.na;
  const size_t plane = (size_t)na * n;
  const uint32_t bufb = 2 * na * 128;
  const Adj7Layout L(na, a.nscratch, a.nunit, a.nout, a.nglist, a.nrec, a.nfin);
  int4 *su = (int4 *)(sm + L.unit);
  int *so = (int *)(sm + L.out);
  uint32_t *sg = (uint32_t *)(sm + L.gl);
  uint32_t *sr = (uint32_t *)(sm + L.rec);
  int *sf = (int *)(sm + L.fin);
  for (int i = threadIdx.x; i < 2 * a.nunit; i += blockDim.x) su[i] = __ldg(a.unit + i);
  for (int i = threadIdx.x; i < a.nout; i += blockDim.x) so[i] = __ldg(a.out + i);
  for (int i = threadIdx.x; i < a.nglist; i += blockDim.x) sg[i] = __ldg(a.glist + i);
  for (int i = threadIdx.x; i < a.nrec; i += blockDim.x) sr[i] = __ldg(a.rec + i);
  for (int i = threadIdx.x; i < 2 * a.nfin; i += blockDim.x) sf[i] = __ldg(a.fin + i);
  for (int i = threadIdx.x; i < a.nscratch * 32; i += blockDim.x) ((uint32_t *)(sm + L.scr))[i] = 0u;
  const R *sc = (const R *)a.sc;
  const int rs = __ldg(a.list + warp * 2), rn = __ldg(a.list + warp * 2 + 1);
  double gb = 0.0;
  int gj = -1;
  int buf = 0;
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  if (it0 < it1) {
    const size_t o = (it0 % a.npts) * plane;
    const int j0 = (int)(it0 / a.npts) * NPB;
    stage_rows<NPB, R>(sm, (const R *)a.Tb + o, na, n, j0, ADJ_WORKERS * 32);
    stage_rows<NPB, R>(sm + na * 128, (const R *)a.h + o, na, n, j0, ADJ_WORKERS * 32);
  }
  cp_async_commit();
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * NPB + ln;
    const bool act = lact && j < n;
    if (j != gj) {
      if (a.gbias && gj >= 0 && gj < n && lact && gb != 0.0)
        atomicAdd(a.gbias + (size_t)gj * a.gstride, gb);
      gb = 0.0;
      gj = j;
    }
    if (it + 1 < it1) {
      unsigned char *oth = sm + (buf ^ 1) * bufb;
      const size_t o = ((it + 1) % a.npts) * plane;
      const int j0 = (int)((it + 1) / a.npts) * NPB;
      stage_rows<NPB, R>(oth, (const R *)a.Tb + o, na, n, j0, ADJ_WORKERS * 32);
      stage_rows<NPB, R>(oth + na * 128, (const R *)a.h + o, na, n, j0, ADJ_WORKERS * 32);
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const uint32_t lc = buf * bufb + ln * sizeof(R);
    for (int r = warp; r < 2 * na; r += ADJ_WORKERS)
      if (lact) srow<R>(sm, lc + r * 128) *= __ldg(sc + r);
    __syncthreads();
    R *Sb = (R *)a.Sb + pt * plane;
    for (int u = rs; u < rs + rn; ++u) {
      const int4 U0 = su[2 * u], U1 = su[2 * u + 1];
      const int nk = U0.z & 0xff;
      const bool partial = (U0.z >> 8) != 0;
      const uint32_t rec = smem_u32(sr + U0.x);
      const uint32_t gl = smem_u32(sg + U1.x);
      const uint32_t lcs = smem_u32(sm) + lc;
      switch (nk) {
#define A7CASE(N)                                                                        \
  case N:                                                                                \
    adj7_unit<R, N>(lcs, rec, gl, U0.y, partial, so + U0.w, sm + L.scr, sc + 2 * na, Sb, n, \
                    j, ln, lact, act, gb);                                                \
    break;
        A7CASE(1) A7CASE(2) A7CASE(3) A7CASE(4) A7CASE(5) A7CASE(6) A7CASE(7) A7CASE(8)
#undef A7CASE
        default:
          if constexpr (sizeof(R) == 4) {  // the FP32 plan holds up to 16 outputs
            switch (nk) {
#define A7CASE(N)                                                                        \
  case N:                                                                                \
    adj7_unit<R, N>(lcs, rec, gl, U0.y, partial, so + U0.w, sm + L.scr, sc + 2 * na, Sb, n, \
                    j, ln, lact, act, gb);                                                \
    break;
              A7CASE(9) A7CASE(10) A7CASE(11) A7CASE(12) A7CASE(13) A7CASE(14) A7CASE(15)
              A7CASE(16)
#undef A7CASE
              default: break;
            }
          }
          break;
      }
    }
    __syncthreads();
    // outputs whose g lists were split: scale, store, and clear the row
    for (int i = warp; i < a.nfin; i += ADJ_WORKERS) {
      const int b = sf[2 * i], row = sf[2 * i + 1];
      R *cell = (R *)(sm + L.scr + row * 128) + ln;
      const R v = *cell * __ldg(sc + 2 * na + b);
      __syncwarp();
      if (lact) *cell = (R)0;
      if (act) Sb[(size_t)b * n + j] = v;
      if (b == 0) gb += (double)v;
    }
    // no barrier here: the next item's copy goes to the buffer that every
    // warp left at the barrier after the units, and the scratch rows are
    // added to only after the next item's first barrier
    buf ^= 1;
  }
  cp_async_wait<0>();
  if (a.gbias && gj >= 0 && gj < n && lact && gb != 0.0)
    atomicAdd(a.gbias + (size_t)gj * a.gstride, gb);
}

static int sm_count_b() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// blocks of a persistent launch: as many as are resident at once on the
// device (occupancy of this kernel at this shared-memory size), at most one
// per work item, so no block waits for a second wave
static int persistent_grid(const void *k, int threads, size_t smem, long items) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long g = (long)grid_sms() * per_sm;
  return (int)std::max(1L, std::min(g, items));
}

// ------------------------------------------------------------- autotuner
// The v5 kernels come in variants that compute bit-identical outputs (table
// records read from global memory, or copied once into the shared memory
// left beside the state).  Which is faster depends on the precision and on
// the table sizes, so the first launch for a (plan, kernel, width,
// precision) with at least a few waves of work runs every variant once on
// the caller's stream, timed with CUDA events, and keeps the fastest for the
// later launches.  While the stream is being captured into a graph no
// timing is possible and the default variant runs.  launch(v, last) runs
// variant v; side effects that accumulate (the adjoint's bias gradient)
// happen only when last is set, which it is for exactly one launch.
struct TuneKey {
  uint64_t plan;
  int which, n, prec;
  int d0 = 0, k = 0, na = 0;  // the plan's table set, for the report only
  bool operator<(const TuneKey &o) const {
    return std::tie(plan, which, n, prec) < std::tie(o.plan, o.which, o.n, o.prec);
  }
};
static std::map<TuneKey, int> g_tune;
static std::map<TuneKey, std::vector<float>> g_tune_ms;  // timed trial per variant
static std::map<TuneKey, std::vector<int>> g_tune_id;   // variant ids of the trials
static std::mutex g_tune_mu;

// "kernel d0 k na width prec chosen ms0 ms1 ..." lines, one per tuned
// launch shape (the chosen variant's id, then the trial time of each)
std::string tune_report() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  static const char *names[] = {"bell_fwd", "bell_fwd_train", "bell_adj"};
  std::string out;
  char b[64];
  for (auto &kv : g_tune) {
    auto ids = g_tune_id.find(kv.first);
    const int chosen = ids != g_tune_id.end() && kv.second < (int)ids->second.size()
                           ? ids->second[kv.second]
                           : kv.second;
    std::snprintf(b, sizeof b, "%s %d %d %d %d %s %d", names[kv.first.which], kv.first.d0,
                  kv.first.k, kv.first.na, kv.first.n, kv.first.prec == 8 ? "f64" : "f32",
                  chosen);
    out += b;
    auto it = g_tune_ms.find(kv.first);
    if (it != g_tune_ms.end())
      for (float ms : it->second) {
        std::snprintf(b, sizeof b, " %.4f", ms);
        out += b;
      }
    out += "\n";
  }
  return out;
}

// variants pinned by the caller: [0] forward, [1] adjoint; -1 = autotune
static std::atomic<int> g_force[2] = {{-1}, {-1}};

int tune_force(int which, int variant) {
  if (which == 2) {  // the tanh series forward on (1) or off (0, -1: the default)
    if (variant < -1 || variant > 1) return RC_BAD_ARG;
    g_series_fwd = variant == 1;
    return RC_OK;
  }
  if (which < 0 || which > 1 || variant < -1 || variant > 7) return RC_BAD_ARG;
  g_force[which] = variant;
  return RC_OK;
}

template <typename L>
static int tuned_launch(const TuneKey &key, int nvar, int dflt, long items, cudaStream_t st,
                        L launch) {
  {
    const int f = g_force[key.which == 2 ? 1 : 0];
    if (f >= 0) return launch(f < nvar ? f : dflt, true);
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return launch(it->second, true);
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (nvar < 2 || cudaStreamIsCapturing(st, &cs) != cudaSuccess ||
      cs != cudaStreamCaptureStatusNone || items < (long)sm_count_b() * 8)
    return launch(dflt, true);
  cudaEvent_t e0, e1;
  CKB(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    set_error("autotuner: cudaEventCreate failed");
    return RC_DEVICE;
  }
  float best = 0.f;
  int bv = dflt, rc = RC_OK;
  std::vector<float> times(nvar, -1.f);
  // one untimed run of each first, so that module loading and first-touch
  // costs do not favour the variant that runs later
  for (int v = 0; v < nvar && rc == RC_OK; ++v) rc = launch(v, false);
  for (int v = 0; v < nvar && rc == RC_OK; ++v) {
    cudaEventRecord(e0, st);
    rc = launch(v, v == nvar - 1);
    cudaEventRecord(e1, st);
    if (rc == RC_OK && cudaEventSynchronize(e1) == cudaSuccess) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      times[v] = ms;
      if (v == 0 || ms < best) {
        best = ms;
        bv = v;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = bv;
  g_tune_ms[key] = times;
  return RC_OK;  // every variant wrote the same values
}

// tuned_launch over a list of variant ids (launch(id, last)); a pinned
// variant runs if it applies, else the default; the record keeps the ids
template <typename L>
static int tuned_ids(const TuneKey &key, const std::vector<int> &ids, int dflt, long items,
                     cudaStream_t st, L launch) {
  const int f = g_force[key.which == 2 ? 1 : 0];
  if (f >= 0) {
    for (int id : ids)
      if (id == f) return launch(f, true);
    return launch(ids[dflt], true);
  }
  const int rc = tuned_launch(key, (int)ids.size(), dflt, items, st,
                              [&](int i, bool last) { return launch(ids[i], last); });
  if (rc == RC_OK) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end() && it->second < (int)ids.size() && g_tune_id.count(key) == 0) {
      g_tune_id[key] = ids;
    }
  }
  return rc;
}

template <typename R, int KK>
static int fwd5_dispatch(const DevBellPlan &bp, const DevTables &t, int n, int npts,
                         const void *S, void *T, void *h, bool train, cudaStream_t st) {
  constexpr int NPB = sizeof(R) == 8 ? 16 : 32;
  static_assert(NPB * sizeof(R) == 128, "one state row is 128 bytes");
  size_t smem = ((size_t)bp.nrows5 + t.na) * 128;
  if (!bp.f5_ok || smem > 227 * 1024 || n % (16 / (int)sizeof(R))) return RC_UNSUPPORTED;
  Fwd5Args a;
  a.n = n; a.na = t.na; a.npts = npts; a.iact = t.iact; a.dt_off = bp.dt_off5;
  a.nrows = bp.nrows5; a.gy = (n + NPB - 1) / NPB; a.zuv = bp.zuv5;
  a.nrec32 = bp.nrec32;
  a.tpc = t.tpc; a.list = bp.f5_list; a.arec = (const int4 *)bp.f5_arec;
  a.rec = (const uint2 *)bp.f5_rec; a.rec32 = bp.f6_rec; a.cpdst = bp.f5_cpdst;
  a.sc = sizeof(R) == 8 ? (const void *)bp.sc64 : (const void *)bp.sc32;
  a.S = S; a.T = T; a.h = h;
  if (t.iact == 0 && bp.f9.ok && g_series_fwd) {
    Fwd9Args c;
    c.n = n; c.na = t.na; c.npts = npts; c.iact = t.iact; c.gy = a.gy;
    c.pbase = bp.f9.pbase; c.qbase = bp.f9.qbase; c.tpc = t.tpc;
    c.list = bp.f9.list; c.hdr = (const int4 *)bp.f9.hdr; c.rec = (const uint4 *)bp.f9.rec;
    c.sc = a.sc;
    c.sdeg = sizeof(R) == 8 ? (const void *)bp.f9.sdeg64 : (const void *)bp.f9.sdeg32;
    c.S = S; c.T = T; c.h = h;
    auto k = train ? k_tanh_fwd9<R, KK, NPB, true> : k_tanh_fwd9<R, KK, NPB, false>;
    CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bp.f9.smem));
    const int grid = persistent_grid((const void *)k, BELL_WORKERS * 32, bp.f9.smem, (long)npts * a.gy);
    LAUNCH("k_bell_fwd", st, k<<<grid, BELL_WORKERS * 32, bp.f9.smem, st>>>(c));
    CKB(cudaGetLastError());
    return RC_OK;
  }
  // variant 0: records in global memory; 1: records in shared memory;
  // 2: v8 (lean per-degree loops over 16-bit offset records); 3: the
  // register-tiled Horner forward (bell_tile.cu; FP32, dense sets), the
  // default wherever it applies
  const bool srec_fits = smem + (size_t)bp.nrec32 * 4 <= 227 * 1024;
  const bool v8_ok = bp.f8.ok && bp.f8.smem <= 227 * 1024;
  const bool tile_ok = sizeof(R) == 4 && tile_fwd_applies(bp.tile, n);
  auto launch = [&](int v, bool) -> int {
    if (v == 3) return bell_fwd_tile(bp.tile, t, n, npts, S, T, h, train, st);
    if (v == 2) {
      Fwd8Args b;
      b.n = n; b.na = t.na; b.npts = npts; b.iact = t.iact; b.gy = a.gy; b.nrec = bp.f8.nrec;
      b.sbase1 = bp.f8.sbase1; b.bbase = bp.f8.bbase; b.uvbase = bp.f8.uvbase;
      b.dtbase = bp.f8.dtbase; b.recbase = bp.f8.recbase; b.zuv = bp.f8.zuv;
      b.tpc = t.tpc; b.list = bp.f8.list; b.hdr = (const int4 *)bp.f8.hdr; b.rec = bp.f8.rec;
      b.cpdst = bp.f8.cpdst; b.sc = a.sc; b.S = S; b.T = T; b.h = h;
      auto k = train ? k_bell_fwd8<R, KK, NPB, true> : k_bell_fwd8<R, KK, NPB, false>;
      CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bp.f8.smem));
      const int grid = persistent_grid((const void *)k, BELL_WORKERS * 32, bp.f8.smem, (long)npts * a.gy);
      LAUNCH("k_bell_fwd", st, k<<<grid, BELL_WORKERS * 32, bp.f8.smem, st>>>(b));
      CKB(cudaGetLastError());
      return RC_OK;
    }
    const bool srec = v == 1;
    const size_t sm = smem + (srec ? (size_t)bp.nrec32 * 4 : 0);
    auto k = srec ? (train ? k_bell_fwd5<R, KK, NPB, true, true> : k_bell_fwd5<R, KK, NPB, false, true>)
                  : (train ? k_bell_fwd5<R, KK, NPB, true, false> : k_bell_fwd5<R, KK, NPB, false, false>);
    CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int grid = persistent_grid((const void *)k, BELL_WORKERS * 32, sm, (long)npts * a.gy);
    LAUNCH("k_bell_fwd", st, k<<<grid, BELL_WORKERS * 32, sm, st>>>(a));
    CKB(cudaGetLastError());
    return RC_OK;
  };
  // every variant that applies is timed; the default (the choice under
  // graph capture, and for launches too small to time) is the tiled
  // kernel, else v8, else v5
  std::vector<int> ids{0};
  if (srec_fits) ids.push_back(1);
  if (v8_ok) ids.push_back(2);
  if (tile_ok) ids.push_back(3);
  return tuned_ids(TuneKey{bp.id, train ? 1 : 0, n, (int)sizeof(R), t.d0, t.k, t.na}, ids,
                   (int)ids.size() - 1,
                   (long)npts * a.gy, st, launch);
}

template <typename R, int KK>
static int fwd2_dispatch(const DevBellPlan &bp, const DevTables &t, int n, int npts,
                         const void *S, void *T, void *h, bool train, cudaStream_t st) {
  {
    int rc3 = fwd5_dispatch<R, KK>(bp, t, n, npts, S, T, h, train, st);
    if (rc3 != RC_UNSUPPORTED) return rc3;
  }
  constexpr int NPB = sizeof(R) == 8 ? 16 : 32;
  const size_t smem = ((size_t)t.na + bp.nslot + KK + 2) * NPB * sizeof(R);
  if (smem > 227 * 1024) return RC_UNSUPPORTED;
  Fwd2Args a;
  a.n = n; a.na = t.na; a.nslot = bp.nslot; a.npts = npts; a.iact = t.iact;
  a.workers = bp.workers; a.tpc = t.tpc; a.list = bp.fw_list;
  a.arec = (const int4 *)bp.fw_arec; a.grec = (const int4 *)bp.fw_grec;
  a.gc = sizeof(R) == 8 ? (const void *)bp.fw_gc64 : (const void *)bp.fw_gc32;
  a.S = S; a.T = T; a.h = h;
  const int gy = (n + NPB - 1) / NPB;
  const int per_sm = std::max(1, (int)((228 * 1024) / (smem + 1024)));
  const int gx = std::max(1, std::min(npts, grid_sms() * per_sm / gy));
  dim3 grid(gx, gy);
  if (train) {
    auto k = k_bell_fwd2<R, KK, NPB, true>;
    CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH("k_bell_fwd", st, k<<<grid, BELL_WORKERS * 32, smem, st>>>(a));
  } else {
    auto k = k_bell_fwd2<R, KK, NPB, false>;
    CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH("k_bell_fwd", st, k<<<grid, BELL_WORKERS * 32, smem, st>>>(a));
  }
  CKB(cudaGetLastError());
  return RC_OK;
}

template <typename R>
static int fwd2_k(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *S,
                  void *T, void *h, bool train, cudaStream_t st) {
  switch (t.k) {
    case 1: return fwd2_dispatch<R, 1>(bp, t, n, npts, S, T, h, train, st);
    case 2: return fwd2_dispatch<R, 2>(bp, t, n, npts, S, T, h, train, st);
    case 3: return fwd2_dispatch<R, 3>(bp, t, n, npts, S, T, h, train, st);
    case 4: return fwd2_dispatch<R, 4>(bp, t, n, npts, S, T, h, train, st);
    case 5: return fwd2_dispatch<R, 5>(bp, t, n, npts, S, T, h, train, st);
    case 6: return fwd2_dispatch<R, 6>(bp, t, n, npts, S, T, h, train, st);
    case 7: return fwd2_dispatch<R, 7>(bp, t, n, npts, S, T, h, train, st);
    case 8: return fwd2_dispatch<R, 8>(bp, t, n, npts, S, T, h, train, st);
    default: return RC_UNSUPPORTED;
  }
}

int bell_fwd2(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *S,
              void *T, void *h, bool train, int prec, cudaStream_t st) {
  if (!bp.ready) return RC_UNSUPPORTED;
  return prec == PREC_F64 ? fwd2_k<double>(bp, t, n, npts, S, T, h, train, st)
                          : fwd2_k<float>(bp, t, n, npts, S, T, h, train, st);
}

template <typename R>
static int adj2_t(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *Tb,
                  const void *h, void *Sb, double *gbias, int gstride, cudaStream_t st) {
  constexpr int NPB = sizeof(R) == 8 ? 16 : 32;
  const size_t smem = (size_t)2 * t.na * NPB * sizeof(R);
  if (smem > 227 * 1024) return RC_UNSUPPORTED;
  if (bp.a5_pair && (size_t)4 * t.na * 128 <= 227 * 1024 && n % (16 / (int)sizeof(R)) == 0) {
    size_t smem5 = (size_t)4 * t.na * 128;
    Adj5Args b;
    b.n = n; b.na = t.na; b.npts = npts; b.gstride = gstride; b.list = bp.aj_list;
    b.orec = (const int4 *)bp.a3_orec; b.pair = (const uint2 *)bp.a5_pair;
    b.norec = bp.norec; b.npair = bp.npair5;
    b.sc = sizeof(R) == 8 ? (const void *)bp.sc64 : (const void *)bp.sc32;
    b.Tb = Tb; b.h = h; b.Sb = Sb; b.gbias = gbias;
    b.gy = (n + NPB - 1) / NPB;
    const size_t extra = (size_t)bp.norec * 16 + (size_t)bp.npair5 * 8;
    const bool srec_fits = smem5 + extra <= 227 * 1024;
    // variant 0: pairs in global memory; 1: pairs in shared memory
    auto launch = [&](int v, bool last) -> int {
      Adj5Args bv = b;
      if (!last) bv.gbias = nullptr;  // a timing run adds nothing
      const bool srec = v == 1;
      const size_t sm = smem5 + (srec ? extra : 0);
      auto k = srec ? k_bell_adj5<R, NPB, true> : k_bell_adj5<R, NPB, false>;
      CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      const int grid = persistent_grid((const void *)k, ADJ_WORKERS * 32, sm, (long)npts * b.gy);
      LAUNCH("k_bell_adj", st, k<<<grid, ADJ_WORKERS * 32, sm, st>>>(bv));
      CKB(cudaGetLastError());
      return RC_OK;
    };
    const DevBellPlan::A7Dev &A7 = bp.a7[sizeof(R) == 8 ? 1 : 0];
    const Adj7Layout L7(t.na, A7.nscratch, A7.nunit, A7.nout, A7.nglist, A7.nrec, A7.nfin);
    const bool v7_fits = A7.ok && L7.total <= 227 * 1024;
    auto launch_all = [&](int v, bool last) -> int {
      if (v < 2) return launch(v, last);
      // variant 2: grouped correlation (v7)
      Adj7Args c;
      c.n = n; c.na = t.na; c.npts = npts; c.gstride = gstride; c.gy = b.gy;
      c.nunit = A7.nunit; c.nout = A7.nout; c.nglist = A7.nglist; c.nrec = A7.nrec;
      c.nfin = A7.nfin; c.nscratch = A7.nscratch;
      c.list = A7.list; c.unit = (const int4 *)A7.unit; c.out = A7.out;
      c.glist = A7.glist; c.rec = A7.rec; c.fin = A7.fin;
      c.sc = b.sc; c.Tb = Tb; c.h = h; c.Sb = Sb; c.gbias = last ? gbias : nullptr;
      auto k = k_bell_adj7<R, NPB>;
      CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L7.total));
      const int grid = persistent_grid((const void *)k, ADJ_WORKERS * 32, L7.total, (long)npts * b.gy);
      LAUNCH("k_bell_adj", st, k<<<grid, ADJ_WORKERS * 32, L7.total, st>>>(c));
      CKB(cudaGetLastError());
      return RC_OK;
    };
    // variant 3: the register-tiled correlation (bell_tile.cu; FP32, dense
    // sets).  Every variant that applies is timed; the default is the tiled
    // kernel where it applies, else v7, else the last that applies
    auto launch_t = [&](int v, bool last) -> int {
      if (v == 3)
        return bell_adj_tile(bp.tile, n, npts, Tb, h, Sb, last ? gbias : nullptr, gstride, st);
      return launch_all(v, last);
    };
    std::vector<int> ids{0};
    if (srec_fits) ids.push_back(1);
    if (v7_fits) ids.push_back(2);
    if (sizeof(R) == 4 && tile_adj_applies(bp.tile, n)) ids.push_back(3);
    int dflt = (int)ids.size() - 1;
    if (v7_fits && ids.back() != 3) dflt = srec_fits ? 2 : 1;
    return tuned_ids(TuneKey{bp.id, 2, n, (int)sizeof(R), t.d0, t.k, t.na}, ids, dflt,
                     (long)npts * b.gy, st,
                     launch_t);
  }
  Adj2Args a;
  a.n = n; a.na = t.na; a.npts = npts; a.gstride = gstride; a.list = bp.aj_list;
  a.orec = (const int4 *)bp.aj_orec; a.pair = bp.aj_pair;
  a.c = sizeof(R) == 8 ? (const void *)bp.aj_c64 : (const void *)bp.aj_c32;
  a.Tb = Tb; a.h = h; a.Sb = Sb; a.gbias = gbias;
  const int gy = (n + NPB - 1) / NPB;
  const int per_sm = std::max(1, (int)((228 * 1024) / (smem + 1024)));
  const int gx = std::max(1, std::min(npts, grid_sms() * per_sm / gy));
  dim3 grid(gx, gy);
  auto k = k_bell_adj2<R, NPB>;
  CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  LAUNCH("k_bell_adj", st, k<<<grid, ADJ_WORKERS * 32, smem, st>>>(a));
  CKB(cudaGetLastError());
  return RC_OK;
}

int bell_adj2(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *Tb,
              const void *h, void *Sb, double *gbias, int gstride, int prec,
              cudaStream_t st) {
  if (!bp.ready) return RC_UNSUPPORTED;
  return prec == PREC_F64 ? adj2_t<double>(bp, t, n, npts, Tb, h, Sb, gbias, gstride, st)
                          : adj2_t<float>(bp, t, n, npts, Tb, h, Sb, gbias, gstride, st);
}

// ------------------------------------------------- first-layer adjoint, staged
struct AdjL2sArgs {
  int n, na, npts, gy;
  const int *up;           // [na][D0]: slot of g + e_i | (g_i + 1) << 16, or -1
  const void *Tb, *h;      // [P][na][n] (h unused when h is formed in the kernel)
  const double *X;         // [P][D0]
  double *g;               // dW_2 [n][D0 + 1], accumulated (null in row mode)
  double *rows;            // [P][nw] (row mode)
  size_t nw, woff;
  // h formed in the kernel (graded slots): the layer's weights [n][D0 + 1],
  // s^(q)(S^0) [P][k + 2][n] kept by the forward, the order, the first slot
  // of each degree and a - e_i | i << 16 per slot (k_layer2v's monomials)
  const double *W;
  const void *sig;
  const int *par;
  int k;
  int ds[KMAX + 2];
};

// The first hidden layer's Bell adjoint fused with dW_2 (the k_adj_l2v sums)
//   Sb^0 = sum_g Tb^g h^g,  Sb^{e_i} = sum_g (g_i + 1) Tb^{g + e_i} h^g,
//   dW_2[j][0] += Sb^0,  dW_2[j][1 + i] += Sb^0 x_i + Sb^{e_i},
// one (point, NPB-neuron tile) at a time per block: the item's Tb and h rows
// are staged in shared memory (the next item's copy in flight meanwhile) and
// the 32 warps split the slots g.  dW_2 is linear in each slot's share, so
// every warp keeps its own FP64 partial of the tile's dW_2 rows and adds it
// in once per tile; only the per-point rows (Jacobian mode) are summed over
// the warps per item.  Every Tb row is read from HBM once instead of D0 + 1
// times through the caches.
// AN: the first layer is analytic (S^0 = W x + b, S^{e_i} = W_i), so
// h^g = s^(|g|+1)(S^0) W^g, formed here exactly as k_layer2v forms it (the
// monomial W^g = prod_i W_i^{g_i} in R, built once per neuron tile along
// unit steps; the s^(q) the forward kept, rounded to R, times it): no h
// plane is written by the forward nor read here, only k + 2 rows of s^(q)
// per item beside its Tb rows.  A warp's slots come in graded order, so it
// steps its multiplier at each degree boundary.  (Summing each degree with
// W^g and multiplying by s^(p+1) once was measured slower: the degree runs
// are short, 1 to 4 slots per warp.)
template <typename R, int D0, int NPB, bool AN>
__global__ void __launch_bounds__(1024) k_adj_l2s(AdjL2sArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  const int na = a.na, n = a.n;
  // one buffer: Tb rows, then h rows (AN: the k + 2 rows of s^(q))
  const uint32_t bsz = (AN ? (uint32_t)(na + KMAX + 2) : 2u * na) * 128;
  // AN: the tile's monomials [na] rows, the degree starts
  const uint32_t moff = 2 * bsz, dsoff = moff + (AN ? (uint32_t)na * 128 : 0u);
  const uint32_t upoff = dsoff + (AN ? 128u : 0u);
  const uint32_t redoff = upoff + ((uint32_t)na * D0 * 8 + 127) / 128 * 128;
  // (byte offset of the Tb row of g + e_i, multiplier g_i + 1) per (g, i);
  // a missing child reads row 0 with multiplier 0
  uint2 *up = (uint2 *)(sm + upoff);
  for (int e = threadIdx.x; e < na * D0; e += blockDim.x) {
    const int u = __ldg(a.up + e);
    up[e] = u >= 0 ? make_uint2((uint32_t)(u & 0xffff) * 128, __float_as_uint((float)(u >> 16)))
                   : make_uint2(0u, 0u);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool lact = lane < NPB;
  const int ln = lact ? lane : 0;
  const uint32_t lo = ln * sizeof(R);
  const size_t plane = (size_t)na * n;
  const long nitem = (long)a.npts * a.gy;
  const long it0 = (long)blockIdx.x * nitem / gridDim.x;
  const long it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
  auto stage = [&](long it, uint32_t dst) {
    const size_t pofs = (size_t)(it % a.npts) * plane;
    const int j0 = (int)(it / a.npts) * NPB;
    stage_rows<NPB, R>(sm + dst, (const R *)a.Tb + pofs, na, n, j0, 1024);
    if (AN)
      stage_rows<NPB, R>(sm + dst + na * 128,
                         (const R *)a.sig + (size_t)(it % a.npts) * (a.k + 2) * n, a.k + 2, n,
                         j0, 1024);
    else
      stage_rows<NPB, R>(sm + dst + na * 128, (const R *)a.h + pofs, na, n, j0, 1024);
  };
  if (it0 < it1) stage(it0, 0);
  cp_async_commit();
  // AN: the monomials W^g of tile tl's neurons (every thread; barriers inside)
  const int *sds = (const int *)(sm + dsoff);
  auto build_m = [&](int tl) {
    const int j = tl * NPB + ln;
    const double *wr = a.W + (size_t)(j < n ? j : n - 1) * (D0 + 1);
    if (warp == 0 && lact) srow<R>(sm, moff + lo) = (R)1;
    __syncthreads();
    for (int p = 1; p <= a.k; ++p) {
      for (int ia = sds[p] + warp; ia < sds[p + 1]; ia += 32) {
        const int pk = __ldg(a.par + ia);
        if (lact)
          srow<R>(sm, moff + ia * 128 + lo) =
              (R)((double)srow<R>(sm, moff + (pk & 0xffff) * 128 + lo) * wr[1 + (pk >> 16)]);
      }
      __syncthreads();
    }
  };
  int mtile = -1;
  if (AN && it0 < it1) {
    if (threadIdx.x < KMAX + 2) ((int *)(sm + dsoff))[threadIdx.x] = a.ds[threadIdx.x];
    __syncthreads();
    mtile = (int)(it0 / a.npts);
    build_m(mtile);
  }
  double acc[D0 + 1];
#pragma unroll
  for (int o = 0; o <= D0; ++o) acc[o] = 0.0;
  int tile = it0 < it1 ? (int)(it0 / a.npts) : 0;
  // this warp's partial of the tile's dW_2 rows
  auto flush = [&](int tl) {
    const int j = tl * NPB + ln;
    if (a.g && lact && j < n) {
      double *gr = a.g + (size_t)j * (D0 + 1);
#pragma unroll
      for (int o = 0; o <= D0; ++o)
        if (acc[o] != 0.0) atomicAdd(gr + o, acc[o]);
    }
#pragma unroll
    for (int o = 0; o <= D0; ++o) acc[o] = 0.0;
  };
  for (long it = it0; it < it1; ++it) {
    const uint32_t buf = (uint32_t)((it - it0) & 1) * bsz;
    cp_async_wait<0>();
    __syncthreads();  // this item's rows are in; every warp is done with the last item
    if (it + 1 < it1) stage(it + 1, buf ? 0 : bsz);
    cp_async_commit();
    const int pt = (int)(it % a.npts), tl = (int)(it / a.npts);
    if (tl != tile) {
      flush(tile);
      tile = tl;
    }
    if (AN && tl != mtile) {  // block-uniform: every warp is past the last item
      build_m(tl);
      mtile = tl;
    }
    const uint32_t tb = buf + lo, hb = tb + na * 128;
    R s[D0 + 1];
#pragma unroll
    for (int o = 0; o <= D0; ++o) s[o] = (R)0;
    if (AN) {
      // h^g = (R)s^(p+1) * W^g, p = |g|: the slots of a warp rise in degree,
      // so its multiplier steps at each degree boundary
      int p = 0, pend = sds[1];
      R dq = srow<R>(sm, hb + 128);  // this item's s^(1) row
      for (int g = warp; g < na; g += 32) {
        while (g >= pend) {
          ++p;
          pend = sds[p + 1];
          dq = srow<R>(sm, hb + (p + 1) * 128);
        }
        const R hg = dq * srow<R>(sm, moff + g * 128 + lo);
        s[0] += srow<R>(sm, tb + g * 128) * hg;
#pragma unroll
        for (int i = 0; i < D0; ++i) {
          const uint2 u = up[g * D0 + i];
          s[1 + i] += (R)__uint_as_float(u.y) * srow<R>(sm, tb + u.x) * hg;
        }
      }
    } else {
      for (int g = warp; g < na; g += 32) {
        const R hg = srow<R>(sm, hb + g * 128);
        s[0] += srow<R>(sm, tb + g * 128) * hg;
#pragma unroll
        for (int i = 0; i < D0; ++i) {
          const uint2 u = up[g * D0 + i];
          s[1 + i] += (R)__uint_as_float(u.y) * srow<R>(sm, tb + u.x) * hg;
        }
      }
    }
    const double *x = a.X + (size_t)pt * D0;
    if (!a.rows) {
      acc[0] += (double)s[0];
#pragma unroll
      for (int i = 0; i < D0; ++i) acc[1 + i] += (double)s[0] * __ldg(x + i) + (double)s[1 + i];
      continue;
    }
    // Jacobian rows: the point's sums over the warps, in a fixed order
    if (lact)
#pragma unroll
      for (int o = 0; o <= D0; ++o) srow<R>(sm, redoff + (warp * (D0 + 1) + o) * 128 + lo) = s[o];
    __syncthreads();
    const int j = tl * NPB + ln;
    if (warp == 0 && lact && j < n) {
      R v[D0 + 1];
#pragma unroll
      for (int o = 0; o <= D0; ++o) {
        v[o] = (R)0;
        for (int w = 0; w < 32; ++w) v[o] += srow<R>(sm, redoff + (w * (D0 + 1) + o) * 128 + lo);
      }
      double *row = a.rows + (size_t)pt * a.nw + a.woff + (size_t)j * (D0 + 1);
      row[0] = (double)v[0];
#pragma unroll
      for (int i = 0; i < D0; ++i) row[1 + i] = (double)v[0] * x[i] + (double)v[1 + i];
    }
  }
  cp_async_wait<0>();
  if (it0 < it1) flush(tile);
}

// shared memory of k_adj_l2s: two item buffers (Tb rows, then h rows, or
// with h formed in the kernel the item's s^(q) rows), then (an) the
// monomials and the degree starts, the (g, i) table and the per-warp row sums
static size_t l2s_smem(int na, int d0, bool an) {
  return (an ? (size_t)2 * (na + KMAX + 2) * 128 + (size_t)na * 128 + 128
             : (size_t)4 * na * 128) +
         ((size_t)na * d0 * 8 + 127) / 128 * 128 + (size_t)32 * (d0 + 1) * 128;
}

bool bell_adj_l2s_analytic(int d0, int na, int n, int prec) {
  const int rsz = prec == PREC_F64 ? 8 : 4;
  return d0 >= 1 && d0 <= 8 && na <= 65535 && n % (16 / rsz) == 0 &&
         l2s_smem(na, d0, true) <= 227 * 1024;
}

template <typename R, int D0>
static int adj_l2s_k(const AdjL2sArgs &a, cudaStream_t st) {
  constexpr int NPB = sizeof(R) == 8 ? 16 : 32;
  const bool an = a.W != nullptr;
  const size_t smem = l2s_smem(a.na, D0, an);
  if (smem > 227 * 1024 || a.na > 65535 || a.n % (16 / (int)sizeof(R))) return RC_UNSUPPORTED;
  AdjL2sArgs b = a;
  b.gy = (a.n + NPB - 1) / NPB;
  auto k = an ? k_adj_l2s<R, D0, NPB, true> : k_adj_l2s<R, D0, NPB, false>;
  CKB(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = persistent_grid((const void *)k, 1024, smem, (long)a.npts * b.gy);
  LAUNCH("k_bell_adj_l2", st, k<<<grid, 1024, smem, st>>>(b));
  CKB(cudaGetLastError());
  return RC_OK;
}

template <typename R>
static int adj_l2s_t(int d0, const AdjL2sArgs &a, cudaStream_t st) {
  switch (d0) {
    case 1: return adj_l2s_k<R, 1>(a, st);
    case 2: return adj_l2s_k<R, 2>(a, st);
    case 3: return adj_l2s_k<R, 3>(a, st);
    case 4: return adj_l2s_k<R, 4>(a, st);
    case 5: return adj_l2s_k<R, 5>(a, st);
    case 6: return adj_l2s_k<R, 6>(a, st);
    case 7: return adj_l2s_k<R, 7>(a, st);
    case 8: return adj_l2s_k<R, 8>(a, st);
    default: return RC_UNSUPPORTED;
  }
}

int bell_adj_l2s(int d0, int n, int na, int npts, const int *up, const void *Tb, const void *h,
                 const double *X, double *g, double *rows, size_t nw, size_t woff, int prec,
                 cudaStream_t st, const L2Analytic *an) {
  if (npts <= 0) return RC_OK;
  AdjL2sArgs a;
  a.n = n; a.na = na; a.npts = npts; a.gy = 0; a.up = up; a.Tb = Tb; a.h = h; a.X = X;
  a.g = g; a.rows = rows; a.nw = nw; a.woff = woff;
  a.W = nullptr; a.sig = nullptr; a.par = nullptr; a.k = 0;
  for (int p = 0; p < KMAX + 2; ++p) a.ds[p] = na;
  if (an) {
    if (an->k < 1 || an->k > KMAX) return RC_UNSUPPORTED;
    a.W = an->W; a.sig = an->sig; a.par = an->par; a.k = an->k;
    for (int p = 0; p <= an->k + 1; ++p) a.ds[p] = an->dstart[p];
  }
  return prec == PREC_F64 ? adj_l2s_t<double>(d0, a, st) : adj_l2s_t<float>(d0, a, st);
}

}  // namespace dnnf90
