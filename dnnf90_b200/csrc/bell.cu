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
#include <string>

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

void DevBellPlan::release() {
  void *ps[] = {fw_list, fw_arec, fw_grec, fw_gc64, fw_gc32, aj_list, aj_orec, aj_pair,
                aj_c64, aj_c32};
  for (void *p : ps)
    if (p) cudaFree(p);
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
  d.release();
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
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

template <typename R, int KK>
static int fwd2_dispatch(const DevBellPlan &bp, const DevTables &t, int n, int npts,
                         const void *S, void *T, void *h, bool train, cudaStream_t st) {
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
  const int gx = std::max(1, std::min(npts, sm_count_b() * per_sm / gy + 1));
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
  Adj2Args a;
  a.n = n; a.na = t.na; a.npts = npts; a.gstride = gstride; a.list = bp.aj_list;
  a.orec = (const int4 *)bp.aj_orec; a.pair = bp.aj_pair;
  a.c = sizeof(R) == 8 ? (const void *)bp.aj_c64 : (const void *)bp.aj_c32;
  a.Tb = Tb; a.h = h; a.Sb = Sb; a.gbias = gbias;
  const int gy = (n + NPB - 1) / NPB;
  const int per_sm = std::max(1, (int)((228 * 1024) / (smem + 1024)));
  const int gx = std::max(1, std::min(npts, sm_count_b() * per_sm / gy + 1));
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

}  // namespace dnnf90
