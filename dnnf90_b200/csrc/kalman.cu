// kalman.cu - the extended Kalman filter of lib/kalman_module.f90 on the
// device: the rank-one update of kf_update_grad (:353-490) over a sequence
// of observation rows, for the dense (global) and the node-wise decoupled
// covariance.
//
// Covariance store.  P is symmetric block diagonal (one block of nw for the
// dense filter, one block per neuron over (bias, fan-in) for the decoupled
// one, kf_block_map :172-189).  Each block keeps only its upper triangle,
// as 32 x 32 FP64 tiles (I <= J, row-major inside the tile, zero padding
// past the block edge); the diagonal tiles are kept whole.  The downdate
// and the symmetrisation of the reference,
//     P <- (P - kv pj^T) / lambda,  P_ij <- (P_ij + P_ji) / 2,  P_ii += q,
// give, for an element whose old value a is the same on both sides,
//     P_ij <- ((a - kv_i pj_j)/lambda + (a - kv_j pj_i)/lambda) / 2,
// an expression symmetric in (i, j), so each stored element is updated from
// its own value alone and the triangle never needs the transposed entry.
//
// One observation is two launches.  The tile pass applies observation k
// (downdate, process noise, and w += kv xi on the diagonal tiles) and, in
// the same read of each tile, forms the products of the NEW covariance with
// the next row: row sums of tile (I, J) land in partial slot J of the rows
// of I, column sums in slot I of the rows of J, so that every (slot, row)
// is written once and no atomics are needed.  The reduce pass sums the
// slots into P j for that row, forms j.Pj block by block, and its last CTA
// (found with a counter, no waiting) turns the block sums into the global
// denominator, applies the innovation gate and advances lambda.  A call
// therefore reads and writes the covariance once per observation, plus one
// read-only pass for the first row.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "engine.hpp"

namespace dnnf90 {

#define CKK(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));   \
      return e_ == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;   \
    }                                                                  \
  } while (0)

constexpr int KT = 32;          // tile side
constexpr int KTE = KT * KT;    // elements per tile
constexpr int RED_THREADS = 256;

// tile pass modes
constexpr int KM_PJ = 0;        // products with the first row only
constexpr int KM_UPD_PJ = 1;    // apply observation k, products with row k+1
constexpr int KM_UPD = 2;       // apply the last observation of the call

struct KfRowArgs {
  const double *rows;  // [nobs][ld]
  size_t ld;
  const double *xi;    // [nobs] innovations (target - prediction)
  const double *scale; // [nobs] or null (1)
};

__device__ __forceinline__ double row_scale(const KfRowArgs &a, int k) {
  return a.scale ? a.scale[k] : 1.0;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_kf_tiles(const int4 *__restrict__ tiles,
                                                  double *__restrict__ P, int nw,
                                                  const double *__restrict__ pj,
                                                  KfState *__restrict__ st, double *__restrict__ w,
                                                  KfRowArgs ra, int knext,
                                                  double *__restrict__ part) {
  if (st->status) return;
  const int4 t = tiles[blockIdx.x];   // x: block offset, y: block size, z: I, w: J
  const int o = t.x, n = t.y, I = t.z, J = t.w;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double s_pjR[KT], s_kvR[KT], s_pjC[KT], s_kvC[KT], s_jR[KT], s_jC[KT];
  __shared__ double s_col[8][KT + 1];
  double lam = 1.0, denom = 1.0, sg = 1.0, xi = 0.0, q = 0.0;
  if (MODE != KM_PJ) {
    lam = st->lamk;
    denom = st->denom;
    sg = st->sg;
    xi = st->xi;
    q = st->q;
  }
  if (threadIdx.x < KT) {
    const int R = I * KT + lane, C = J * KT + lane;
    if (MODE != KM_PJ) {
      const double pr = R < n ? sg * pj[o + R] : 0.0;
      const double pc = C < n ? sg * pj[o + C] : 0.0;
      s_pjR[lane] = pr;
      s_kvR[lane] = pr / denom;
      s_pjC[lane] = pc;
      s_kvC[lane] = pc / denom;
    }
    if (MODE != KM_UPD) {
      const double sn = row_scale(ra, knext);
      const double *jn = ra.rows + (size_t)knext * ra.ld;
      s_jR[lane] = R < n ? sn * jn[o + R] : 0.0;
      s_jC[lane] = C < n ? sn * jn[o + C] : 0.0;
    }
  }
  __syncthreads();
  double *tp = P + (size_t)blockIdx.x * KTE;
  double v[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) v[m] = tp[(warp + 8 * m) * KT + lane];
  const int C = J * KT + lane;
  if (MODE != KM_PJ) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int r = warp + 8 * m, R = I * KT + r;
      if (R < n && C < n) {
        const double a = v[m];
        if (R == C) {
          double d = (a - s_kvR[r] * s_pjR[r]) / lam;
          if (q > 0.0) d += q;
          v[m] = d;
        } else {
          const double x = __fma_rn(-s_kvR[r], s_pjC[lane], a);
          const double y = __fma_rn(-s_kvC[lane], s_pjR[r], a);
          v[m] = 0.5 * (x / lam + y / lam);
        }
      }
      tp[r * KT + lane] = v[m];
    }
    if (I == J && threadIdx.x < KT) {
      const int R = I * KT + lane;
      if (R < n) w[o + R] = w[o + R] + s_kvR[lane] * xi;
    }
  }
  if (MODE != KM_UPD) {
    // row sums -> slot J of the rows of tile I
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      double s = v[m] * s_jC[lane];
#pragma unroll
      for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      const int R = I * KT + warp + 8 * m;
      if (lane == 0 && R < n) part[(size_t)J * nw + o + R] = s;
    }
    if (I != J) {  // column sums -> slot I of the rows of tile J
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m) s += v[m] * s_jR[warp + 8 * m];
      s_col[warp][lane] = s;
      __syncthreads();
      if (threadIdx.x < KT) {
        double c = 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u) c += s_col[u][lane];
        if (C < n) part[(size_t)I * nw + o + C] = c;
      }
    }
  }
}

// P j of row k from the partial slots, j.Pj per CTA, and in the last CTA
// the scalars of observation k (denominator, gate, lambda).
__global__ void __launch_bounds__(RED_THREADS) k_kf_reduce(int nw, const int *__restrict__ rt,
                                                           const double *__restrict__ part,
                                                           double *__restrict__ pj, KfRowArgs ra,
                                                           int k, int kbase,
                                                           double *__restrict__ dotp,
                                                           unsigned *__restrict__ ctr,
                                                           KfState *__restrict__ st) {
  if (st->status) return;
  const int R = blockIdx.x * RED_THREADS + threadIdx.x;
  double prod = 0.0;
  if (R < nw) {
    double s = 0.0;
    const int ns = rt[R];
    for (int i = 0; i < ns; ++i) s += part[(size_t)i * nw + R];
    pj[R] = s;
    prod = row_scale(ra, k) * ra.rows[(size_t)k * ra.ld + R] * s;
  }
  __shared__ double s_red[RED_THREADS / 32];
  __shared__ bool s_last;
#pragma unroll
  for (int off = 16; off; off >>= 1) prod += __shfl_xor_sync(0xffffffffu, prod, off);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = prod;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int u = 0; u < RED_THREADS / 32; ++u) b += s_red[u];
    dotp[blockIdx.x] = b;
    __threadfence();
    s_last = atomicAdd(ctr, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double dot = 0.0;
  for (unsigned b = 0; b < gridDim.x; ++b) dot += ((volatile double *)dotp)[b];
  *ctr = 0;
  const double lam = st->lam;
  double denom = lam + dot;
  if (!(denom > 0.0)) {
    st->status = kbase + k + 1;
    return;
  }
  double xi = row_scale(ra, k) * ra.xi[k];
  double sg = 1.0;
  const double gate = st->gate;
  if (gate > 0.0) {
    const double jpj = denom - lam;
    if (xi * xi > gate * gate * denom) {
      const double s2 = gate * gate * lam / (xi * xi - gate * gate * jpj);
      sg = sqrt(s2);
      xi = sg * xi;
      denom = lam + s2 * jpj;
      st->ngated += 1;
    }
  }
  st->lamk = lam;
  st->denom = denom;
  st->sg = sg;
  st->xi = xi;
  st->lam = __dadd_rn(__dmul_rn(st->lam0, lam), 1.0) - st->lam0;
}

__global__ void k_kf_init_tiles(const int4 *__restrict__ tiles, double *__restrict__ P, double p0) {
  const int4 t = tiles[blockIdx.x];
  double *tp = P + (size_t)blockIdx.x * KTE;
  for (int e = threadIdx.x; e < KTE; e += blockDim.x) {
    const int r = e / KT, c = e - r * KT;
    const int R = t.z * KT + r, C = t.w * KT + c;
    tp[e] = (R == C && R < t.y) ? p0 : 0.0;
  }
}

void KfDev::release() {
  cudaFree(P);
  cudaFree(tiles);
  cudaFree(rt);
  cudaFree(part);
  cudaFree(pj);
  cudaFree(dotp);
  cudaFree(ctr);
  cudaFree(st);
  cudaFree(stage);
  *this = KfDev();
}

int kf_create(KfDev &d, const std::vector<int> &bsz, const std::vector<int> &boff, double p0,
              double lam_ini, double lam0, double q, double gate) {
  d.release();
  int nw = 0;
  for (size_t b = 0; b < bsz.size(); ++b) nw = std::max(nw, boff[b] + bsz[b]);
  std::vector<int4> tl;
  std::vector<int> rt(nw, 0);
  d.tmax = 0;
  for (size_t b = 0; b < bsz.size(); ++b) {
    const int n = bsz[b], o = boff[b], tb = (n + KT - 1) / KT;
    d.tmax = std::max(d.tmax, tb);
    for (int I = 0; I < tb; ++I)
      for (int J = I; J < tb; ++J) tl.push_back(make_int4(o, n, I, J));
    for (int r = 0; r < n; ++r) rt[o + r] = tb;
  }
  d.nw = nw;
  d.ntile = (int)tl.size();
  d.nred = (nw + RED_THREADS - 1) / RED_THREADS;
  CKK(cudaMalloc(&d.P, (size_t)d.ntile * KTE * sizeof(double)));
  CKK(cudaMalloc(&d.tiles, tl.size() * sizeof(int4)));
  CKK(cudaMalloc(&d.rt, nw * sizeof(int)));
  CKK(cudaMalloc(&d.part, (size_t)d.tmax * nw * sizeof(double)));
  CKK(cudaMalloc(&d.pj, nw * sizeof(double)));
  CKK(cudaMalloc(&d.dotp, d.nred * sizeof(double)));
  CKK(cudaMalloc(&d.ctr, sizeof(unsigned)));
  CKK(cudaMalloc(&d.st, sizeof(KfState)));
  CKK(cudaMemcpy(d.tiles, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CKK(cudaMemcpy(d.rt, rt.data(), nw * sizeof(int), cudaMemcpyHostToDevice));
  CKK(cudaMemset(d.ctr, 0, sizeof(unsigned)));
  KfState s{};
  s.lam = lam_ini;
  s.lam0 = lam0;
  s.q = q;
  s.gate = gate;
  CKK(cudaMemcpy(d.st, &s, sizeof(s), cudaMemcpyHostToDevice));
  LAUNCH("k_kf_init_tiles", 0, k_kf_init_tiles<<<d.ntile, 256>>>(d.tiles, d.P, p0));
  CKK(cudaGetLastError());
  CKK(cudaDeviceSynchronize());
  return RC_OK;
}

int kf_run(KfDev &d, int nobs, const double *rows, size_t ld, const double *xi,
           const double *scale, double *w, cudaStream_t s, int kbase, bool has_next) {
  if (nobs <= 0) return RC_OK;
  KfRowArgs ra{rows, ld, xi, scale};
  if (kbase == 0) {  // start of a sequence: the products with its first row
    CKK(cudaMemsetAsync(&d.st->status, 0, sizeof(int), s));
    LAUNCH("k_kf_tiles", s,
           (k_kf_tiles<KM_PJ><<<d.ntile, 256, 0, s>>>(d.tiles, d.P, d.nw, d.pj, d.st, w, ra, 0,
                                                       d.part)));
  }
  for (int k = 0; k < nobs; ++k) {
    LAUNCH("k_kf_reduce", s,
           (k_kf_reduce<<<d.nred, RED_THREADS, 0, s>>>(d.nw, d.rt, d.part, d.pj, ra, k, kbase,
                                                       d.dotp, d.ctr, d.st)));
    if (k + 1 < nobs || has_next)
      LAUNCH("k_kf_tiles", s,
             (k_kf_tiles<KM_UPD_PJ><<<d.ntile, 256, 0, s>>>(d.tiles, d.P, d.nw, d.pj, d.st, w,
                                                             ra, k + 1, d.part)));
    else
      LAUNCH("k_kf_tiles", s,
             (k_kf_tiles<KM_UPD><<<d.ntile, 256, 0, s>>>(d.tiles, d.P, d.nw, d.pj, d.st, w, ra,
                                                          0, d.part)));
  }
  CKK(cudaGetLastError());
  return RC_OK;
}

int kf_state(const KfDev &d, KfState *out, cudaStream_t s) {
  CKK(cudaMemcpyAsync(out, d.st, sizeof(KfState), cudaMemcpyDeviceToHost, s));
  CKK(cudaStreamSynchronize(s));
  return RC_OK;
}

int kf_read_cov(const KfDev &d, const std::vector<int> &bsz, const std::vector<int> &boff,
                bool dense, double *out, cudaStream_t s) {
  std::vector<double> h((size_t)d.ntile * KTE);
  std::vector<int4> tl(d.ntile);
  CKK(cudaMemcpyAsync(h.data(), d.P, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKK(cudaMemcpyAsync(tl.data(), d.tiles, tl.size() * sizeof(int4), cudaMemcpyDeviceToHost, s));
  CKK(cudaStreamSynchronize(s));
  // output offset of each block: dense [nw][nw]; decoupled blocks one after another
  std::vector<size_t> bout(bsz.size(), 0);
  for (size_t b = 1; b < bsz.size(); ++b) bout[b] = bout[b - 1] + (size_t)bsz[b - 1] * bsz[b - 1];
  size_t b = 0;
  for (int i = 0; i < d.ntile; ++i) {
    const int4 t = tl[i];
    while (boff[b] != t.x) ++b;
    const int n = t.y;
    for (int r = 0; r < KT; ++r)
      for (int c = 0; c < KT; ++c) {
        const int R = t.z * KT + r, C = t.w * KT + c;
        if (R >= n || C >= n) continue;
        const double v = h[(size_t)i * KTE + r * KT + c];
        if (dense) {
          out[(size_t)(t.x + R) * d.nw + t.x + C] = v;
          out[(size_t)(t.x + C) * d.nw + t.x + R] = v;
        } else {
          out[bout[b] + (size_t)R * n + C] = v;
          out[bout[b] + (size_t)C * n + R] = v;
        }
      }
  }
  return RC_OK;
}

}  // namespace dnnf90
