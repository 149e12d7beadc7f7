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
//     P_ij <- ((a - kv_i pj_j) + (a - kv_j pj_i)) / (2 lambda),
// an expression symmetric in (i, j), so each stored element is updated from
// its own value alone and the triangle never needs the transposed entry
// (the reference divides each term by lambda before the average; the two
// differ by rounding only).
//
// One observation is two launches.  The tile pass applies observation k
// (downdate, process noise, and w += kv xi on the diagonal tiles) and, in
// the same read of each tile, forms the products of the NEW covariance with
// the next row: row sums of tile (I, J) land in partial slot J of the rows
// of I, column sums in slot I of the rows of J, so that every (slot, row)
// is written once and no atomics are needed.  The reduce pass sums the
// slots into P j for that row, forms j.Pj per row tile, and its last CTA
// (found with a counter, no waiting) sums the row tiles' shares in a fixed
// order into the global denominator, applies the innovation gate and
// advances lambda.  A call therefore reads and writes the covariance once
// per observation, plus one read-only pass for the first row.
//
// Small filters run a whole call as one cooperative launch (k_kf_seq): the
// same tile code, reduce and scalar step as phases between bounded grid
// barriers, with the same summation orders, so both paths give the same
// bits.  The iterated EKF (kf_iekf_iter) reuses the two-launch kernels, and
// the per-point pass (dnnf90_kf_pass) calls kf_run once per point with
// that point's row formed on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
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

// which update path kf_run takes: -1 by size (the one-launch sequence for
// small filters), 0 two launches per update, 1 the one-launch sequence
static std::atomic<int> g_kf_path{-1};

int kf_force_path(int path) {
  if (path < -1 || path > 1) return RC_BAD_ARG;
  g_kf_path = path;
  return RC_OK;
}

constexpr int KT = 32;          // tile side
constexpr int KTE = KT * KT;    // elements per tile
constexpr int RED_THREADS = 512;

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

// iterated EKF: the prior weights and the current ones (wprior null: a
// plain update)
struct KfIekf {
  const double *wprior;
  const double *w;
  int final;
};

__device__ __forceinline__ double row_scale(const KfRowArgs &a, int k) {
  return a.scale ? a.scale[k] : 1.0;
}

// (I, J) of tile t in the row-major upper triangle of tb x tb tiles, where
// row I starts at t0(I) = I tb - I (I - 1) / 2
__device__ __forceinline__ void tri_tile(int t, int tb, int &I, int &J) {
  const double b = 2.0 * tb + 1.0;
  int i = (int)((b - sqrt(b * b - 8.0 * t)) * 0.5);
  auto t0 = [tb](int r) { return (long long)r * tb - (long long)r * (r - 1) / 2; };
  while (i > 0 && t0(i) > t) --i;
  while (i + 1 < tb && t0(i + 1) <= t) ++i;
  I = i;
  J = i + (int)(t - t0(i));
}

// the scalars of the observation a tile pass applies
struct KfScal {
  double lam, denom, sg, xi, q;
};

// Where tile t sits: block offset o, block size n, tile (I, J) and the
// block's partial slots.  DENSE (a single block of nw) derives the position
// from the index, so that nothing the vector loads need waits on a table
// read; the decoupled filter reads its tile table.
template <bool DENSE>
__device__ __forceinline__ void kf_tile_at(int t, const int4 *__restrict__ tiles, int nw,
                                           double *part, int &o, int &n, int &I, int &J,
                                           double *&pslot) {
  if (DENSE) {
    o = 0;
    n = nw;
    tri_tile(t, (nw + KT - 1) / KT, I, J);
    pslot = part;
  } else {
    // x: block offset, y: block size, z: I | J << 16, w: the block's partial slots
    const int4 d = tiles[t];
    o = d.x;
    n = d.y;
    I = d.z & 0xffff;
    J = d.z >> 16;
    pslot = part + d.w;
  }
}

// One tile of the pass, its elements v already loaded: the update of
// observation k (MODE != KM_PJ) and the products of the result with the
// next row (MODE != KM_UPD).  Every thread of the CTA calls it.
template <int MODE, bool CG = false>
__device__ __forceinline__ void kf_tile_body(double *tp, double (&v)[4], int o, int n, int I,
                                             int J, double *pslot, const double *__restrict__ pj,
                                             const KfScal &sc, double *__restrict__ w,
                                             const double *__restrict__ wb, const KfRowArgs &ra,
                                             int knext) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tb = (n + KT - 1) / KT;
  __shared__ double s_pjR[KT], s_kvR[KT], s_pjC[KT], s_kvC[KT], s_jR[KT], s_jC[KT];
  __shared__ double s_col[8][KT + 1];
  if (threadIdx.x < KT) {
    const int R = I * KT + lane, C = J * KT + lane;
    if (MODE != KM_PJ) {
      // CG: P j was written by other CTAs of the same launch (the
      // one-launch sequence), so it is read past L1
      const double pr = R < n ? sc.sg * (CG ? __ldcg(pj + o + R) : pj[o + R]) : 0.0;
      const double pc = C < n ? sc.sg * (CG ? __ldcg(pj + o + C) : pj[o + C]) : 0.0;
      s_pjR[lane] = pr;
      s_kvR[lane] = pr / sc.denom;
      s_pjC[lane] = pc;
      s_kvC[lane] = pc / sc.denom;
    }
    if (MODE != KM_UPD) {
      const double sn = row_scale(ra, knext);
      const double *jn = ra.rows + (size_t)knext * ra.ld;
      s_jR[lane] = R < n ? sn * jn[o + R] : 0.0;
      s_jC[lane] = C < n ? sn * jn[o + C] : 0.0;
    }
  }
  __syncthreads();
  const int C = J * KT + lane;
  if (MODE != KM_PJ) {
    // 1/lambda once per tile: an FP64 division per element would cost as
    // much as the element's HBM traffic (lambda = 1 is exact either way)
    const double rl = 1.0 / sc.lam, hl = 0.5 * rl;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int r = warp + 8 * m, R = I * KT + r;
      if (R < n && C < n) {
        const double a = v[m];
        if (R == C) {
          double d = __fma_rn(-s_kvR[r], s_pjR[r], a) * rl;
          if (sc.q > 0.0) d += sc.q;
          v[m] = d;
        } else {
          const double x = __fma_rn(-s_kvR[r], s_pjC[lane], a);
          const double y = __fma_rn(-s_kvC[lane], s_pjR[r], a);
          v[m] = (x + y) * hl;
        }
      }
      __stcs(tp + r * KT + lane, v[m]);
    }
    if (I == J && threadIdx.x < KT) {
      const int R = I * KT + lane;
      if (R < n) w[o + R] = __fma_rn(s_kvR[lane], sc.xi, wb[o + R]);
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
      if (lane == 0 && R < n) pslot[((size_t)I * tb + J) * KT + warp + 8 * m] = s;
    }
    if (I != J) {  // column sums -> slot I of the rows of tile J
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m) s = __fma_rn(v[m], s_jR[warp + 8 * m], s);
      s_col[warp][lane] = s;
      __syncthreads();
      if (threadIdx.x < KT) {
        double c = 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u) c += s_col[u][lane];
        if (C < n) pslot[((size_t)J * tb + I) * KT + lane] = c;
      }
    }
  }
}

// One CTA per tile.
template <int MODE, bool DENSE>
__global__ void __launch_bounds__(256, 8) k_kf_tiles(const int4 *__restrict__ tiles,
                                                     double *__restrict__ P, int nw,
                                                     const double *__restrict__ pj,
                                                     KfState *__restrict__ st,
                                                     double *__restrict__ w,
                                                     const double *__restrict__ wb,
                                                     KfRowArgs ra, int knext,
                                                     double *__restrict__ part) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the tile's own elements first: their addresses depend on nothing else,
  // so the HBM reads are in flight while the scalars and vectors arrive.
  // The covariance streams through with evict-first loads and stores, so
  // that the partial slots written beside it stay in L2 for the reduce.
  double *tp = P + (size_t)blockIdx.x * KTE;
  double v[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) v[m] = __ldcs(tp + (warp + 8 * m) * KT + lane);
  int o, n, I, J;
  double *pslot;
  kf_tile_at<DENSE>(blockIdx.x, tiles, nw, part, o, n, I, J, pslot);
  if (st->status) return;
  KfScal sc{1.0, 1.0, 1.0, 0.0, 0.0};
  if (MODE != KM_PJ) sc = KfScal{st->lamk, st->denom, st->sg, st->xi, st->q};
  kf_tile_body<MODE>(tp, v, o, n, I, J, pslot, pj, sc, w, wb, ra, knext);
}

// Sum of the row tiles' shares dotp[2b] (and dotp[2b + 1]) over b < n in a
// fixed order that does not depend on the block size: thread i < 256 adds
// b = i, i + 256, ... in turn, and the 256 partial sums are added pairwise
// (i + 128, i + 64, ...).  Every thread of the block calls it (at least 256
// of them); the sums are returned to all.  The shares come from other CTAs,
// so they are read past L1.
__device__ __forceinline__ void kf_dot_sum(const double *dotp, int n, double &dot, double &cor) {
  __shared__ double s_d[256], s_c[256];
  const int i = threadIdx.x;
  if (i < 256) {
    double d = 0.0, c = 0.0;
    for (int b = i; b < n; b += 256) {
      d += __ldcg(dotp + 2 * b);
      c += __ldcg(dotp + 2 * b + 1);
    }
    s_d[i] = d;
    s_c[i] = c;
  }
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (i < h) {
      s_d[i] += s_d[i + h];
      s_c[i] += s_c[i + h];
    }
    __syncthreads();
  }
  dot = s_d[0];
  cor = s_c[0];
  __syncthreads();
}

// P j of row k from the partial slots, j.Pj per CTA, and in the last CTA
// the scalars of observation k (denominator, gate, lambda).  One CTA per
// row tile: its slots are contiguous ([slot][32]), warp g of 16 sums slots
// g, g + 16, ..., and the sixteen sums of a row are added in a fixed order.
__global__ void __launch_bounds__(RED_THREADS) k_kf_reduce(const int4 *__restrict__ rtl,
                                                           const double *__restrict__ part,
                                                           double *__restrict__ pj, KfRowArgs ra,
                                                           int k, int kbase, KfIekf ie,
                                                           double *__restrict__ dotp,
                                                           unsigned *__restrict__ ctr,
                                                           KfState *__restrict__ st) {
  if (st->status) return;
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int4 rt = rtl[blockIdx.x];  // x: first weight, y: rows, z: slots, w: slot offset
  const double *src = part + rt.w;
  __shared__ double s_sum[RED_THREADS / 32][33];
  __shared__ bool s_last;
  double s = 0.0;
#pragma unroll 8
  for (int i = g; i < rt.z; i += RED_THREADS / 32) s += src[(size_t)i * KT + lane];
  s_sum[g][lane] = s;
  __syncthreads();
  if (g == 0) {
    double p = 0.0, prod = 0.0, corr = 0.0;
#pragma unroll
    for (int u = 0; u < RED_THREADS / 32; ++u) p += s_sum[u][lane];
    if (lane < rt.y) {
      const int R = rt.x + lane;
      const double jf = row_scale(ra, k) * ra.rows[(size_t)k * ra.ld + R];
      pj[R] = p;
      prod = jf * p;
      if (ie.wprior) corr = jf * (ie.wprior[R] - ie.w[R]);
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      prod += __shfl_xor_sync(0xffffffffu, prod, off);
      corr += __shfl_xor_sync(0xffffffffu, corr, off);
    }
    if (lane == 0) {
      dotp[2 * blockIdx.x] = prod;
      dotp[2 * blockIdx.x + 1] = corr;
      __threadfence();
      s_last = atomicAdd(ctr, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double dot, cor;
  kf_dot_sum(dotp, gridDim.x, dot, cor);
  if (threadIdx.x != 0) return;
  *ctr = 0;
  const double lam = st->lam;
  double denom = lam + dot;
  if (!(denom > 0.0)) {
    st->status = kbase + k + 1;
    return;
  }
  double xi, sg = 1.0;
  if (ie.wprior) {
    // iterated EKF (kf_iekf_iter :534-640): the innovation linearised at the
    // prior, xi = -scale R - jf.(w- - w_i); no gate; lambda advances only
    // with the covariance on the final iteration
    xi = -row_scale(ra, k) * ra.xi[k] - cor;
  } else {
    xi = row_scale(ra, k) * ra.xi[k];
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
  }
  st->lamk = lam;
  st->denom = denom;
  st->sg = sg;
  st->xi = xi;
  if (!ie.wprior || ie.final) st->lam = __dadd_rn(__dmul_rn(st->lam0, lam), 1.0) - st->lam0;
}

// w = w- + kv xi without touching the covariance (a non-final IEKF iteration)
__global__ void k_kf_wonly(int nw, double *__restrict__ w, const double *__restrict__ wb,
                           const double *__restrict__ pj, const KfState *__restrict__ st) {
  if (st->status) return;
  const int R = blockIdx.x * blockDim.x + threadIdx.x;
  if (R < nw) w[R] = wb[R] + (st->sg * pj[R] / st->denom) * st->xi;
}

// ---------------------------------------------------- whole sequence, one launch
// For a small filter the two launches of an update cost more than their
// work.  k_kf_seq runs a whole call as one cooperative launch: the tile
// pass, the reduce and the scalars of every observation as phases separated
// by grid barriers, with the same per-tile code and the same summation
// orders as the two-kernel path, so the results are bit-identical.  The
// scalars are formed by every CTA from the same values; lambda and the gate
// count live in registers and CTA 0 writes them back at the end.

constexpr long KF_BAR_LIMIT = 1L << 24;  // polls before a grid barrier gives up

// barrier among the CTAs of a cooperative launch (sense by generation);
// false, with status -1, when a wait runs out or another CTA gave up
__device__ bool kf_grid_sync(KfBar *b, KfState *st) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = *(volatile unsigned *)&b->gen;
    __threadfence();
    if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      ok = 0;
      for (long i = 0; i < KF_BAR_LIMIT; ++i) {
        if (*(volatile unsigned *)&b->gen != g) {
          ok = 1;
          break;
        }
        if (*(volatile int *)&st->status < 0) break;
        if (i > 32) __nanosleep(32);
      }
      if (!ok) atomicCAS(&st->status, 0, -1);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// the tiles of this CTA (t = blockIdx, blockIdx + grid, ...)
template <int MODE, bool DENSE>
__device__ __forceinline__ void kf_seq_tiles(const int4 *__restrict__ tiles, int ntile,
                                             double *__restrict__ P, int nw,
                                             const double *__restrict__ pj, const KfScal &sc,
                                             double *__restrict__ w, const KfRowArgs &ra,
                                             int knext, double *__restrict__ part) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    double *tp = P + (size_t)t * KTE;
    double v[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) v[m] = __ldcs(tp + (warp + 8 * m) * KT + lane);
    int o, n, I, J;
    double *pslot;
    kf_tile_at<DENSE>(t, tiles, nw, part, o, n, I, J, pslot);
    kf_tile_body<MODE, true>(tp, v, o, n, I, J, pslot, pj, sc, w, w, ra, knext);
    __syncthreads();  // the tile's vectors are read before the next tile writes them
  }
}

template <bool DENSE>
__global__ void __launch_bounds__(256) k_kf_seq(const int4 *__restrict__ tiles, int ntile,
                                                double *__restrict__ P, int nw,
                                                const int4 *__restrict__ rtl, int nred,
                                                double *__restrict__ part, double *__restrict__ pj,
                                                double *__restrict__ dotp,
                                                KfState *__restrict__ st, KfBar *__restrict__ bar,
                                                double *__restrict__ w, KfRowArgs ra, int nobs,
                                                int kbase, int first, int has_next) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ double s_sum[16][33];
  __shared__ KfScal s_sc;
  __shared__ int s_fail;
  if (*(volatile int *)&st->status) return;
  double lam = st->lam;
  const double lam0 = st->lam0, q = st->q, gate = st->gate;
  int ngated = st->ngated;
  KfScal sc{1.0, 1.0, 1.0, 0.0, q};
  if (first) {
    kf_seq_tiles<KM_PJ, DENSE>(tiles, ntile, P, nw, pj, sc, w, ra, 0, part);
    if (!kf_grid_sync(bar, st)) return;
  }
  for (int k = 0; k < nobs; ++k) {
    // reduce: P j of row k and the row tiles' shares of j.Pj, in the order
    // of k_kf_reduce (16 slot groups: this warp takes groups warp, warp + 8)
    for (int rt = blockIdx.x; rt < nred; rt += gridDim.x) {
      const int4 r = rtl[rt];
      const double *src = part + r.w;
      double s0 = 0.0, s1 = 0.0;
      for (int i = warp; i < r.z; i += 16) s0 += __ldcg(src + (size_t)i * KT + lane);
      for (int i = warp + 8; i < r.z; i += 16) s1 += __ldcg(src + (size_t)i * KT + lane);
      s_sum[warp][lane] = s0;
      s_sum[warp + 8][lane] = s1;
      __syncthreads();
      if (warp == 0) {
        double p = 0.0, prod = 0.0;
#pragma unroll
        for (int u = 0; u < 16; ++u) p += s_sum[u][lane];
        if (lane < r.y) {
          const int R = r.x + lane;
          pj[R] = p;
          prod = row_scale(ra, k) * ra.rows[(size_t)k * ra.ld + R] * p;
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) prod += __shfl_xor_sync(0xffffffffu, prod, off);
        if (lane == 0) {
          dotp[2 * rt] = prod;
          dotp[2 * rt + 1] = 0.0;
        }
      }
      __syncthreads();
    }
    if (!kf_grid_sync(bar, st)) return;
    // the scalars of observation k, the same in every CTA
    double dot, cor;
    kf_dot_sum(dotp, nred, dot, cor);
    if (threadIdx.x == 0) {
      double denom = lam + dot;
      int fail = !(denom > 0.0);
      double xi = row_scale(ra, k) * ra.xi[k], sg = 1.0;
      if (!fail && gate > 0.0) {
        const double jpj = denom - lam;
        if (xi * xi > gate * gate * denom) {
          const double s2 = gate * gate * lam / (xi * xi - gate * gate * jpj);
          sg = sqrt(s2);
          xi = sg * xi;
          denom = lam + s2 * jpj;
          ++ngated;
        }
      }
      s_sc = KfScal{lam, denom, sg, xi, q};
      s_fail = fail;
    }
    __syncthreads();
    if (s_fail) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->status = kbase + k + 1;
        st->lam = lam;
        st->ngated = ngated;
      }
      return;
    }
    sc = s_sc;
    lam = __dadd_rn(__dmul_rn(lam0, lam), 1.0) - lam0;
    if (k + 1 < nobs || has_next) {
      kf_seq_tiles<KM_UPD_PJ, DENSE>(tiles, ntile, P, nw, pj, sc, w, ra, k + 1, part);
      if (!kf_grid_sync(bar, st)) return;
    } else {
      kf_seq_tiles<KM_UPD, DENSE>(tiles, ntile, P, nw, pj, sc, w, ra, 0, part);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->lam = lam;
    st->ngated = ngated;
    st->lamk = sc.lam;
    st->denom = sc.denom;
    st->sg = sc.sg;
    st->xi = sc.xi;
  }
}

__global__ void k_kf_init_tiles(const int4 *__restrict__ tiles, double *__restrict__ P, double p0) {
  const int4 t = tiles[blockIdx.x];
  double *tp = P + (size_t)blockIdx.x * KTE;
  for (int e = threadIdx.x; e < KTE; e += blockDim.x) {
    const int r = e / KT, c = e - r * KT;
    const int R = (t.z & 0xffff) * KT + r, C = (t.z >> 16) * KT + c;
    tp[e] = (R == C && R < t.y) ? p0 : 0.0;
  }
}

void KfDev::release() {
  cudaFree(P);
  cudaFree(tiles);
  cudaFree(rtl);
  cudaFree(part);
  cudaFree(pj);
  cudaFree(dotp);
  cudaFree(ctr);
  cudaFree(st);
  cudaFree(bar);
  cudaFree(stage);
  cudaFree(wprior);
  *this = KfDev();
}

int kf_create(KfDev &d, const std::vector<int> &bsz, const std::vector<int> &boff, double p0,
              double lam_ini, double lam0, double q, double gate) {
  d.release();
  int nw = 0;
  for (size_t b = 0; b < bsz.size(); ++b) nw = std::max(nw, boff[b] + bsz[b]);
  // tiles (I <= J) of each block's triangle, and the block's partial slots:
  // [row tile K][slot s][32] at a per-block offset
  std::vector<int4> tl, rtl;
  size_t pslots = 0;
  for (size_t b = 0; b < bsz.size(); ++b) {
    const int n = bsz[b], o = boff[b], tb = (n + KT - 1) / KT;
    if (tb > 0xffff) {
      set_error("kalman: covariance block too large");
      return RC_UNSUPPORTED;
    }
    for (int I = 0; I < tb; ++I)
      for (int J = I; J < tb; ++J) tl.push_back(make_int4(o, n, I | J << 16, (int)pslots));
    for (int K = 0; K < tb; ++K)
      rtl.push_back(make_int4(o + K * KT, std::min(KT, n - K * KT), tb,
                              (int)(pslots + (size_t)K * tb * KT)));
    pslots += (size_t)tb * tb * KT;
    if (pslots > (size_t)INT32_MAX) {
      set_error("kalman: covariance too large for the partial-slot index");
      return RC_UNSUPPORTED;
    }
  }
  d.nw = nw;
  d.dense = bsz.size() == 1;
  d.ntile = (int)tl.size();
  d.nred = (int)rtl.size();
  CKK(cudaMalloc(&d.P, (size_t)d.ntile * KTE * sizeof(double)));
  CKK(cudaMalloc(&d.tiles, tl.size() * sizeof(int4)));
  CKK(cudaMalloc(&d.rtl, rtl.size() * sizeof(int4)));
  CKK(cudaMalloc(&d.part, pslots * sizeof(double)));
  CKK(cudaMalloc(&d.pj, nw * sizeof(double)));
  CKK(cudaMalloc(&d.dotp, 2 * d.nred * sizeof(double)));
  CKK(cudaMalloc(&d.wprior, nw * sizeof(double)));
  CKK(cudaMalloc(&d.ctr, sizeof(unsigned)));
  CKK(cudaMalloc(&d.st, sizeof(KfState)));
  CKK(cudaMalloc(&d.bar, sizeof(KfBar)));
  CKK(cudaMemset(d.bar, 0, sizeof(KfBar)));
  {
    int coop = 0, dev = 0, per_sm = 0;
    CKK(cudaGetDevice(&dev));
    CKK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    CKK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, d.dense ? k_kf_seq<true> : k_kf_seq<false>, 256, 0));
    d.seq_grid = coop && per_sm > 0 ? std::min(grid_sms() * per_sm, std::max(d.ntile, d.nred))
                                    : 0;
  }
  CKK(cudaMemcpy(d.tiles, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CKK(cudaMemcpy(d.rtl, rtl.data(), rtl.size() * sizeof(int4), cudaMemcpyHostToDevice));
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
           const double *scale, double *w, cudaStream_t s, int kbase, bool has_next,
           bool first) {
  if (nobs <= 0) return RC_OK;
  KfRowArgs ra{rows, ld, xi, scale};
  int path = g_kf_path.load();
  // a stream being captured into a graph takes the two-launch path, whose
  // kernels are plain launches
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    path = 0;
  // measured: one launch wins up to about 2K tiles (MLP 3-32-32-1 dense, 741
  // tiles, 70K against 63K updates/s; 2-128-128-1 decoupled, 2063 tiles, 46K
  // against 43K) and loses from 10K tiles on (3-64-64-1: 13K against 21K)
  if (d.seq_grid > 0 && (path == 1 || (path < 0 && d.ntile <= 8 * d.seq_grid))) {
    if (kbase == 0) CKK(cudaMemsetAsync(&d.st->status, 0, sizeof(int), s));
    int fi = first ? 1 : 0, hn = has_next ? 1 : 0, ntile = d.ntile, nw = d.nw, nred = d.nred;
    void *args[] = {&d.tiles, &ntile, &d.P, &nw, &d.rtl, &nred, &d.part, &d.pj, &d.dotp,
                    &d.st, &d.bar, &w, &ra, &nobs, &kbase, &fi, &hn};
    const void *fn = d.dense ? (const void *)k_kf_seq<true> : (const void *)k_kf_seq<false>;
    CKK(cudaMemsetAsync(d.bar, 0, sizeof(KfBar), s));  // a barrier that gave up leaves a count
    int pi = prof_begin("k_kf_seq", s);
    const cudaError_t e = cudaLaunchCooperativeKernel(fn, d.seq_grid, 256, args, 0, s);
    prof_end(pi, s);
    note_launch();
    CKK(e);
    return RC_OK;
  }
  if (kbase == 0) CKK(cudaMemsetAsync(&d.st->status, 0, sizeof(int), s));
  if (first) {  // the products with the call's first row
    LAUNCH("k_kf_tiles_pj", s,
           (d.dense ? k_kf_tiles<KM_PJ, true> : k_kf_tiles<KM_PJ, false>)<<<d.ntile, 256, 0, s>>>(
               d.tiles, d.P, d.nw, d.pj, d.st, w, w, ra, 0, d.part));
  }
  const KfIekf plain{nullptr, nullptr, 0};
  for (int k = 0; k < nobs; ++k) {
    LAUNCH("k_kf_reduce", s,
           (k_kf_reduce<<<d.nred, RED_THREADS, 0, s>>>(d.rtl, d.part, d.pj, ra, k, kbase,
                                                       plain, d.dotp, d.ctr, d.st)));
    if (k + 1 < nobs || has_next)
      LAUNCH("k_kf_tiles", s,
             (d.dense ? k_kf_tiles<KM_UPD_PJ, true> : k_kf_tiles<KM_UPD_PJ, false>)<<<
                 d.ntile, 256, 0, s>>>(d.tiles, d.P, d.nw, d.pj, d.st, w, w, ra, k + 1, d.part));
    else
      LAUNCH("k_kf_tiles", s,
             (d.dense ? k_kf_tiles<KM_UPD, true> : k_kf_tiles<KM_UPD, false>)<<<
                 d.ntile, 256, 0, s>>>(d.tiles, d.P, d.nw, d.pj, d.st, w, w, ra, 0, d.part));
  }
  CKK(cudaGetLastError());
  return RC_OK;
}

int kf_iekf(KfDev &d, const double *row, const double *resid, const double *scale, double *w,
            bool final, cudaStream_t s, int kbase, bool reset) {
  KfRowArgs ra{row, (size_t)d.nw, resid, scale};
  const KfIekf ie{d.wprior, w, final ? 1 : 0};
  if (reset) CKK(cudaMemsetAsync(&d.st->status, 0, sizeof(int), s));
  LAUNCH("k_kf_tiles_pj", s,
         (d.dense ? k_kf_tiles<KM_PJ, true> : k_kf_tiles<KM_PJ, false>)<<<d.ntile, 256, 0, s>>>(
             d.tiles, d.P, d.nw, d.pj, d.st, w, w, ra, 0, d.part));
  LAUNCH("k_kf_reduce", s,
         (k_kf_reduce<<<d.nred, RED_THREADS, 0, s>>>(d.rtl, d.part, d.pj, ra, 0, kbase, ie,
                                                     d.dotp, d.ctr, d.st)));
  if (final)
    LAUNCH("k_kf_tiles", s,
           (d.dense ? k_kf_tiles<KM_UPD, true> : k_kf_tiles<KM_UPD, false>)<<<d.ntile, 256, 0,
                                                                              s>>>(
               d.tiles, d.P, d.nw, d.pj, d.st, w, d.wprior, ra, 0, d.part));
  else
    LAUNCH("k_kf_wonly", s,
           (k_kf_wonly<<<(d.nw + 255) / 256, 256, 0, s>>>(d.nw, w, d.wprior, d.pj, d.st)));
  CKK(cudaGetLastError());
  return RC_OK;
}

// xi = -R for one point from its output derivatives out[na][nout] (the
// first component) and a residual rule, in the order of the host's
// residual (R = sum_k c_k T_k, or c_k T_0 T_k for a nonlinear term)
__global__ void k_kf_resid(DevRule r, const double *__restrict__ out, int nout,
                           double *__restrict__ xi, double sign) {
  if (threadIdx.x != 0) return;
  double R = 0.0;
  for (int k = 0; k < r.nterm; ++k)
    R = r.nonlin[k] ? R + r.coeff[k] * out[0] * out[(size_t)r.ind[k] * nout]
                    : R + r.coeff[k] * out[(size_t)r.ind[k] * nout];
  *xi = sign * R;
}

int kf_resid_xi(const DevRule &r, const double *out, int nout, double *xi, cudaStream_t s,
                double sign) {
  LAUNCH("k_kf_resid", s, (k_kf_resid<<<1, 32, 0, s>>>(r, out, nout, xi, sign)));
  CKK(cudaGetLastError());
  return RC_OK;
}

// One observation of a system (the trainer's loop over sys_nres,
// app/sgd_batch_module.f90:497-545): from one point's output derivatives
// out[na][nout], residual ir of a system rule (calc_sys_residual,
// app/pinn_module.f90:86-125) as xi = sign * R_ir, and its seed dR_ir/dT
// in seed[nout][na] (set_sys_seed :127-162 with a one in slot ir, fac 1,
// unweighted).
__global__ void k_kf_sys_seed(DevRule r, const double *__restrict__ out, int na, int nout,
                              const double *__restrict__ src, int ir,
                              double *__restrict__ seed, double *__restrict__ xi, double sign) {
  for (int i = threadIdx.x; i < nout * na; i += blockDim.x) seed[i] = 0.0;
  __syncthreads();
  if (threadIdx.x != 0) return;
  auto T = [&](int f) {  // factor f: (component, slot), 0-based
    return out[(size_t)r.sfac[2 * f + 1] * nout + r.sfac[2 * f]];
  };
  double R = src ? -src[ir] : 0.0;
  for (int k = 0; k < r.nterm; ++k) {
    if (r.sys[3 * k] != ir) continue;
    const int nf = r.sys[3 * k + 1], f0 = r.sys[3 * k + 2];
    double prod = r.coeff[k];
    for (int m = 0; m < nf; ++m) prod = prod * T(f0 + m);
    R = R + prod;
    for (int m = 0; m < nf; ++m) {
      double other = r.coeff[k];
      for (int mm = 0; mm < nf; ++mm)
        if (mm != m) other = other * T(f0 + mm);
      const int at = r.sfac[2 * (f0 + m)] * na + r.sfac[2 * (f0 + m) + 1];
      seed[at] = seed[at] + other;
    }
  }
  *xi = sign * R;
}

int kf_sys_seed(const DevRule &r, const double *out, int na, int nout, const double *src,
                int ir, double *seed, double *xi, double sign, cudaStream_t s) {
  LAUNCH("k_kf_sys_seed", s,
         (k_kf_sys_seed<<<1, 256, 0, s>>>(r, out, na, nout, src, ir, seed, xi, sign)));
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
        const int R = (t.z & 0xffff) * KT + r, C = (t.z >> 16) * KT + c;
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
