// gemm_f64.cu - the plain path's layer GEMMs in FP64 on the tensor cores
// (DMMA, mma.sync m8n8k4 f64), hand-written for the three products of the
// derivative-carrying step:
//   FWD  S[M][N]  = A[M][K] W[N][1..K]^T (+ W[N][0] on rows r % na == 0)
//        A = T_{l-1} plane, W a layer's weight rows (bias first)
//        (lib/train_module.f90:267-278)
//   DT   Tb[M][N] = A[M][K] W[K][1..N]     A = Sb plane (:430-444)
//   DW   G[j][1 + i] += sum_r A[r][j] B[r][i]  A = Sb, B = T_{l-1} (:408-422)
//
// Block tile 128 x 64, 8 warps of 32 x 32 (4 x 4 fragments of 8 x 8), a
// k-block of 16 in a three-stage cp.async ring.  Shared tiles are padded so
// that every fragment load of a warp (8-byte words) is free of bank
// conflicts.  FWD and DT run over all M tiles; DW splits its reduction over
// the rows across the grid and adds each block's partial with FP64 atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "engine.hpp"
#include "gemm_f64.hpp"

namespace dnnf90 {

namespace {

constexpr int BM = 128, BN = 64, BK = 16, NST = 3, NTH = 256;
// padded row strides (doubles) of the staged tiles
constexpr int SA_MK = BK + 4;   // A as [m][k] (FWD, DT)
constexpr int SA_KM = BM + 4;   // A as [k][m] (DW)
constexpr int SB_NK = BK + 4;   // B as [n][k] (FWD)
constexpr int SB_KN = BN + 4;   // B as [k][n] (DT, DW)
constexpr int A_WORDS = BK * SA_KM > BM * SA_MK ? BK * SA_KM : BM * SA_MK;
constexpr int B_WORDS = BN * SB_NK > BK * SB_KN ? BN * SB_NK : BK * SB_KN;
constexpr int STAGE_WORDS = A_WORDS + B_WORDS;
constexpr size_t SMEM = (size_t)NST * STAGE_WORDS * 8;

__device__ __forceinline__ uint32_t saddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// asynchronous copies, zero-filled when src_bytes is 0
__device__ __forceinline__ void cp16(double *dst, const double *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp8(double *dst, const double *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

struct F64Args {
  int M, N, K, na;
  const double *A;
  int lda;
  const double *B;  // FWD/DT: W (row length ldb); DW: B operand [K][ldb]
  int ldb;
  double *C;        // FWD/DT
  int ldc;
  int cvec;         // C is 16-byte aligned with an even ldc: pairs stored as one 16-byte store
  double *G;        // DW: [M][gld], column offset 1
  int gld;
  int kper;         // DW: rows (K) per block
};

// stage k-block kb of tile (m0, n0) into stage buffer s
template <int MODE>
__device__ __forceinline__ void load_stage(const F64Args &g, double *s, int m0, int n0, int k0,
                                           int kend) {
  double *sa = s, *sb = s + A_WORDS;
  const int t = threadIdx.x;
  if (MODE != MODE_F64_DW) {
    // A[m][k]: BM rows x BK doubles = 8 pieces of 16 bytes per row
    for (int e = t; e < BM * (BK / 2); e += NTH) {
      const int r = e >> 3, kk = (e & 7) * 2;
      const int gm = m0 + r, gk = k0 + kk;
      // K is even on every path that comes here (the tiles are 16-byte pieces)
      const bool ok = gm < g.M && gk < kend;
      cp16(sa + r * SA_MK + kk, g.A + (ok ? (size_t)gm * g.lda + gk : 0), ok ? 16 : 0);
    }
    if (MODE == MODE_F64_FWD) {
      // W[n][1 + k] as [n][k]: 8-byte pieces (the bias column breaks 16-byte alignment)
      for (int e = t; e < BN * BK; e += NTH) {
        const int n = e / BK, kk = e % BK;
        const int gn = n0 + n, gk = k0 + kk;
        const bool ok = gn < g.N && gk < kend;
        cp8(sb + n * SB_NK + kk, g.B + (ok ? (size_t)gn * g.ldb + 1 + gk : 0), ok ? 8 : 0);
      }
    } else {
      // W[k][1 + n] as [k][n]
      for (int e = t; e < BK * BN; e += NTH) {
        const int kk = e / BN, n = e % BN;
        const int gn = n0 + n, gk = k0 + kk;
        const bool ok = gn < g.N && gk < kend;
        cp8(sb + kk * SB_KN + n, g.B + (ok ? (size_t)gk * g.ldb + 1 + gn : 0), ok ? 8 : 0);
      }
    }
  } else {
    // A[r][j] rows r = k0.. as [k][m]; B[r][i] as [k][n]; 16-byte pieces
    for (int e = t; e < BK * (BM / 2); e += NTH) {
      const int kk = e / (BM / 2), m = (e % (BM / 2)) * 2;
      const int gk = k0 + kk, gm = m0 + m;
      const bool ok = gk < kend && gm < g.M;
      cp16(sa + kk * SA_KM + m, g.A + (ok ? (size_t)gk * g.lda + gm : 0), ok ? 16 : 0);
    }
    for (int e = t; e < BK * (BN / 2); e += NTH) {
      const int kk = e / (BN / 2), n = (e % (BN / 2)) * 2;
      const int gk = k0 + kk, gn = n0 + n;
      const bool ok = gk < kend && gn < g.N;
      cp16(sb + kk * SB_KN + n, g.B + (ok ? (size_t)gk * g.ldb + gn : 0), ok ? 16 : 0);
    }
  }
}

// one k-block of products from stage s into the warp's 4 x 4 fragments
template <int MODE>
__device__ __forceinline__ void compute_stage(const double *s, int wm, int wn, int lane,
                                              double (&acc)[4][4][2]) {
  const double *sa = s, *sb = s + A_WORDS;
  const int r8 = lane >> 2, c4 = lane & 3;
#pragma unroll
  for (int ks = 0; ks < BK; ks += 4) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = wm + i * 8 + r8, k = ks + c4;
      a[i] = MODE == MODE_F64_DW ? sa[k * SA_KM + m] : sa[m * SA_MK + k];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = wn + j * 8 + r8, k = ks + c4;
      b[j] = MODE == MODE_F64_FWD ? sb[n * SB_NK + k] : sb[k * SB_KN + n];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
  }
}

template <int MODE>
__global__ void __launch_bounds__(NTH) k_gemm_f64(F64Args g) {
  extern __shared__ __align__(16) double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
  const int n0 = blockIdx.y * BN;
  const int r8 = lane >> 2, c2 = (lane & 3) * 2;
  if (MODE != MODE_F64_DW) {
    // this block's M tiles blockIdx.x, + gridDim.x, ...; one cp.async ring
    // runs through all their k-blocks, so no tile waits for its ring to fill
    const int tiles = (g.M + BM - 1) / BM;
    const int nkb = (g.K + BK - 1) / BK;
    const int mine = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int total = mine * nkb;
    auto issue = [&](int s) {
      if (s < total) {
        const int t = s / nkb, kb = s - t * nkb;
        load_stage<MODE>(g, sm + (s % NST) * STAGE_WORDS, (blockIdx.x + t * gridDim.x) * BM, n0,
                         kb * BK, g.K);
      }
      commit();
    };
#pragma unroll
    for (int s = 0; s < NST - 1; ++s) issue(s);
    double acc[4][4][2];
    for (int s = 0; s < total; ++s) {
      wait_group<NST - 2>();
      __syncthreads();  // stage s is in; every warp is done with stage s - 1
      issue(s + NST - 1);
      const int t = s / nkb, kb = s - t * nkb;
      if (kb == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
      }
      compute_stage<MODE>(sm + (s % NST) * STAGE_WORDS, wm, wn, lane, acc);
      if (kb != nkb - 1) continue;
      // epilogue: rows m0 + wm + i*8 + r8, columns n0 + wn + j*8 + c2 (+0, +1)
      const int m0 = (blockIdx.x + t * gridDim.x) * BM;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm + i * 8 + r8;
        if (m >= g.M) continue;
        const bool brow = MODE == MODE_F64_FWD && (m % g.na) == 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int n = n0 + wn + j * 8 + c2;
          double v0 = acc[i][j][0], v1 = acc[i][j][1];
          if (brow) {
            if (n < g.N) v0 += g.B[(size_t)n * g.ldb];
            if (n + 1 < g.N) v1 += g.B[(size_t)(n + 1) * g.ldb];
          }
          double *c = g.C + (size_t)m * g.ldc + n;
          if (g.cvec && n + 1 < g.N) {  // n is even
            *(double2 *)c = make_double2(v0, v1);
          } else {
            if (n < g.N) c[0] = v0;
            if (n + 1 < g.N) c[1] = v1;
          }
        }
      }
    }
    wait_group<0>();
  } else {
    // rows [r0, r1) of the reduction for output tile (blockIdx.z, blockIdx.y)
    const int m0 = blockIdx.z * BM;
    const int r0 = blockIdx.x * g.kper, r1 = min(g.K, r0 + g.kper);
    if (r0 >= r1) return;
    const int nkb = (r1 - r0 + BK - 1) / BK;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
    for (int s = 0; s < NST - 1; ++s) {
      if (s < nkb) load_stage<MODE>(g, sm + s * STAGE_WORDS, m0, n0, r0 + s * BK, r1);
      commit();
    }
    for (int kb = 0; kb < nkb; ++kb) {
      wait_group<NST - 2>();
      __syncthreads();
      const int nx = kb + NST - 1;
      if (nx < nkb) load_stage<MODE>(g, sm + (nx % NST) * STAGE_WORDS, m0, n0, r0 + nx * BK, r1);
      commit();
      compute_stage<MODE>(sm + (kb % NST) * STAGE_WORDS, wm, wn, lane, acc);
    }
    wait_group<0>();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + wm + i * 8 + r8;
      if (m >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = n0 + wn + j * 8 + c2;
        double *o = g.G + (size_t)m * g.gld + 1 + n;
        if (n < g.N) atomicAdd(o, acc[i][j][0]);
        if (n + 1 < g.N) atomicAdd(o + 1, acc[i][j][1]);
      }
    }
  }
}

int sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace

int gemm_f64(int mode, int M, int N, int K, int na, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double *G, int gld, cudaStream_t st) {
  // 16-byte pieces of A (and of B in DW) need even leading dimensions and
  // 16-byte aligned bases
  if ((lda & 1) || ((uintptr_t)A & 15) || (mode == MODE_F64_DW && ((ldb & 1) || ((uintptr_t)B & 15))) ||
      (mode != MODE_F64_DW && (K & 1)) || (mode == MODE_F64_DW && (M & 1 || N & 1)))
    return RC_UNSUPPORTED;
  F64Args g;
  g.M = M; g.N = N; g.K = K; g.na = na; g.A = A; g.lda = lda; g.B = B; g.ldb = ldb;
  g.C = C; g.ldc = ldc; g.G = G; g.gld = gld; g.kper = 0;
  g.cvec = C && ((uintptr_t)C & 15) == 0 && (ldc & 1) == 0;
  const int ntn = (N + BN - 1) / BN;
  cudaError_t e;
  if (mode == MODE_F64_FWD || mode == MODE_F64_DT) {
    const int tiles = (M + BM - 1) / BM;
    // two blocks per SM fit the shared memory; one wave of persistent blocks
    const int gx = std::max(1, std::min(tiles, sms() * 2 / std::max(1, ntn)));
    dim3 grid(gx, ntn);
    if (mode == MODE_F64_FWD) {
      cudaFuncSetAttribute(k_gemm_f64<MODE_F64_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
      LAUNCH("k_gemm_f64_fwd", st, (k_gemm_f64<MODE_F64_FWD><<<grid, NTH, SMEM, st>>>(g)));
    } else {
      cudaFuncSetAttribute(k_gemm_f64<MODE_F64_DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
      LAUNCH("k_gemm_f64_dt", st, (k_gemm_f64<MODE_F64_DT><<<grid, NTH, SMEM, st>>>(g)));
    }
  } else {
    // DW: output tiles (N tiles x M tiles), the row reduction split so that
    // about two blocks per SM run, each over a multiple of BK rows
    const int mt = (M + BM - 1) / BM;
    const int want = std::max(1, sms() * 2 / std::max(1, ntn * mt));
    int kper = (K + want - 1) / want;
    kper = std::max(BK, (kper + BK - 1) / BK * BK);
    g.kper = kper;
    dim3 grid((K + kper - 1) / kper, ntn, mt);
    cudaFuncSetAttribute(k_gemm_f64<MODE_F64_DW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    LAUNCH("k_gemm_f64_dw", st, (k_gemm_f64<MODE_F64_DW><<<grid, NTH, SMEM, st>>>(g)));
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("k_gemm_f64: ") + cudaGetErrorString(e));
    return RC_DEVICE;
  }
  return RC_OK;
}

}  // namespace dnnf90
