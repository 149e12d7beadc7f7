// gemm_f64.cu - the plain path's layer GEMMs in FP64 on the tensor cores
// (DMMA, mma.sync m8n8k4 f64), hand-written for the three products of the
// derivative-carrying step:
//   FWD  S[M][N]  = A[M][K] W[N][1..K]^T (+ W[N][0] on rows r % na == 0)
//        A = T_{l-1} plane, W a layer's weight rows (bias first)
//        (lib/train_module.f90:267-278)
//   DT   Tb[M][N] = A[M][K] W[K][1..N]     A = Sb plane (:430-444)
//   DW   G[j][1 + i] += sum_r A[r][j] B[r][i]  A = Sb, B = T_{l-1} (:408-422)
//
// Block tile 64 x 64, 4 warps of 32 x 32 (4 x 4 fragments of 8 x 8), a
// k-block of 16 in a three-stage cp.async ring; four blocks per SM.  FWD
// and DT finish a tile every K / 16 = 8 k-blocks, and a warp's stores wait
// for its last products: with four independent blocks per SM (one warp of
// each per scheduler) the blocks drift apart and one block's epilogue
// overlaps the others' products (measured at K = 128: 8 warps per block,
// two blocks per SM, ran FWD at 28.5 TFLOP/s; this shape at 30.7).
//
// Fragments.  One m8n8k4 product sums over the four k its lanes hold, and
// a warp's fragments cover its 32 x 32 tile whichever rows and columns each
// fragment takes, so the kernel assigns k, m and n to lanes so that every
// shared load is 16 bytes wide (two fragments, or two k-steps, per load):
//   - [m][k] tiles (A of FWD and DT, B of FWD): lane k = 4 c4 + ks, so a
//     lane's four k of a k-block are adjacent; fragment rows 8 i + r8;
//   - [k][x] tiles (A and B of DW, B of DT): fragment i (j) takes rows
//     (columns) x = 16 (i >> 1) + 2 r8 + (i & 1), so fragments 2 ii and
//     2 ii + 1 are adjacent; DT stores W row k of its k-block at row
//     4 (k & 3) + (k >> 2), where its k = 4 c4 + ks lands at 4 ks + c4.
// (r8 = lane / 4, c4 = lane % 4: the m8n8k4 fragment coordinates.)  The
// padded row strides (18 doubles for [m][k]; BM + 4 and BN + 4 for [k][x],
// BM, BN in {64, 128}) put the eight lanes of each 16-byte load phase on
// eight distinct 16-byte bank groups.  FWD and DT run over all M tiles in
// one ring; DW splits its reduction over the rows across the grid and adds
// each block's partial with FP64 atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "engine.hpp"
#include "gemm_f64.hpp"

namespace dnnf90 {

namespace {

// block shape (compile-time; 64 x 64 x 3 stages measured fastest at K = 128)
#ifndef F64_BM
#define F64_BM 64
#endif
#ifndef F64_BN
#define F64_BN 64
#endif
#ifndef F64_NST
#define F64_NST 3
#endif
constexpr int MI = 4, NJ = 4;   // 8 x 8 fragments per warp in m and in n
constexpr int BM = F64_BM, BN = F64_BN, BK = 16, NST = F64_NST;
constexpr int WARPS_M = BM / 32, WARPS_N = BN / 32, NTH = 32 * WARPS_M * WARPS_N;
// blocks per SM (at most 128 registers a thread for 512 / NTH)
#ifndef F64_BLOCKS
#define F64_BLOCKS (512 / NTH)
#endif
constexpr int BLOCKS = F64_BLOCKS;
// padded row strides (doubles) of the staged tiles
constexpr int SA_MK = BK + 2;   // A as [m][k] (FWD, DT)
constexpr int SA_KM = BM + 4;   // A as [k][m] (DW)
constexpr int SB_NK = BK + 2;   // B as [n][k] (FWD)
constexpr int SB_KN = BN + 4;   // B as [k][n] (DT, DW)
constexpr int A_WORDS = BK * SA_KM > BM * SA_MK ? BK * SA_KM : BM * SA_MK;
constexpr int B_WORDS = BN * SB_NK > BK * SB_KN ? BN * SB_NK : BK * SB_KN;
constexpr int STAGE_WORDS = A_WORDS + B_WORDS;
constexpr size_t SMEM = (size_t)NST * STAGE_WORDS * 8;
static_assert(8 * MI == 32 && 8 * NJ == 32 && (BN == 64 || BN == 128) && (BM == 64 || BM == 128),
              "warps of 32 x 32");
static_assert(A_WORDS % 2 == 0 && STAGE_WORDS % 2 == 0, "16-byte aligned tiles");
static_assert((BM * BK / 2) % NTH == 0 && (BN * BK / 2) % NTH == 0, "whole pieces per thread");

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
// not volatile: the products depend only on their operands, so the
// compiler may interleave them
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}
__device__ __forceinline__ double2 lds2(const double *p) { return *(const double2 *)p; }

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
  const double *bias;  // FWD: the weight rows (bias first, row length ldw)
  int ldw;
};

// the weight operand without its bias column, Wp[r][c] = W[r][1 + c] (W rows
// of ldw doubles): FWD reads it as [n][k], DT as [k][n]
__global__ void k_pack_w(const double *W, int ldw, int rows, int cols, double *Wp) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * cols) return;
  const int r = e / cols, c = e - r * cols;
  Wp[e] = W[(size_t)r * ldw + 1 + c];
}

// the shared row of DT's W row k of a k-block
__device__ __forceinline__ int dt_row(int k) { return 4 * (k & 3) + (k >> 2); }

// stage k-block [k0, k0 + BK) of tile (m0, n0) into stage buffer s
template <int MODE, bool PK>
__device__ __forceinline__ void load_stage(const F64Args &g, double *s, int m0, int n0, int k0,
                                           int kend) {
  double *sa = s, *sb = s + A_WORDS;
  const int t = threadIdx.x;
  if (MODE != MODE_F64_DW) {
    // A[m][k]: BM rows x 8 pieces of 16 bytes (K is even on every path here)
#pragma unroll
    for (int p = 0; p < BM * (BK / 2) / NTH; ++p) {
      const int e = t + p * NTH, r = e >> 3, kk = (e & 7) * 2;
      const int gm = m0 + r, gk = k0 + kk;
      const bool ok = gm < g.M && gk < kend;
      cp16(sa + r * SA_MK + kk, g.A + (ok ? (size_t)gm * g.lda + gk : 0), ok ? 16 : 0);
    }
    if (MODE == MODE_F64_FWD) {
      if (PK) {
        // packed Wp[n][k] (row length K)
#pragma unroll
        for (int p = 0; p < BN * (BK / 2) / NTH; ++p) {
          const int e = t + p * NTH, n = e >> 3, kk = (e & 7) * 2;
          const int gn = n0 + n, gk = k0 + kk;
          const bool ok = gn < g.N && gk < kend;
          cp16(sb + n * SB_NK + kk, g.B + (ok ? (size_t)gn * g.ldb + gk : 0), ok ? 16 : 0);
        }
      } else {
        // W[n][1 + k]: 8-byte pieces (the bias column breaks 16-byte alignment)
#pragma unroll
        for (int p = 0; p < BN * BK / NTH; ++p) {
          const int e = t + p * NTH, n = e / BK, kk = e % BK;
          const int gn = n0 + n, gk = k0 + kk;
          const bool ok = gn < g.N && gk < kend;
          cp8(sb + n * SB_NK + kk, g.B + (ok ? (size_t)gn * g.ldb + 1 + gk : 0), ok ? 8 : 0);
        }
      }
    } else if (PK) {
      // DT, packed Wp[k][n] (row length N, even)
#pragma unroll
      for (int p = 0; p < BK * (BN / 2) / NTH; ++p) {
        const int e = t + p * NTH, kk = e / (BN / 2), n = e % (BN / 2) * 2;
        const int gk = k0 + kk, gn = n0 + n;
        const bool ok = gk < kend && gn < g.N;
        cp16(sb + dt_row(kk) * SB_KN + n, g.B + (ok ? (size_t)gk * g.ldb + gn : 0), ok ? 16 : 0);
      }
    } else {
      // DT, W[k][1 + n]
#pragma unroll
      for (int p = 0; p < BK * BN / NTH; ++p) {
        const int e = t + p * NTH, kk = e / BN, n = e % BN;
        const int gk = k0 + kk, gn = n0 + n;
        const bool ok = gk < kend && gn < g.N;
        cp8(sb + dt_row(kk) * SB_KN + n, g.B + (ok ? (size_t)gk * g.ldb + 1 + gn : 0), ok ? 8 : 0);
      }
    }
  } else {
    // A[r][j] rows r = k0.. as [k][m]; B[r][i] as [k][n]; 16-byte pieces
#pragma unroll
    for (int p = 0; p < BK * (BM / 2) / NTH; ++p) {
      const int e = t + p * NTH, kk = e / (BM / 2), m = e % (BM / 2) * 2;
      const int gk = k0 + kk, gm = m0 + m;
      const bool ok = gk < kend && gm < g.M;
      cp16(sa + kk * SA_KM + m, g.A + (ok ? (size_t)gk * g.lda + gm : 0), ok ? 16 : 0);
    }
#pragma unroll
    for (int p = 0; p < BK * (BN / 2) / NTH; ++p) {
      const int e = t + p * NTH, kk = e / (BN / 2), n = e % (BN / 2) * 2;
      const int gk = k0 + kk, gn = n0 + n;
      const bool ok = gk < kend && gn < g.N;
      cp16(sb + kk * SB_KN + n, g.B + (ok ? (size_t)gk * g.ldb + gn : 0), ok ? 16 : 0);
    }
  }
}

// one k-block of products from a stage into the warp's 4 x 4 fragments
template <int MODE>
__device__ __forceinline__ void compute_stage(const double *s, int wm, int wn, int lane,
                                              double (&acc)[MI][NJ][2]) {
  const double *sa = s, *sb = s + A_WORDS;
  const int r8 = lane >> 2, c4 = lane & 3;
  if (MODE == MODE_F64_DW) {
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      const double *pa = sa + (4 * ks + c4) * SA_KM + wm + 2 * r8;
      const double *pb = sb + (4 * ks + c4) * SB_KN + wn + 2 * r8;
      double a[MI], b[NJ];
#pragma unroll
      for (int ii = 0; ii < MI / 2; ++ii) {
        const double2 v = lds2(pa + 16 * ii);
        a[2 * ii] = v.x;
        a[2 * ii + 1] = v.y;
      }
#pragma unroll
      for (int jj = 0; jj < NJ / 2; ++jj) {
        const double2 v = lds2(pb + 16 * jj);
        b[2 * jj] = v.x;
        b[2 * jj + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma(acc[i][j], a[i], b[j]);
    }
  } else {
    // k = 4 c4 + ks: half h holds k-steps 2h and 2h + 1 in one 16-byte load
#pragma unroll
    for (int h = 0; h < BK / 8; ++h) {
      double2 a[MI];
#pragma unroll
      for (int i = 0; i < MI; ++i) a[i] = lds2(sa + (wm + 8 * i + r8) * SA_MK + 4 * c4 + 2 * h);
#ifdef F64_FWD_ALLB
      if (MODE == MODE_F64_FWD) {
        double2 bf[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) bf[j] = lds2(sb + (wn + 8 * j + r8) * SB_NK + 4 * c4 + 2 * h);
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
          for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j) dmma(acc[i][j], e ? a[i].y : a[i].x, e ? bf[j].y : bf[j].x);
      } else
#endif
      if (MODE == MODE_F64_FWD) {
        // one B fragment pair at a time: both k-steps of fragment j
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
          const double2 b = lds2(sb + (wn + 8 * j + r8) * SB_NK + 4 * c4 + 2 * h);
#pragma unroll
          for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int i = 0; i < MI; ++i) dmma(acc[i][j], e ? a[i].y : a[i].x, e ? b.y : b.x);
        }
      } else {
        // one pair of B fragments (2 jj, 2 jj + 1) of one k-step at a time
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const double *pb = sb + (4 * (2 * h + e) + c4) * SB_KN + wn + 2 * r8;
#pragma unroll
          for (int jj = 0; jj < NJ / 2; ++jj) {
            const double2 b = lds2(pb + 16 * jj);
#pragma unroll
            for (int i = 0; i < MI; ++i) {
              dmma(acc[i][2 * jj], e ? a[i].y : a[i].x, b.x);
              dmma(acc[i][2 * jj + 1], e ? a[i].y : a[i].x, b.y);
            }
          }
        }
      }
    }
  }
}

// a run of four output columns n .. n + 3 (DT, DW: fragments 2 jj and 2 jj + 1)
__device__ __forceinline__ void store4(const F64Args &g, double *c, int n, double v0, double v1,
                                       double v2, double v3) {
  if (g.cvec && n + 3 < g.N) {  // n is even
    *(double2 *)c = make_double2(v0, v1);
    *(double2 *)(c + 2) = make_double2(v2, v3);
  } else {
    if (n < g.N) c[0] = v0;
    if (n + 1 < g.N) c[1] = v1;
    if (n + 2 < g.N) c[2] = v2;
    if (n + 3 < g.N) c[3] = v3;
  }
}

// FWD/DT: write one finished 128 x BN tile (rows from m0) of the warp's fragments
template <int MODE>
__device__ __forceinline__ void epilogue_fd(const F64Args &g, const double (&acc)[MI][NJ][2],
                                            int m0, int n0, int wm, int wn, int r8, int c4) {
  if (MODE == MODE_F64_FWD) {
    // rows m0 + wm + 8 i + r8, columns n0 + wn + 8 j + 2 c4 (+0, +1); the
    // bias goes to the rows m % na == 0, the first at offset off0
    const int rem = m0 % g.na, off0 = rem ? g.na - rem : 0;
#pragma unroll
    for (int i = 0; i < MI; ++i) {
      const int off = wm + 8 * i + r8, m = m0 + off;
      if (m >= g.M) continue;
      const bool brow =
          g.na >= BM ? off == off0 : off >= off0 && (off - off0) % g.na == 0;
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int n = n0 + wn + 8 * j + 2 * c4;
        double v0 = acc[i][j][0], v1 = acc[i][j][1];
        if (brow) {
          if (n < g.N) v0 += g.bias[(size_t)n * g.ldw];
          if (n + 1 < g.N) v1 += g.bias[(size_t)(n + 1) * g.ldw];
        }
        double *c = g.C + (size_t)m * g.ldc + n;
        if (g.cvec && n + 1 < g.N) {
          *(double2 *)c = make_double2(v0, v1);
        } else {
          if (n < g.N) c[0] = v0;
          if (n + 1 < g.N) c[1] = v1;
        }
      }
    }
  } else {
    // rows m0 + wm + 8 i + r8; fragments 2 jj, 2 jj + 1 hold columns
    // n0 + wn + 16 jj + 4 c4 + (0, 2) and (1, 3)
#pragma unroll
    for (int i = 0; i < MI; ++i) {
      const int m = m0 + wm + 8 * i + r8;
      if (m >= g.M) continue;
#pragma unroll
      for (int jj = 0; jj < NJ / 2; ++jj) {
        const int n = n0 + wn + 16 * jj + 4 * c4;
        store4(g, g.C + (size_t)m * g.ldc + n, n, acc[i][2 * jj][0], acc[i][2 * jj + 1][0],
               acc[i][2 * jj][1], acc[i][2 * jj + 1][1]);
      }
    }
  }
}

template <int MODE, bool PK>
__global__ void __launch_bounds__(NTH, BLOCKS) k_gemm_f64(F64Args g) {
  extern __shared__ __align__(16) double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp % WARPS_M) * 32, wn = (warp / WARPS_M) * 32;
  const int n0 = blockIdx.y * BN;
  const int r8 = lane >> 2, c4 = lane & 3;
  if (MODE != MODE_F64_DW) {
    // this block's M tiles blockIdx.x, + gridDim.x, ...; one cp.async ring
    // runs through all their k-blocks, so no tile waits for its ring to fill
    const int tiles = (g.M + BM - 1) / BM;
    const int nkb = (g.K + BK - 1) / BK;
    const int mine = blockIdx.x < tiles ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    int it = 0, ikb = 0, wslot = 0;  // the next k-block to stage and its ring slot
    auto issue = [&]() {
      if (it < mine) {
        load_stage<MODE, PK>(g, sm + wslot * STAGE_WORDS, (blockIdx.x + it * gridDim.x) * BM, n0,
                         ikb * BK, g.K);
        if (++ikb == nkb) {
          ikb = 0;
          ++it;
        }
      }
      commit();
      wslot = wslot == NST - 1 ? 0 : wslot + 1;
    };
#pragma unroll
    for (int s = 0; s < NST - 1; ++s) issue();
    int rslot = 0;
    auto mrow = [&](int t) { return (blockIdx.x + t * gridDim.x) * BM; };
    // the k-blocks of tile t into acc
    auto run_tile = [&](double (&acc)[MI][NJ][2], int t) {
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
      for (int kb = 0; kb < nkb; ++kb) {
        wait_group<NST - 2>();
        __syncthreads();  // this k-block is in; every warp is done with the previous one
        issue();
        compute_stage<MODE>(sm + rslot * STAGE_WORDS, wm, wn, lane, acc);
        rslot = rslot == NST - 1 ? 0 : rslot + 1;
      }
    };
    for (int t = 0; t < mine; ++t) {
      double acc[MI][NJ][2];
      run_tile(acc, t);
      epilogue_fd<MODE>(g, acc, mrow(t), n0, wm, wn, r8, c4);
    }
    wait_group<0>();
  } else {
    // rows [r0, r1) of the reduction for output tile (blockIdx.z, blockIdx.y)
    const int m0 = blockIdx.z * BM;
    const int r0 = blockIdx.x * g.kper, r1 = min(g.K, r0 + g.kper);
    if (r0 >= r1) return;
    const int nkb = (r1 - r0 + BK - 1) / BK;
    double acc[MI][NJ][2];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    int ikb = 0, wslot = 0;
    auto issue = [&]() {
      if (ikb < nkb) load_stage<MODE, PK>(g, sm + wslot * STAGE_WORDS, m0, n0, r0 + ikb * BK, r1);
      ++ikb;
      commit();
      wslot = wslot == NST - 1 ? 0 : wslot + 1;
    };
#pragma unroll
    for (int s = 0; s < NST - 1; ++s) issue();
    int rslot = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      wait_group<NST - 2>();
      __syncthreads();
      issue();
      compute_stage<MODE>(sm + rslot * STAGE_WORDS, wm, wn, lane, acc);
      rslot = rslot == NST - 1 ? 0 : rslot + 1;
    }
    wait_group<0>();
    // rows m0 + wm + 16 (i >> 1) + 2 r8 + (i & 1); columns as DT
#pragma unroll
    for (int i = 0; i < MI; ++i) {
      const int m = m0 + wm + 16 * (i >> 1) + 2 * r8 + (i & 1);
      if (m >= g.M) continue;
#pragma unroll
      for (int jj = 0; jj < NJ / 2; ++jj) {
        const int n = n0 + wn + 16 * jj + 4 * c4;
        double *o = g.G + (size_t)m * g.gld + 1 + n;
        const double v[4] = {acc[i][2 * jj][0], acc[i][2 * jj + 1][0], acc[i][2 * jj][1],
                             acc[i][2 * jj + 1][1]};
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (n + q < g.N) atomicAdd(o + q, v[q]);
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

template <int MODE, bool PK>
void launch_f64(const char *name, dim3 grid, const F64Args &g, cudaStream_t st) {
  cudaFuncSetAttribute(k_gemm_f64<MODE, PK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)SMEM);
  LAUNCH(name, st, (k_gemm_f64<MODE, PK><<<grid, NTH, SMEM, st>>>(g)));
}

}  // namespace

int gemm_f64(int mode, int M, int N, int K, int na, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double *G, int gld, cudaStream_t st, double *pack) {
  // 16-byte pieces of A (and of B in DW) need even leading dimensions and
  // 16-byte aligned bases
  if ((lda & 1) || ((uintptr_t)A & 15) || (mode == MODE_F64_DW && ((ldb & 1) || ((uintptr_t)B & 15))) ||
      (mode != MODE_F64_DW && (K & 1)) || (mode == MODE_F64_DW && (M & 1 || N & 1)))
    return RC_UNSUPPORTED;
  F64Args g;
  g.M = M; g.N = N; g.K = K; g.na = na; g.A = A; g.lda = lda; g.B = B; g.ldb = ldb;
  g.C = C; g.ldc = ldc; g.G = G; g.gld = gld; g.kper = 0;
  g.cvec = C && ((uintptr_t)C & 15) == 0 && (ldc & 1) == 0;
  g.bias = B;
  g.ldw = ldb;
  // the weight operand packed without its bias column, so that it loads in
  // 16-byte pieces (DT needs an even N for that)
  bool pk = false;
  if (pack && ((uintptr_t)pack & 15) == 0 &&
      (mode == MODE_F64_FWD || (mode == MODE_F64_DT && (N & 1) == 0))) {
    const int rows = mode == MODE_F64_FWD ? N : K, cols = mode == MODE_F64_FWD ? K : N;
    const int tot = rows * cols;
    LAUNCH("k_pack_w", st, (k_pack_w<<<(tot + 255) / 256, 256, 0, st>>>(B, ldb, rows, cols, pack)));
    g.B = pack;
    g.ldb = mode == MODE_F64_FWD ? K : N;
    pk = true;
  }
  const int ntn = (N + BN - 1) / BN;
  cudaError_t e;
  if (mode == MODE_F64_FWD || mode == MODE_F64_DT) {
    const int tiles = (M + BM - 1) / BM;
    // one wave of persistent blocks
    const int gx = std::max(1, std::min(tiles, sms() * BLOCKS / std::max(1, ntn)));
    const dim3 grid(gx, ntn);
    if (mode == MODE_F64_FWD)
      pk ? launch_f64<MODE_F64_FWD, true>("k_gemm_f64_fwd", grid, g, st)
         : launch_f64<MODE_F64_FWD, false>("k_gemm_f64_fwd", grid, g, st);
    else
      pk ? launch_f64<MODE_F64_DT, true>("k_gemm_f64_dt", grid, g, st)
         : launch_f64<MODE_F64_DT, false>("k_gemm_f64_dt", grid, g, st);
  } else {
    // DW: output tiles (N tiles x M tiles), the row reduction split so that
    // about two blocks per SM run, each over a multiple of BK rows
    const int mt = (M + BM - 1) / BM;
    const int want = std::max(1, sms() * BLOCKS / std::max(1, ntn * mt));
    int kper = (K + want - 1) / want;
    kper = std::max(BK, (kper + BK - 1) / BK * BK);
    g.kper = kper;
    launch_f64<MODE_F64_DW, false>("k_gemm_f64_dw", dim3((K + kper - 1) / kper, ntn, mt), g, st);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("k_gemm_f64: ") + cudaGetErrorString(e));
    return RC_DEVICE;
  }
  return RC_OK;
}

}  // namespace dnnf90
