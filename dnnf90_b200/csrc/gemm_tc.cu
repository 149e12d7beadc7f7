// gemm_tc.cu - split-BF16 layer GEMMs on the tcgen05 tensor cores.
//
// Two kernels: k_tc_gemm for the products with the weights (FWD, DT) and the
// natural-gradient metric J^T J (its DW mode, gemm_tc_syrk), and k_tc_dw, the
// layers' weight gradient, fed by TMA (further below).
//
// k_tc_gemm: one persistent kernel, warp-specialised (FWD/DT 800 threads, DW 416):
//   producers  warps 0-15 (FWD/DT; 0-7 for DW): read FP32 operand rows from
//              HBM (coalesced 16-byte loads; FWD/DT keep the next two K
//              blocks in flight in registers), split every value x into three bf16 terms
//              x1 = bf16(x), x2 = bf16(x - x1), x3 = bf16(x - x1 - x2) and
//              store them in the 128-byte-swizzled canonical layout the
//              tensor core reads (one tile per term)
//   MMA warp   (the last) issuer: per 16-deep k-step six tcgen05.mma (kind::f16,
//              bf16 x bf16 -> FP32) for the cross terms of order <= 2:
//              a3b1, a2b2, a1b3, a2b1, a1b2, a1b1, smallest first, into an
//              accumulator in tensor memory (two buffers, so the epilogue of
//              one tile overlaps the products of the next)
//   epilogue   the warps after the producers (FWD/DT 8, two per tensor-memory
//              lane quadrant taking alternate 32-column boxes; DW 4):
//              tcgen05.ld of the accumulator (lane = row), bias
//              on the alpha = 0 rows, FP32 store; or, for the weight
//              gradient, FP32 partials of 512 rows added into FP64
//              registers and reduced to HBM with FP64 atomics
// Hand-offs are mbarriers: producer -> MMA (full), MMA -> producer (empty,
// through tcgen05.commit), MMA -> epilogue (tmem full), epilogue -> MMA
// (tmem empty).  Every wait is bounded; a wait that runs out sets a flag
// that the host reads after the launch, and the kernel returns.
//
// Modes:
//   FWD  S[M][N]  = A[M][K] W^T  (+ bias[N] on rows r % na == 0),
//        A = T_{l-1} plane (K-major), W pre-split and pre-swizzled
//   DT   Tb[M][N] = A[M][K] W    (A = Sb plane, K = n, N = m)
//   DW   G[j][1+i] += sum_r A[r][j] B[r][i]  (both MN-major tiles, K = rows
//        split across blocks): the metric J^T J (A = B = J)
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"
#include "gemm_tc.hpp"

namespace dnnf90 {

#define CKT(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));   \
      return e_ == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;   \
    }                                                                  \
  } while (0)

namespace tc {

constexpr int MODE_FWD = 0, MODE_DT = 1, MODE_DW = 2;
// Warp roles per mode: producers first, then 4 epilogue warps, then the MMA
// warp.  FWD/DT run 16 producer warps that keep two K blocks of loads in
// flight; DW keeps 8 (its epilogue holds 64 FP64 partials per thread).
template <int MODE>
struct Roles {
  static constexpr int PW = MODE == MODE_DW ? 8 : 16;  // producer warps
  static constexpr int EW = MODE == MODE_DW ? 4 : 8;   // epilogue warps
  static constexpr int NPROD = PW * 32;
  static constexpr int MMA = PW + EW;
  static constexpr int NT = (PW + EW + 1) * 32;
};
constexpr int BM = 128;       // rows per tile (MMA M)
constexpr int BK = 64;        // K per block: one 128-byte bf16 swizzle row
constexpr int ROWB = 128;     // bytes per swizzled row
constexpr long WAIT_LIMIT = 1L << 26;  // polls before a wait gives up (seconds)

__device__ __forceinline__ uint32_t su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t cnt) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(cnt) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(su32(b))
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t par) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(par)
      : "memory");
  return ok != 0;
}
// bounded wait; false (and the error flag set) when the limit runs out.
// The flag (a global read, an L2 round trip) is looked at once every 64
// polls, and the thread backs off only after 1024: a hand-off is seen
// within one try_wait of its phase completing.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t par, int *flag, int code) {
  for (long it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try(b, par)) return true;
    if ((it & 63) == 63 && *(volatile int *)flag) return false;
    if (it > 1024) __nanosleep(32);
  }
  atomicCAS(flag, 0, code);
  return false;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// smem matrix descriptor, SWIZZLE_128B, sm100 version bits
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version for sm_100
  d |= 2ull << 61;  // SWIZZLE_128B
  return d;
}
// instruction descriptor: kind::f16, A = B = bf16, D = f32, M = 128
__host__ __device__ constexpr uint32_t idesc(int n, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id,
                                    uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(b))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// the three bf16 terms of four FP32 values, packed two per word: x1 =
// bf16(x), x2 = bf16(x - x1), x3 = bf16(x - x1 - x2), rounded to nearest
// even two at a time (the residuals are exact in FP32)
__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) {
  return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ void split4(float4 x, uint2 &p1, uint2 &p2, uint2 &p3) {
  const __nv_bfloat162 a1 = __floats2bfloat162_rn(x.x, x.y), b1 = __floats2bfloat162_rn(x.z, x.w);
  const float2 fa = __bfloat1622float2(a1), fb = __bfloat1622float2(b1);
  float r0 = x.x - fa.x, r1 = x.y - fa.y, r2 = x.z - fb.x, r3 = x.w - fb.y;
  const __nv_bfloat162 a2 = __floats2bfloat162_rn(r0, r1), b2 = __floats2bfloat162_rn(r2, r3);
  const float2 ga = __bfloat1622float2(a2), gb = __bfloat1622float2(b2);
  r0 -= ga.x;
  r1 -= ga.y;
  r2 -= gb.x;
  r3 -= gb.y;
  const __nv_bfloat162 a3 = __floats2bfloat162_rn(r0, r1), b3 = __floats2bfloat162_rn(r2, r3);
  p1 = make_uint2(bf2_bits(a1), bf2_bits(b1));
  p2 = make_uint2(bf2_bits(a2), bf2_bits(b2));
  p3 = make_uint2(bf2_bits(a3), bf2_bits(b3));
}

// byte offset of (row, k) in a K-major SW128 tile of 8-row atoms
__device__ __forceinline__ uint32_t kmaj_off(int row, int k) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * ROWB + ((((k >> 3) ^ (row & 7)) & 7) << 4) +
                    (k & 7) * 2);
}
// byte offset of (mn, k) in an MN-major SW128 tile: atoms of 64 mn x 8 k,
// mn blocks LBO = 1024 apart, k atoms SBO = mnb * 1024 apart
__device__ __forceinline__ uint32_t mnmaj_off(int mn, int k, int mnb) {
  const int r = k & 7;
  return (uint32_t)((k >> 3) * mnb * 1024 + (mn >> 6) * 1024 + r * ROWB +
                    (((((mn >> 3) & 7) ^ r)) << 4) + (mn & 7) * 2);
}

struct Args {
  int mode;
  int M, N, K, na;
  const float *A;  // FWD/DT: [M][K]; DW: [K][Mdw] (Sb)
  const float *B;  // DW only: [K][Ndw] (T_{l-1})
  int lda, ldb;
  const uint8_t *W;     // FWD/DT: pre-split weights, [3][nkb][BN rows][128 B] per N tile
  const float *bias;    // FWD: [N]
  float *C;             // FWD/DT: [M][ldc]
  int ldc;
  double *G;            // DW: [Mdw][gld], column offset 1
  int gld;
  int BN;               // N per tile
  int ntn;              // N tiles
  int kchunk;           // DW: K blocks per TMEM partial
  int kblocks_per_cta;  // DW: K blocks per block of the grid
  int gcol0;            // DW: first column of G written (1 past the bias column, or 0)
  int *flag;            // wait time-out / error flag
};

// FWD/DT epilogue staging: per epilogue warp one 32 x 32 FP32 box, rows of
// 128 bytes with the 16-byte pieces in the 128-byte swizzle the tensor map
// of C names, stored to HBM by one TMA bulk tensor store per box
constexpr int STG_BYTES = 8 * 32 * 32 * 4;

template <int MODE>
__global__ void __launch_bounds__(Roles<MODE>::NT, 1)
    k_tc_gemm(Args g, const __grid_constant__ CUtensorMap cmap) {
  constexpr int NPROD_WARPS = Roles<MODE>::PW, NPROD = Roles<MODE>::NPROD;
  constexpr int MMA_WARP = Roles<MODE>::MMA;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int BN = g.BN;
  const int nkb = (MODE == MODE_DW) ? 0 : (g.K + BK - 1) / BK;
  // ---- shared memory layout
  // FWD/DT: [B resident: 3 * nkb * BN * 128][stages: NST * 3 * 128 * 128]
  // DW:     [stages: NST * (3 * 8*2*1024 (A, 64 k x 128 mn) + 3 * 8*mnbB*1024 (B))]
  const int mnbB = (MODE == MODE_DW) ? (BN + 63) / 64 : 0;
  const uint32_t a_tile = (MODE == MODE_DW) ? 8 * 2 * 1024 : BM * ROWB;      // one term
  const uint32_t b_tile = (MODE == MODE_DW) ? 8 * mnbB * 1024 : BN * ROWB;   // one term
  const uint32_t stage_bytes = (MODE == MODE_DW) ? 3 * (a_tile + b_tile) : 3 * a_tile;
  const uint32_t bres = (MODE == MODE_DW) ? 0 : 3 * nkb * b_tile;
  const int NST = (MODE == MODE_DW) ? 3 : 2;
  uint8_t *sB = sm;
  uint8_t *sStage = sm + bres;
  uint64_t *bars = (uint64_t *)(sStage + NST * stage_bytes);
  uint64_t *full = bars, *empty = bars + NST, *tfull = bars + 2 * NST, *tempty = bars + 2 * NST + 2;
  uint32_t *tmem_hold = (uint32_t *)(bars + 2 * NST + 4);
  // FWD/DT: epilogue staging, 1024-aligned after the barriers
  uint8_t *sStg = sStage + NST * stage_bytes + 1024;

  const int ntn = g.ntn;
  const int tn = blockIdx.y;  // N tile of this block
  const int n0 = tn * BN;
  const int m0 = (MODE == MODE_DW) ? blockIdx.z * BM : 0;  // DW: output-row tile
  // tile sequence of this block
  int tiles_m = 0, first_m = 0, step_m = 1, kb_begin = 0, kb_end = 0;
  if (MODE == MODE_DW) {
    const int nkb_all = (g.K + BK - 1) / BK;
    kb_begin = blockIdx.x * g.kblocks_per_cta;
    kb_end = min(nkb_all, kb_begin + g.kblocks_per_cta);
  } else {
    tiles_m = (g.M + BM - 1) / BM;
    first_m = blockIdx.x;
    step_m = gridDim.x;
  }
  (void)ntn;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(full + s, NPROD);
      mbar_init(empty + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull + b, 1);
      mbar_init(tempty + b, Roles<MODE>::EW * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  const uint32_t tcols = (MODE == MODE_DW) ? 128u : (BN <= 64 ? 128u : 256u);
  if (warp == MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_hold)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // resident weights (FWD/DT): copied once by the producers
  if (MODE != MODE_DW && warp < NPROD_WARPS) {
    const uint4 *src = (const uint4 *)(g.W + (size_t)tn * bres);
    uint4 *dst = (uint4 *)sB;
    for (int i = threadIdx.x; i < (int)(bres / 16); i += NPROD) dst[i] = src[i];
    fence_proxy_async();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_hold;
  int *flag = g.flag;

  if (warp < NPROD_WARPS) {
    // ------------------------------------------------------------ producers
    // Every global load of the next K block is issued before the current
    // block is split and stored, so two blocks of loads are in flight.
    const int t = threadIdx.x;  // 0..NPROD-1
    int stage = 0;
    uint32_t ph = 0;
    auto next_stage = [&]() {
      if (++stage == NST) { stage = 0; ph ^= 1u; }
    };
    if (MODE != MODE_DW) {
      constexpr int PF = BM * BK / 4 / NPROD;  // float4 per thread per block
      auto load = [&](float4 *v, int mt, int kb) {
        const int k0 = kb * BK;
#pragma unroll
        for (int it = 0; it < PF; ++it) {
          const int e = it * NPROD + t;
          const int row = e >> 4, c4 = e & 15;
          const int gr = mt * BM + row, gk = k0 + c4 * 4;
          v[it] = (gr < g.M && gk < g.K) ? __ldg((const float4 *)(g.A + (size_t)gr * g.lda + gk))
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      };
      // split one block into the next free stage
      auto consume = [&](const float4 (&v)[PF]) -> bool {
        if (!mbar_wait(empty + stage, ph ^ 1u, flag, 1)) return false;
        uint8_t *st = sStage + stage * stage_bytes;
#pragma unroll
        for (int it = 0; it < PF; ++it) {
          const int e = it * NPROD + t;
          const int row = e >> 4, c4 = e & 15;
          uint2 p1, p2, p3;
          split4(v[it], p1, p2, p3);
          const uint32_t off = kmaj_off(row, c4 * 4);
          *(uint2 *)(st + off) = p1;
          *(uint2 *)(st + a_tile + off) = p2;
          *(uint2 *)(st + 2 * a_tile + off) = p3;
        }
        fence_proxy_async();
        mbar_arrive(full + stage);
        next_stage();
        return true;
      };
      // blocks (M tile, K block) in order; b0/b1/b2 rotate roles so that the
      // loads of the two blocks after the one being split are in flight
      int pm0 = first_m, pk0 = 0, pm1 = pm0, pk1 = 1, pm2, pk2;
      if (pk1 == nkb) { pk1 = 0; pm1 += step_m; }
      pm2 = pm1; pk2 = pk1 + 1;
      if (pk2 == nkb) { pk2 = 0; pm2 += step_m; }
      auto rotate = [&]() {
        pm0 = pm1; pk0 = pk1; pm1 = pm2; pk1 = pk2;
        if (++pk2 == nkb) { pk2 = 0; pm2 += step_m; }
      };
      float4 b0[PF], b1[PF], b2[PF];
      if (pm0 < tiles_m) load(b0, pm0, pk0);
      if (pm1 < tiles_m) load(b1, pm1, pk1);
      for (;;) {
        if (pm0 >= tiles_m) break;
        if (pm2 < tiles_m) load(b2, pm2, pk2);
        if (!consume(b0)) goto done;
        rotate();
        if (pm0 >= tiles_m) break;
        if (pm2 < tiles_m) load(b0, pm2, pk2);
        if (!consume(b1)) goto done;
        rotate();
        if (pm0 >= tiles_m) break;
        if (pm2 < tiles_m) load(b1, pm2, pk2);
        if (!consume(b2)) goto done;
        rotate();
      }
    } else {
      // A: 64 rows x 128 j of Sb (32 threads per row); B: 64 rows x 64 i
      // of T_{l-1} (16 threads per row)
      constexpr int PA = 64 * 32 / NPROD, PB = 64 * 16 / NPROD;
      const int Mdw = g.M;
      auto load = [&](float4 *va, float4 *vb, int kb) {
        const int r0 = kb * BK;
#pragma unroll
        for (int it = 0; it < PA; ++it) {
          const int e = it * NPROD + t;
          const int kr = e >> 5, j = (e & 31) * 4;
          const int gr = r0 + kr;
          va[it] = (gr < g.K && m0 + j < Mdw)
                       ? __ldg((const float4 *)(g.A + (size_t)gr * g.lda + m0 + j))
                       : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int it = 0; it < PB; ++it) {
          const int e = it * NPROD + t;
          const int kr = e >> 4, i = n0 + (e & 15) * 4;
          const int gr = r0 + kr;
          vb[it] = (gr < g.K && i < g.N) ? __ldg((const float4 *)(g.B + (size_t)gr * g.ldb + i))
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
        }
      };
      float4 ca[PA], cb[PB], na_[PA], nb_[PB];
      if (kb_begin < kb_end) load(ca, cb, kb_begin);
      for (int kb = kb_begin; kb < kb_end; ++kb) {
        if (kb + 1 < kb_end) load(na_, nb_, kb + 1);
        if (!mbar_wait(empty + stage, ph ^ 1u, flag, 1)) goto done;
        uint8_t *st = sStage + stage * stage_bytes;
        uint8_t *sb = st + 3 * a_tile;
#pragma unroll
        for (int it = 0; it < PA; ++it) {
          const int e = it * NPROD + t;
          const int kr = e >> 5, j = (e & 31) * 4;
          uint2 p1, p2, p3;
          split4(ca[it], p1, p2, p3);
          const uint32_t off = mnmaj_off(j, kr, 2);
          *(uint2 *)(st + off) = p1;
          *(uint2 *)(st + a_tile + off) = p2;
          *(uint2 *)(st + 2 * a_tile + off) = p3;
        }
#pragma unroll
        for (int it = 0; it < PB; ++it) {
          const int e = it * NPROD + t;
          const int kr = e >> 4, il = (e & 15) * 4;
          uint2 p1, p2, p3;
          split4(cb[it], p1, p2, p3);
          const uint32_t off = mnmaj_off(il, kr, mnbB);
          *(uint2 *)(sb + off) = p1;
          *(uint2 *)(sb + b_tile + off) = p2;
          *(uint2 *)(sb + 2 * b_tile + off) = p3;
        }
        fence_proxy_async();
        mbar_arrive(full + stage);
        next_stage();
#pragma unroll
        for (int it = 0; it < PA; ++it) ca[it] = na_[it];
#pragma unroll
        for (int it = 0; it < PB; ++it) cb[it] = nb_[it];
      }
    }
  } else if (warp == MMA_WARP) {
    // ------------------------------------------------------------ MMA issuer
    int stage = 0;
    uint32_t ph = 0;
    auto next_stage = [&]() {
      if (++stage == NST) { stage = 0; ph ^= 1u; }
    };
    // term pairs, smallest first: (a3,b1) (a2,b2) (a1,b3) (a2,b1) (a1,b2) (a1,b1)
    const int pa[6] = {2, 1, 0, 1, 0, 0};
    const int pb[6] = {0, 1, 2, 0, 1, 0};
    if (MODE != MODE_DW) {
      const uint32_t id = idesc(BN, 0, 0);
      int buf = 0;
      uint32_t tph = 0;
      for (int mt = first_m; mt < tiles_m; mt += step_m) {
        if (!mbar_wait(tempty + buf, tph ^ 1u, flag, 2)) goto done;
        tc_fence_after();
        const uint32_t dcol = tmem + (uint32_t)(buf * BN);
        for (int kb = 0; kb < nkb; ++kb) {
          if (!mbar_wait(full + stage, ph, flag, 3)) goto done;
          tc_fence_after();
          if (lane == 0) {
            const uint32_t sa = su32(sStage + stage * stage_bytes);
            const uint32_t sbb = su32(sB);
            const int ksteps = min(BK, g.K - kb * BK) / 16;
            for (int ks = 0; ks < ksteps; ++ks) {
#pragma unroll
              for (int p = 0; p < 6; ++p) {
                const uint64_t ad = sdesc(sa + pa[p] * a_tile + ks * 32, 16, 1024);
                const uint64_t bd =
                    sdesc(sbb + (pb[p] * nkb + kb) * b_tile + ks * 32, 16, 1024);
                mma(dcol, ad, bd, id, (kb | ks | p) ? 1u : 0u);
              }
            }
            mma_commit(empty + stage);
          }
          __syncwarp();
          next_stage();
        }
        if (lane == 0) mma_commit(tfull + buf);
        __syncwarp();
        if (++buf == 2) { buf = 0; tph ^= 1u; }
      }
    } else {
      const uint32_t id = idesc(BN, 1, 1);
      int buf = 0;
      uint32_t tph = 0;
      int inchunk = 0;
      for (int kb = kb_begin; kb < kb_end; ++kb) {
        if (inchunk == 0) {
          if (!mbar_wait(tempty + buf, tph ^ 1u, flag, 2)) goto done;
          tc_fence_after();
        }
        if (!mbar_wait(full + stage, ph, flag, 3)) goto done;
        tc_fence_after();
        if (lane == 0) {
          const uint32_t sa = su32(sStage + stage * stage_bytes);
          const uint32_t sbb = sa + 3 * a_tile;
          const uint32_t dcol = tmem + (uint32_t)(buf * 64);
#pragma unroll
          for (int ks = 0; ks < BK / 16; ++ks) {
#pragma unroll
            for (int p = 0; p < 6; ++p) {
              // one 16-deep step spans two 8-row k atoms
              const uint64_t ad = sdesc(sa + pa[p] * a_tile + ks * 2 * (2 * 1024), 1024, 2 * 1024);
              const uint64_t bd =
                  sdesc(sbb + pb[p] * b_tile + ks * 2 * (mnbB * 1024), 1024, mnbB * 1024);
              mma(dcol, ad, bd, id, (inchunk | ks | p) ? 1u : 0u);
            }
          }
          mma_commit(empty + stage);
        }
        __syncwarp();
        next_stage();
        if (++inchunk == g.kchunk || kb + 1 == kb_end) {
          if (lane == 0) mma_commit(tfull + buf);
          __syncwarp();
          inchunk = 0;
          if (++buf == 2) { buf = 0; tph ^= 1u; }
        }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;           // TMEM lane quadrant of this warp
    const int row = q * 32 + lane;    // accumulator row = TMEM lane
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    if (MODE != MODE_DW) {
      int buf = 0;
      uint32_t tph = 0;
      for (int mt = first_m; mt < tiles_m; mt += step_m) {
        if (!mbar_wait(tfull + buf, tph, flag, 4)) goto done;
        tc_fence_after();
        const int gr = mt * BM + row;
        const bool ok = gr < g.M;
        const bool brow = (MODE == MODE_FWD) && ok && (gr % g.na == 0);
        // the two warps of a lane quadrant take alternate 32-column boxes,
        // each through its own staging box
        uint8_t *stg = sStg + (warp - NPROD_WARPS) * (32 * 32 * 4);
        for (int c0 = 32 * ((warp - NPROD_WARPS) >> 2); c0 < BN; c0 += 64) {
          float v[32];
          tmem_ld32(lane_addr + (uint32_t)(buf * BN + c0), v);
          if (brow) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
              if (n0 + c0 + i < g.N) v[i] += g.bias[n0 + c0 + i];
          }
          // the previous store of this box has read the staging
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 8; ++j)
            *(float4 *)(stg + lane * 128 + ((j ^ (lane & 7)) << 4)) =
                make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            // rows past M and columns past N are clipped by the tensor map
            asm volatile(
                "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    &cmap),
                "r"(n0 + c0), "r"(mt * BM + q * 32), "r"(su32(stg))
                : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          }
        }
        tc_fence_before();
        mbar_arrive(tempty + buf);
        if (++buf == 2) { buf = 0; tph ^= 1u; }
      }
    } else {
      double acc[64];
#pragma unroll
      for (int i = 0; i < 64; ++i) acc[i] = 0.0;
      int buf = 0;
      uint32_t tph = 0;
      const int nch = (kb_end - kb_begin + g.kchunk - 1) / g.kchunk;
      for (int ch = 0; ch < nch; ++ch) {
        if (!mbar_wait(tfull + buf, tph, flag, 4)) goto done;
        tc_fence_after();
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 32) {
          float v[32];
          tmem_ld32(lane_addr + (uint32_t)(buf * 64 + c0), v);
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[c0 + i] += (double)v[i];
        }
        tc_fence_before();
        mbar_arrive(tempty + buf);
        if (++buf == 2) { buf = 0; tph ^= 1u; }
      }
      if (m0 + row < g.M && nch > 0) {
        double *dst = g.G + (size_t)(m0 + row) * g.gld + g.gcol0 + n0;
#pragma unroll
        for (int i = 0; i < 64; ++i)
          if (n0 + i < g.N) atomicAdd(dst + i, acc[i]);
      }
    }
  }
done:
  if (MODE != MODE_DW && warp >= NPROD_WARPS && warp < MMA_WARP && lane == 0)
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // epilogue stores complete
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == MMA_WARP)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols)
                 : "memory");
}

// ---------------------------------------------------------------- DW by TMA
// G[j][gcol0 + i] += sum_r A[r][j] B[r][i] (A = Sb [K][Mdw], B = T_{l-1}
// [K][Ndw], FP32), one 128 x 128 output tile per block, the rows split
// across the grid.  Warp roles:
//   warp 0      TMA: one 2-D box of 32 rows x up to 128 columns of A and
//               of B per block of rows into a raw FP32 ring (3 stages)
//   warps 1-16  converters: split the raw values into three bf16 terms in
//               the MN-major 128-byte-swizzled layout (2 stages), two
//               16-byte pieces of each operand per thread
//   warp 17     MMA: per block two 16-deep steps of the six cross terms of
//               order <= 2 into an FP32 accumulator in tensor memory (two
//               buffers of 128 columns)
//   warps 18-21 epilogue: every 16 blocks (512 rows) the FP32 partial is
//               added into an FP64 accumulator kept in tensor memory
//               (columns 256-511, two cells per value), which is added into
//               G with FP64 atomics at the end
// Every wait is bounded; one that runs out sets the error flag, and every
// role then waits (bounded) for its own copies and products in flight.
constexpr int DW_RB = 32;           // rows per block
constexpr int DW_NR = 3;            // raw stages
constexpr int DW_NT = 2;            // term stages
constexpr int DW_CHUNK = 16;        // blocks per FP32 partial
constexpr int DW_CONV = 16;         // converter warps
constexpr int DW_W_MMA = 1 + DW_CONV, DW_W_EPI = DW_W_MMA + 1, DW_WARPS = DW_W_EPI + 4;
constexpr int DW_NTH = DW_WARPS * 32;
constexpr uint32_t DW_RAW = 2 * DW_RB * 128 * 4;   // A and B boxes
constexpr uint32_t DW_TT = DW_RB * 128 * 2;        // one bf16 term of one operand
constexpr uint32_t DW_TERM = 6 * DW_TT;
constexpr size_t DW_SMEM = 1024 + DW_NR * DW_RAW + DW_NT * DW_TERM + 256;

struct DwArgs {
  int Mdw, Ndw, K;       // output rows (A columns), output columns (B columns), rows reduced
  int bwa, bwb;          // box widths: min(128, Mdw), min(128, Ndw)
  int kb_per_cta;        // blocks of DW_RB rows per block of the grid
  double *G;
  int gld, gcol0;
  int *flag;
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
// 2-D tiled TMA load into this block's own shared memory, completing on mbarrier b
__device__ __forceinline__ void tma_load2(void *dst, const CUtensorMap *m, int x, int y,
                                          uint64_t *b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(su32(dst)),
      "l"(m), "r"(x), "r"(y), "r"(su32(b))
      : "memory");
}
__device__ __forceinline__ void tmem_ld32u(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16u(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_st32u(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
      "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
      "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// bounded wait for copies or products still in flight, whatever the flag
// says (the wait that gives up sets the flag; this one only ends)
__device__ __forceinline__ void mbar_drain(uint64_t *b, uint32_t par) {
  for (long it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try(b, par)) return;
    if (it > 64) __nanosleep(64);
  }
}
// mbar_wait agreed across the warp, for warps whose next steps are
// warp-collective (tcgen05.ld / st, __syncwarp)
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *b, uint32_t par, int *flag, int code) {
  return __all_sync(0xffffffffu, mbar_wait(b, par, flag, code));
}
// add 16 FP32 partials p into the 16 FP64 values held as (low, high) word
// pairs in d (zero first when fresh)
__device__ __forceinline__ void add16(uint32_t (&d)[32], const uint32_t (&p)[16], bool fresh) {
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const double x = (fresh ? 0.0 : __hiloint2double((int)d[2 * i + 1], (int)d[2 * i])) +
                     (double)__uint_as_float(p[i]);
    d[2 * i] = (uint32_t)__double2loint(x);
    d[2 * i + 1] = (uint32_t)__double2hiint(x);
  }
}

__global__ void __launch_bounds__(DW_NTH, 1)
    k_tc_dw(DwArgs g, const __grid_constant__ CUtensorMap amap,
            const __grid_constant__ CUtensorMap bmap) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *sm = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sRaw = sm, *sTerm = sm + DW_NR * DW_RAW;
  uint64_t *bars = (uint64_t *)(sTerm + DW_NT * DW_TERM);
  uint64_t *rfull = bars, *rempty = bars + DW_NR, *tfull_s = bars + 2 * DW_NR,
           *tempty_s = bars + 2 * DW_NR + DW_NT, *afull = bars + 2 * DW_NR + 2 * DW_NT,
           *aempty = afull + 2, *fin = afull + 4;
  uint32_t *tmem_hold = (uint32_t *)(fin + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tn = blockIdx.y, tm = blockIdx.z;  // output tile: A columns tm*128.., B columns tn*128..
  const int nkb_all = (g.K + DW_RB - 1) / DW_RB;
  const int kb0 = blockIdx.x * g.kb_per_cta;
  const int nb = max(0, min(nkb_all, kb0 + g.kb_per_cta) - kb0);
  const int nch = (nb + DW_CHUNK - 1) / DW_CHUNK;
  const int mnbB = (g.bwb + 63) / 64;
  int *flag = g.flag;
  if (threadIdx.x == 0) {
    for (int s = 0; s < DW_NR; ++s) {
      mbar_init(rfull + s, 1);
      mbar_init(rempty + s, DW_CONV * 32);
    }
    for (int s = 0; s < DW_NT; ++s) {
      mbar_init(tfull_s + s, DW_CONV * 32);
      mbar_init(tempty_s + s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(afull + b, 1);
      mbar_init(aempty + b, 128);
    }
    mbar_init(fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == DW_W_MMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     su32(tmem_hold))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_hold;

  if (warp == 0) {
    // ------------------------------------------------------------ TMA
    int issued = 0;
    if (lane == 0) {
      const uint32_t bytes = (uint32_t)DW_RB * (g.bwa + g.bwb) * 4;
      for (int i = 0; i < nb; ++i) {
        const int s = i % DW_NR;
        const uint32_t ph = (uint32_t)(i / DW_NR) & 1u;
        if (!mbar_wait(rempty + s, ph ^ 1u, flag, 11)) break;
        mbar_expect_tx(rfull + s, bytes);
        uint8_t *dst = sRaw + s * DW_RAW;
        const int y = (kb0 + i) * DW_RB;
        tma_load2(dst, &amap, tm * 128, y, rfull + s);
        tma_load2(dst + DW_RB * g.bwa * 4, &bmap, tn * 128, y, rfull + s);
        issued = i + 1;
      }
      // the copies still in flight land before the block exits
      for (int i = max(0, issued - DW_NR); i < issued; ++i)
        mbar_drain(rfull + i % DW_NR, (uint32_t)(i / DW_NR) & 1u);
    }
    __syncwarp();
  } else if (warp < DW_W_MMA) {
    // ------------------------------------------------------------ converters
    // piece e = t + 512 p of an operand: row e / 32, columns 4 (e % 32) ..
    // + 3 of the box (rows of bw floats), present when they lie inside it
    const int t = threadIdx.x - 32;  // 0 .. 511
    static_assert(DW_CONV * 32 * 2 == DW_RB * 32, "two pieces of each operand per thread");
    for (int i = 0; i < nb; ++i) {
      const int s = i % DW_NR, ts = i % DW_NT;
      if (!mbar_wait(rfull + s, (uint32_t)(i / DW_NR) & 1u, flag, 13)) break;
      if (!mbar_wait(tempty_s + ts, ((uint32_t)(i / DW_NT) & 1u) ^ 1u, flag, 14)) break;
      const uint8_t *ra = sRaw + s * DW_RAW, *rb = ra + DW_RB * g.bwa * 4;
      uint8_t *ta = sTerm + ts * DW_TERM, *tb = ta + 3 * DW_TT;
      float4 xa[2], xb[2];
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const int e = t + p * DW_CONV * 32, kr = e >> 5, j = (e & 31) * 4;
        if (j < g.bwa) xa[p] = *(const float4 *)(ra + (kr * g.bwa + j) * 4);
        if (j < g.bwb) xb[p] = *(const float4 *)(rb + (kr * g.bwb + j) * 4);
      }
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const int e = t + p * DW_CONV * 32, kr = e >> 5, j = (e & 31) * 4;
        uint2 p1, p2, p3;
        if (j < g.bwa) {
          split4(xa[p], p1, p2, p3);
          const uint32_t off = mnmaj_off(j, kr, 2);
          *(uint2 *)(ta + off) = p1;
          *(uint2 *)(ta + DW_TT + off) = p2;
          *(uint2 *)(ta + 2 * DW_TT + off) = p3;
        }
        if (j < g.bwb) {
          split4(xb[p], p1, p2, p3);
          const uint32_t off = mnmaj_off(j, kr, mnbB);
          *(uint2 *)(tb + off) = p1;
          *(uint2 *)(tb + DW_TT + off) = p2;
          *(uint2 *)(tb + 2 * DW_TT + off) = p3;
        }
      }
      fence_proxy_async();
      mbar_arrive(tfull_s + ts);
      mbar_arrive(rempty + s);
    }
  } else if (warp == DW_W_MMA) {
    // ------------------------------------------------------------ MMA issuer
    const int pa[6] = {2, 1, 0, 1, 0, 0};
    const int pb[6] = {0, 1, 2, 0, 1, 0};
    const uint32_t id = idesc(g.bwb, 1, 1);
    bool any = false;
    for (int i = 0; i < nb; ++i) {
      const int ts = i % DW_NT, ic = i % DW_CHUNK, buf = (i / DW_CHUNK) & 1;
      if (ic == 0 &&
          !mbar_wait_warp(aempty + buf, ((uint32_t)(i / DW_CHUNK / 2) & 1u) ^ 1u, flag, 15))
        break;
      if (!mbar_wait_warp(tfull_s + ts, (uint32_t)(i / DW_NT) & 1u, flag, 16)) break;
      tc_fence_after();
      if (lane == 0) {
        const uint32_t sa = su32(sTerm + ts * DW_TERM), sb = sa + 3 * DW_TT;
        const uint32_t dcol = tmem + (uint32_t)(buf * 128);
#pragma unroll
        for (int ks = 0; ks < DW_RB / 16; ++ks) {
#pragma unroll
          for (int p = 0; p < 6; ++p) {
            // one 16-deep step spans two 8-row k atoms
            const uint64_t ad = sdesc(sa + pa[p] * DW_TT + ks * 2 * (2 * 1024), 1024, 2 * 1024);
            const uint64_t bd =
                sdesc(sb + pb[p] * DW_TT + ks * 2 * (mnbB * 1024), 1024, mnbB * 1024);
            mma(dcol, ad, bd, id, (ic | ks | p) ? 1u : 0u);
          }
        }
        mma_commit(tempty_s + ts);
        if (ic == DW_CHUNK - 1 || i + 1 == nb) mma_commit(afull + buf);
      }
      any = true;
      __syncwarp();
    }
    // the products in flight complete before the block exits
    if (any) {
      if (lane == 0) mma_commit(fin);
      __syncwarp();
      mbar_drain(fin, 0u);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;          // tensor-memory lane quadrant of this warp
    const int row = q * 32 + lane;   // accumulator row
    const uint32_t la = tmem + ((uint32_t)(q * 32) << 16);
    const int ncol = g.bwb;  // a multiple of 16
    int ch = 0;
    for (; ch < nch; ++ch) {
      const int buf = ch & 1;
      if (!mbar_wait_warp(afull + buf, (uint32_t)(ch / 2) & 1u, flag, 18)) break;
      tc_fence_after();
      for (int c0 = 0; c0 < ncol; c0 += 16) {
        uint32_t p[16], d[32];
        tmem_ld16u(la + (uint32_t)(buf * 128 + c0), p);
        if (ch) tmem_ld32u(la + (uint32_t)(256 + 2 * c0), d);
        tmem_wait_ld();
        add16(d, p, ch == 0);
        tmem_st32u(la + (uint32_t)(256 + 2 * c0), d);
      }
      tmem_wait_st();
      tc_fence_before();
      mbar_arrive(aempty + buf);
    }
    const int gr = tm * 128 + row;
    if (ch == nch && nch > 0) {  // warp-uniform: the loads are warp-collective
      const bool mine = row < g.bwa && gr < g.Mdw;
      double *dst = g.G + (size_t)(mine ? gr : 0) * g.gld + g.gcol0 + tn * 128;
      const int nval = mine ? min(g.bwb, g.Ndw - tn * 128) : 0;
      for (int c0 = 0; c0 < ncol; c0 += 16) {
        uint32_t d[32];
        tmem_ld32u(la + (uint32_t)(256 + 2 * c0), d);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (c0 + i < nval)
            atomicAdd(dst + c0 + i, __hiloint2double((int)d[2 * i + 1], (int)d[2 * i]));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == DW_W_MMA)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// host-side split of one FP32 value into three bf16 terms (round to nearest
// even, as __float2bfloat16_rn)
static uint16_t bf16_rn(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);
  uint32_t r = u + 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}
static float bf16_f(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
static size_t kmaj_off_h(int row, int k) {
  return (size_t)((row >> 3) * 1024 + (row & 7) * ROWB + ((((k >> 3) ^ (row & 7)) & 7) << 4) +
                  (k & 7) * 2);
}

// pre-split weights of one GEMM: Bmat(nrow = N, k = K) element source
// fn(n, k), laid out [N tile][term][K block][BN rows][128 B]
template <typename F>
static std::vector<uint8_t> prep_b(int N, int K, int BN, F fn) {
  const int nkb = (K + BK - 1) / BK, ntn = (N + BN - 1) / BN;
  const size_t btile = (size_t)BN * ROWB;
  std::vector<uint8_t> out((size_t)ntn * 3 * nkb * btile, 0);
  for (int tn = 0; tn < ntn; ++tn)
    for (int r = 0; r < BN; ++r) {
      const int n = tn * BN + r;
      if (n >= N) continue;
      for (int k = 0; k < K; ++k) {
        float x = fn(n, k);
        uint16_t h1 = bf16_rn(x);
        float rr = x - bf16_f(h1);
        uint16_t h2 = bf16_rn(rr);
        rr = rr - bf16_f(h2);
        uint16_t h3 = bf16_rn(rr);
        const int kb = k / BK, kk = k % BK;
        const uint16_t hs[3] = {h1, h2, h3};
        for (int p = 0; p < 3; ++p) {
          size_t off = (size_t)tn * 3 * nkb * btile + ((size_t)p * nkb + kb) * btile +
                       kmaj_off_h(r, kk);
          std::memcpy(&out[off], &hs[p], 2);
        }
      }
    }
  return out;
}

}  // namespace tc

// per-network pre-split weights
struct TcWeights {
  std::vector<uint8_t *> fwd, dt;  // per layer (index l-1)
  std::vector<float *> bias;
  std::vector<int> bn_fwd, bn_dt;
  int *flag = nullptr;
};

static bool g_tc_checked = false, g_tc_ok = false;

bool gemm_tc_available() {
  if (!g_tc_checked) {
    g_tc_checked = true;
    int dev = 0, major = 0, minor = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) == cudaSuccess)
      g_tc_ok = (major == 10 && minor == 0);
  }
  return g_tc_ok;
}

void gemm_tc_release_weights(DevNet *net) {
  TcWeights *w = (TcWeights *)net->tc;
  if (!w) return;
  for (auto p : w->fwd) if (p) cudaFree(p);
  for (auto p : w->dt) if (p) cudaFree(p);
  for (auto p : w->bias) if (p) cudaFree(p);
  if (w->flag) cudaFree(w->flag);
  delete w;
  net->tc = nullptr;
}

// N tile of a FWD/DT product with N outputs and depth K: the widest of
// min(N, 128), 64, 32, 16 that divides N and leaves the pre-split weights
// (3 terms x K x BN bf16) resident in shared memory beside the stages; 0
// when none does.  (K = 256 takes BN = 64.)
static int tc_bn(int N, int K) {
  if (N % 16 || K % 16 || N < 16 || K < 16) return 0;
  const int nkb = (K + 63) / 64;
  const int cand[4] = {std::min(N, 128), 64, 32, 16};
  for (int BN : cand) {
    if (BN > N || N % BN) continue;
    const size_t smem = (size_t)3 * nkb * BN * 128 + 2 * 3 * 128 * 128 + 2048 + tc::STG_BYTES;
    if (smem <= 227 * 1024) return BN;
  }
  return 0;
}

// Pre-split weights of a network.  The buffers are allocated on the first
// call and rewritten in place afterwards (a network's shapes never change),
// so kernels captured in a graph keep valid weight addresses across weight
// updates.  The copies are ordered on st and complete before the return.
int gemm_tc_prepare(DevNet *net, const double *hw, cudaStream_t st) {
  if (!gemm_tc_available()) return RC_OK;
  TcWeights *w = (TcWeights *)net->tc;
  const int L = net->nlayer;
  if (!w) {
    w = new TcWeights();
    net->tc = w;
    w->fwd.assign(L, nullptr);
    w->dt.assign(L, nullptr);
    w->bias.assign(L, nullptr);
    w->bn_fwd.assign(L, 0);
    w->bn_dt.assign(L, 0);
    CKT(cudaMalloc(&w->flag, sizeof(int)));
    CKT(cudaMemsetAsync(w->flag, 0, sizeof(int), st));
  }
  for (int l = 3; l < L; ++l) {  // hidden layers with a GEMM
    const int n = net->dims[l - 1], m = net->dims[l - 2];
    const double *Wl = hw + net->woff[l - 1];
    if (const int BN = tc_bn(n, m)) {
      auto b = tc::prep_b(n, m, BN, [&](int j, int k) { return (float)Wl[(size_t)j * (m + 1) + 1 + k]; });
      if (!w->fwd[l - 1]) CKT(cudaMalloc(&w->fwd[l - 1], b.size()));
      CKT(cudaMemcpyAsync(w->fwd[l - 1], b.data(), b.size(), cudaMemcpyHostToDevice, st));
      std::vector<float> bias(n);
      for (int j = 0; j < n; ++j) bias[j] = (float)Wl[(size_t)j * (m + 1)];
      if (!w->bias[l - 1]) CKT(cudaMalloc(&w->bias[l - 1], n * sizeof(float)));
      CKT(cudaMemcpyAsync(w->bias[l - 1], bias.data(), n * sizeof(float), cudaMemcpyHostToDevice, st));
      w->bn_fwd[l - 1] = BN;
      CKT(cudaStreamSynchronize(st));  // b and bias leave scope
    }
    if (const int BN = tc_bn(m, n)) {
      auto b = tc::prep_b(m, n, BN, [&](int i, int j) { return (float)Wl[(size_t)j * (m + 1) + 1 + i]; });
      if (!w->dt[l - 1]) CKT(cudaMalloc(&w->dt[l - 1], b.size()));
      CKT(cudaMemcpyAsync(w->dt[l - 1], b.data(), b.size(), cudaMemcpyHostToDevice, st));
      w->bn_dt[l - 1] = BN;
      CKT(cudaStreamSynchronize(st));
    }
  }
  return RC_OK;
}

static int sm_count_t() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}


// cuTensorMapEncodeTiled from the driver the runtime has loaded, looked up
// once: the library itself does not link libcuda, so it loads (and answers
// its non-device calls) on hosts without a driver
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// tensor map of the FWD/DT output C[M][N] (row stride ldc floats): boxes of
// 32 rows x 32 columns in the 128-byte swizzle
static int c_tensor_map(CUtensorMap *m, float *C, int M, int N, int ldc) {
  const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)M};
  const cuuint64_t strides[1] = {(cuuint64_t)ldc * sizeof(float)};
  const cuuint32_t box[2] = {32, 32};
  const cuuint32_t estr[2] = {1, 1};
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the CUDA driver");
    return RC_DEVICE;
  }
  const CUresult r = enc(
      m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for a layer GEMM output (code " +
              std::to_string((int)r) + ")");
    return RC_DEVICE;
  }
  return RC_OK;
}

static int launch(const tc::Args &a, int mode, dim3 grid, size_t smem, cudaStream_t st) {
  CUtensorMap cmap;
  std::memset(&cmap, 0, sizeof cmap);
  if (mode != tc::MODE_DW) {
    int rc = c_tensor_map(&cmap, a.C, a.M, a.N, a.ldc);
    if (rc) return rc;
    smem += tc::STG_BYTES;
  }
  if (mode == tc::MODE_FWD) {
    CKT(cudaFuncSetAttribute(tc::k_tc_gemm<tc::MODE_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH("k_tc_gemm_fwd", st, tc::k_tc_gemm<tc::MODE_FWD><<<grid, tc::Roles<tc::MODE_FWD>::NT, smem, st>>>(a, cmap));
  } else if (mode == tc::MODE_DT) {
    CKT(cudaFuncSetAttribute(tc::k_tc_gemm<tc::MODE_DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH("k_tc_gemm_dt", st, tc::k_tc_gemm<tc::MODE_DT><<<grid, tc::Roles<tc::MODE_DT>::NT, smem, st>>>(a, cmap));
  } else {
    CKT(cudaFuncSetAttribute(tc::k_tc_gemm<tc::MODE_DW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH("k_tc_gemm_dw", st, tc::k_tc_gemm<tc::MODE_DW><<<grid, tc::Roles<tc::MODE_DW>::NT, smem, st>>>(a, cmap));
  }
  CKT(cudaGetLastError());
  return RC_OK;
}

static int fwd_like(int mode, const uint8_t *W, const float *bias, int BN, int M, int N, int K,
                    int na, const void *A, void *C, int *flag, cudaStream_t st) {
  const int nkb = (K + tc::BK - 1) / tc::BK;
  const int ntn = (N + BN - 1) / BN;
  const size_t bres = (size_t)3 * nkb * BN * tc::ROWB;
  const size_t smem = 1024 + bres + 2 * 3 * tc::BM * tc::ROWB + 1024;
  tc::Args a;
  std::memset(&a, 0, sizeof a);
  a.mode = mode; a.M = M; a.N = N; a.K = K; a.na = na;
  a.A = (const float *)A; a.lda = K; a.W = W; a.bias = bias;
  a.C = (float *)C; a.ldc = N; a.BN = BN; a.ntn = ntn; a.flag = flag;
  const int tiles_m = (M + tc::BM - 1) / tc::BM;
  dim3 grid(std::max(1, std::min(tiles_m, grid_sms() / ntn)), ntn);
  return launch(a, mode, grid, smem, st);
}

int gemm_tc_fwd(const DevNet *net, int l, int M, int n, int m, int na, const void *A, void *C,
                cudaStream_t st) {
  TcWeights *w = (TcWeights *)net->tc;
  if (!w || !w->fwd[l - 1]) return RC_UNSUPPORTED;
  return fwd_like(tc::MODE_FWD, w->fwd[l - 1], w->bias[l - 1], w->bn_fwd[l - 1], M, n, m, na, A,
                  C, w->flag, st);
}

int gemm_tc_dt(const DevNet *net, int l, int M, int n, int m, const void *Sb, void *Tb,
               cudaStream_t st) {
  TcWeights *w = (TcWeights *)net->tc;
  if (!w || !w->dt[l - 1]) return RC_UNSUPPORTED;
  return fwd_like(tc::MODE_DT, w->dt[l - 1], nullptr, w->bn_dt[l - 1], M, m, n, 1, Sb, Tb,
                  w->flag, st);
}

// tensor map of an FP32 operand P[rows][cols] (row stride ld floats):
// boxes of DW_RB rows x bw columns, no swizzle, zeros past the edges
static int f32_box_map(CUtensorMap *m, const float *P, int rows, int cols, int ld, int bw) {
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)tc::DW_RB};
  const cuuint32_t estr[2] = {1, 1};
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is not available from the CUDA driver");
    return RC_DEVICE;
  }
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)P, dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for a weight-gradient operand (code " +
              std::to_string((int)r) + ")");
    return RC_DEVICE;
  }
  return RC_OK;
}

// G[j][gcol0 + i] += sum_r A[r][j] B[r][i], A [K][Mdw] (row stride lda), B
// [K][Ndw] (ldb): k_tc_dw over one wave of blocks, each an output tile of
// 128 x 128 and a contiguous run of rows.  Widths are multiples of 16 and
// the leading dimensions multiples of 4 (16-byte rows for TMA).
static int dw_tma(const float *A, int Mdw, int lda, const float *B, int Ndw, int ldb, int K,
                  double *G, int gld, int gcol0, int *flag, cudaStream_t st) {
  if (Mdw < 16 || Ndw < 16 || Mdw % 16 || Ndw % 16 || lda % 4 || ldb % 4 || lda < Mdw ||
      ldb < Ndw || ((uintptr_t)A & 15) || ((uintptr_t)B & 15) || K < 1)
    return RC_UNSUPPORTED;
  const int ntm = (Mdw + 127) / 128, ntn = (Ndw + 127) / 128;
  if (ntm > 65535 || ntn > 65535) return RC_UNSUPPORTED;
  const int nkb_all = (K + tc::DW_RB - 1) / tc::DW_RB;
  const long tiles = (long)ntm * ntn;
  const int ctas_k =
      (int)std::max<long>(1, std::min<long>(nkb_all, std::max<long>(1, grid_sms() / tiles)));
  tc::DwArgs a;
  std::memset(&a, 0, sizeof a);
  a.Mdw = Mdw; a.Ndw = Ndw; a.K = K;
  a.bwa = std::min(128, Mdw); a.bwb = std::min(128, Ndw);
  a.kb_per_cta = (nkb_all + ctas_k - 1) / ctas_k;
  a.G = G; a.gld = gld; a.gcol0 = gcol0; a.flag = flag;
  CUtensorMap amap, bmap;
  std::memset(&amap, 0, sizeof amap);
  std::memset(&bmap, 0, sizeof bmap);
  int rc = f32_box_map(&amap, A, K, Mdw, lda, a.bwa);
  if (!rc) rc = f32_box_map(&bmap, B, K, Ndw, ldb, a.bwb);
  if (rc) return rc;
  const dim3 grid((nkb_all + a.kb_per_cta - 1) / a.kb_per_cta, ntn, ntm);
  CKT(cudaFuncSetAttribute(tc::k_tc_dw, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)tc::DW_SMEM));
  LAUNCH("k_tc_gemm_dw", st, tc::k_tc_dw<<<grid, tc::DW_NTH, tc::DW_SMEM, st>>>(a, amap, bmap));
  CKT(cudaGetLastError());
  return RC_OK;
}

int gemm_tc_dw(const DevNet *net, int l, int M, int n, int m, const void *Sb, const void *Tm,
               double *G, cudaStream_t st) {
  (void)l;
  TcWeights *w = (TcWeights *)net->tc;
  if (!w) return RC_UNSUPPORTED;
  return dw_tma((const float *)Sb, n, n, (const float *)Tm, m, m, M, G, m + 1, 1, w->flag, st);
}

// G[i][j] += sum_r J[r][i] J[r][j] over an FP32 copy J[nrow][ldj] (ldj a
// multiple of 4, zero past nw): the DW form with both operands J, output
// tiles of 128 rows x 64 columns, the row reduction split across blocks.
int gemm_tc_syrk(const float *J, int nrow, int nw, int ldj, double *G, cudaStream_t st) {
  if (!gemm_tc_available() || nrow < 1 || nw < 1 || ldj % 4 || ldj < nw) return RC_UNSUPPORTED;
  static int *flag = nullptr;
  if (!flag) {
    CKT(cudaMalloc(&flag, sizeof(int)));
    CKT(cudaMemset(flag, 0, sizeof(int)));
  }
  const int BN = 64;
  const int ntn = (nw + BN - 1) / BN, ntm = (nw + tc::BM - 1) / tc::BM;
  if (ntm > 65535) return RC_UNSUPPORTED;
  const int nkb_all = (nrow + tc::BK - 1) / tc::BK;
  const long tiles = (long)ntn * ntm;
  const int ctas_k = (int)std::max<long>(1, std::min<long>(nkb_all, 2 * sm_count_t() / std::max(1L, tiles)));
  tc::Args a;
  std::memset(&a, 0, sizeof a);
  a.mode = tc::MODE_DW; a.M = nw; a.N = nw; a.K = nrow; a.na = 1;
  a.A = J; a.lda = ldj; a.B = J; a.ldb = ldj;
  a.G = G; a.gld = nw; a.gcol0 = 0; a.BN = BN; a.ntn = ntn; a.kchunk = 8;
  a.kblocks_per_cta = (nkb_all + ctas_k - 1) / ctas_k;
  a.flag = flag;
  const size_t stage = 3 * (8 * 2 * 1024) + 3 * (8 * 1 * 1024);
  const size_t smem = 1024 + 3 * stage + 1024;
  dim3 grid((nkb_all + a.kblocks_per_cta - 1) / a.kblocks_per_cta, ntn, ntm);
  int rc = launch(a, tc::MODE_DW, grid, smem, st);
  if (rc) return rc;
  int h = 0;
  CKT(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKT(cudaStreamSynchronize(st));
  if (h) {
    cudaMemset(flag, 0, sizeof(int));
    set_error("tensor-core metric: an mbarrier wait timed out (code " + std::to_string(h) + ")");
    return RC_DEVICE;
  }
  return RC_OK;
}

int gemm_tc_flag(const DevNet *net, cudaStream_t st) {
  TcWeights *w = (TcWeights *)net->tc;
  if (!w) return RC_OK;
  int h = 0;
  CKT(cudaMemcpyAsync(&h, w->flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKT(cudaStreamSynchronize(st));
  if (h) {
    // report once, then clear, so that the next call runs afresh
    cudaMemsetAsync(w->flag, 0, sizeof(int), st);
    cudaStreamSynchronize(st);
    set_error("tensor-core GEMM: an mbarrier wait timed out (code " + std::to_string(h) + ")");
    return RC_DEVICE;
  }
  return RC_OK;
}

}  // namespace dnnf90
