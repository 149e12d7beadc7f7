// bell_tile.cu - register-tiled Bell forward (Horner form) and adjoint
// (correlation form) for dense multi-index sets, FP32 planes.
//
// The recurrences and the tiling are described in tile_plan.hpp.  One block
// of warps (TILE_WARPS_F in the forward, TILE_WARPS_A in the adjoint) owns one item at a time: one point and 32 neurons,
// lane = neuron, so every shared-memory row is 32 consecutive words (one
// 128-byte row of FP32 values, or a 256-byte row of (D, E) pairs) and
// every access of a warp is one row, conflict-free.  The block's warps
// share the item's state and split each phase's units (work lists of
// tile_plan.cpp); the next item's rows stream into the second buffer by
// cp.async while the current one is computed.
//
// A unit keeps its output tile's accumulators in registers.  For each of
// its records it loads one factor tile into registers and streams the other
// factor's tile row by row; every streamed row feeds all outputs of the
// tile it reaches (a tile of side 8 in two dimensions: 36 rows of each
// factor against 330 multiply-adds).  The forward's two chains multiply by
// the same s~, so (D, E) is one packed FP32 multiply-add (FFMA2).
//
// Callers: bell.cu's Bell forward and adjoint dispatch (variant 3 of each,
// the default wherever the plan applies).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "bell.hpp"
#include "engine.hpp"
#include "kernels.cuh"
#include "tile_plan.hpp"

namespace dnnf90 {

namespace {

constexpr int TWF = TILE_WARPS_F, TWA = TILE_WARPS_A;

// ------------------------------------------------------------ tile algebra
// entries of a tile of side L in td dimensions, and the graded index maps
__host__ __device__ constexpr int tsize(int td, int L) { return td == 2 ? L * (L + 1) / 2 : L; }
__host__ __device__ constexpr int tdeg(int td, int e) {
  int s = 0;
  if (td == 1) return e;
  while ((s + 1) * (s + 2) / 2 <= e) ++s;
  return s;
}
__host__ __device__ constexpr int tsecond(int td, int e) {
  return td == 1 ? 0 : e - tdeg(2, e) * (tdeg(2, e) + 1) / 2;
}
__host__ __device__ constexpr int tfirst(int td, int e) {
  return td == 1 ? e : tdeg(2, e) - tsecond(2, e);
}
__host__ __device__ constexpr int tindex(int td, int a1, int a2) {
  return td == 1 ? a1 : (a1 + a2) * (a1 + a2 + 1) / 2 + a2;
}
// index of the sum of entries e and c
__host__ __device__ constexpr int tadd(int td, int e, int c) {
  return tindex(td, tfirst(td, e) + tfirst(td, c), tsecond(td, e) + tsecond(td, c));
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Rows of a [na][n] plane slice (neurons j0 .. j0+31) into shared rows
// perm[r] of dst (128 bytes each), 16-byte pieces; columns at or beyond n
// read as zero.  n is a multiple of 4, so a piece is wholly in or out of the
// row.  (One 128-byte bulk copy per row measured slower: the rows queue
// through the SM's bulk-copy unit one request at a time.)
__device__ __forceinline__ void stage_perm(unsigned char *dst, const float *src, const int *perm,
                                           int na, int n, int j0) {
  for (int c = threadIdx.x; c < na * 8; c += blockDim.x) {
    const int r = c >> 3, piece = c & 7;
    const int col = j0 + piece * 4;
    const int ok = col < n ? 16 : 0;
    cp16(dst + perm[r] * 128 + piece * 16, src + (size_t)r * n + (ok ? col : 0), ok);
  }
}

// copy of n 32-bit words of a table into shared memory
__device__ __forceinline__ void copy_words(void *dst, const void *src, int nwords) {
  for (int i = threadIdx.x; i < nwords; i += blockDim.x)
    ((uint32_t *)dst)[i] = __ldg((const uint32_t *)src + i);
}

// items [it0, it1) of this block: a contiguous share of npts * gy items,
// item = point + npts * (32-neuron tile)
__device__ __forceinline__ void block_items(long nitem, long &it0, long &it1) {
  it0 = (long)blockIdx.x * nitem / gridDim.x;
  it1 = (long)(blockIdx.x + 1) * nitem / gridDim.x;
}

// ------------------------------------------------------------ forward
// shared-memory layout (byte offsets), computed on the host
struct Fwd10Args {
  int n, na, npts, gy, k, iact;
  int nunit, nrec;
  int o_s1, o_d0, o_d1, o_sig, o_list, o_unit, o_rec, o_perm, o_rowslot, o_fact, o_ifact;
  const double *tpc;
  const int *list;       // [k][TWF][2]
  const int4 *unit;      // [nunit]: L | origin << 8, first record, records, out row
  const uint32_t *rec;   // [nrec]: s row | d row << 16
  const int *perm;       // [na]
  const int *rowslot;    // [na]
  const float *fact;     // [na] per row: a!
  const float *ifact;    // [na] per row: 1 / a!
  const float *S;
  float *T, *h;
};

// one record: acc[b + c] += s~_b (D, E)_c over b, c with |b| + |c| <= L - 1
// (b != 0 for the record of delta = 0, whose D tile has side L - 1).
// The loops are template recursions, so that every register index is a
// compile-time constant.  For one streamed row c: outputs b + c, b in the
// prefix of entries of degree <= L - 1 - |c|.
template <int TD, int C, int E, int EN>
struct FwdRow {
  static __device__ __forceinline__ void run(const float *sv, float2 dv, float2 *acc) {
    constexpr int o = tadd(TD, E, C);
    acc[o] = __ffma2_rn(make_float2(sv[E], sv[E]), dv, acc[o]);
    FwdRow<TD, C, E + 1, EN>::run(sv, dv, acc);
  }
};
template <int TD, int C, int EN>
struct FwdRow<TD, C, EN, EN> {
  static __device__ __forceinline__ void run(const float *, float2, float2 *) {}
};
template <int TD, int L, bool Z, int C, int CN>
struct FwdRows {
  static __device__ __forceinline__ void run(const float *sv, const float2 *d, float2 *acc) {
    const float2 dv = d[C * 32];
    FwdRow<TD, C, Z ? 1 : 0, tsize(TD, L - tdeg(TD, C))>::run(sv, dv, acc);
    FwdRows<TD, L, Z, C + 1, CN>::run(sv, d, acc);
  }
};
template <int TD, int L, bool Z, int CN>
struct FwdRows<TD, L, Z, CN, CN> {
  static __device__ __forceinline__ void run(const float *, const float2 *, float2 *) {}
};

template <int TD, int L, bool Z>
__device__ __forceinline__ void tile_fwd(const float *s, const float2 *d,
                                         float2 (&acc)[tsize(TD, L)]) {
  constexpr int NT = tsize(TD, L);
  constexpr int ND = tsize(TD, Z ? L - 1 : L);
  float sv[NT];
#pragma unroll
  for (int e = 0; e < NT; ++e) sv[e] = (Z && e == 0) ? 0.f : s[e * 32];
  FwdRows<TD, L, Z, 0, ND>::run(sv, d, acc);
}

struct FwdCtx {
  const float *S;         // this lane's word of the current S buffer
  const float2 *Dr;       // this lane's word of the buffer of D_{q+1}
  float2 *Dw;             // this lane's word of the buffer of D_q
  const uint32_t *rec;
  const int *rowslot;
  const float *fact;
  float *T, *H;           // this point's planes at this lane's neuron
  int n;
  bool act;
};

template <int TD, int L, bool TRAIN>
__device__ __forceinline__ void fwd_unit(const FwdCtx &c, int4 u, int q, float inv, float2 sg) {
  constexpr int NT = tsize(TD, L);
  float2 acc[NT];
#pragma unroll
  for (int e = 0; e < NT; ++e) acc[e] = make_float2(0.f, 0.f);
  {
    const uint32_t r = c.rec[u.y];
    tile_fwd<TD, L, true>(c.S + (r & 0xffffu) * 32, c.Dr + (r >> 16) * 32, acc);
  }
  int i = u.y + 1;
  const int end = u.y + u.z;
  for (; i < end; ++i) {
    const uint32_t r = c.rec[i];
    tile_fwd<TD, L, false>(c.S + (r & 0xffffu) * 32, c.Dr + (r >> 16) * 32, acc);
  }
  const float2 iv = make_float2(inv, inv);
#pragma unroll
  for (int e = 0; e < NT; ++e) acc[e] = __fmul2_rn(acc[e], iv);
  if (u.x >> 8) acc[0] = sg;  // the origin: D_q(0) = sigma_q, E_q(0) = sigma_{q+1}
  if (q > 0) {
#pragma unroll
    for (int e = 0; e < NT; ++e) c.Dw[(u.w + e) * 32] = acc[e];
  } else if (c.act) {
#pragma unroll
    for (int e = 0; e < NT; ++e) {
      const int row = u.w + e;
      const size_t at = (size_t)c.rowslot[row] * c.n;
      const float f = c.fact[row];
      c.T[at] = f * acc[e].x;
      if (TRAIN) c.H[at] = f * acc[e].y;
    }
  }
}

template <int TD, bool TRAIN>
__global__ void __launch_bounds__(TWF * 32, 1) k_bell_fwd10(Fwd10Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = a.n, na = a.na, K = a.k;
  int *slist = (int *)(sm + a.o_list);
  int4 *sunit = (int4 *)(sm + a.o_unit);
  uint32_t *srec = (uint32_t *)(sm + a.o_rec);
  int *sperm = (int *)(sm + a.o_perm);
  int *srowslot = (int *)(sm + a.o_rowslot);
  float *sfact = (float *)(sm + a.o_fact);
  float *sifact = (float *)(sm + a.o_ifact);
  copy_words(slist, a.list, K * TWF * 2);
  copy_words(sunit, a.unit, a.nunit * 4);
  copy_words(srec, a.rec, a.nrec);
  copy_words(sperm, a.perm, na);
  copy_words(srowslot, a.rowslot, na);
  copy_words(sfact, a.fact, na);
  copy_words(sifact, a.ifact, na);
  __syncthreads();
  const size_t plane = (size_t)na * n;
  const long nitem = (long)a.npts * a.gy;
  long it0, it1;
  block_items(nitem, it0, it1);
  if (it0 < it1)
    stage_perm(sm, a.S + (it0 % a.npts) * plane, sperm, na, n, (int)(it0 / a.npts) * 32);
  cp_commit();
  float *sig = (float *)(sm + a.o_sig) + lane;
  FwdCtx c;
  c.rec = srec;
  c.rowslot = srowslot;
  c.fact = sfact;
  c.n = n;
  int buf = 0;
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * 32 + lane;
    c.act = j < n;
    cp_wait_all();
    __syncthreads();  // this item's S rows are in; every warp is done with the last item
    if (it + 1 < it1)
      stage_perm(sm + (buf ? 0 : a.o_s1), a.S + ((it + 1) % a.npts) * plane, sperm, na, n,
                 (int)((it + 1) / a.npts) * 32);
    cp_commit();
    float *Sb = (float *)(sm + (buf ? a.o_s1 : 0)) + lane;
    // S_a -> S_a / a!, 16 bytes per thread at a time; the origin row keeps
    // S_0 (0! = 1) and is left alone, since warp 0 reads it next
    {
      unsigned char *sb0 = sm + (buf ? a.o_s1 : 0);
#pragma unroll 4
      for (int c = threadIdx.x + 8; c < na * 8; c += blockDim.x) {
        float4 *p = (float4 *)(sb0 + c * 16);
        const float f = sifact[c >> 3];
        float4 v = *p;
        v.x *= f; v.y *= f; v.z *= f; v.w *= f;
        *p = v;
      }
    }
    if (a.iact == 0) {
      // tanh: warp q forms sigma_q = P_q(tanh S_0) (lib/multi_index_bell_module.f90:
      // 406-429, the polynomials of sigma_derivs, in the same order), so that no
      // warp evaluates them all; warps K and K+1 also fill D_K = sigma_K,
      // E_K = sigma_{K+1} (row 0 of buffer K & 1)
      if (warp <= K + 1) {
        const double t = tanh((double)Sb[0]);
        const double *row = a.tpc + warp * (K + 3);
        double v = __ldg(row + warp + 1);
        for (int i = warp; i >= 0; --i) v = v * t + __ldg(row + i);
        sig[warp * 32] = (float)v;
        float2 *dk = (float2 *)(sm + ((K & 1) ? a.o_d1 : a.o_d0)) + lane;
        if (warp == K) dk[0].x = (float)v;
        if (warp == K + 1) dk[0].y = (float)v;
      }
    } else if (warp == 0) {
      double d[TILE_KMAX + 2];
      sigma_derivs(a.iact, a.tpc, K, (double)Sb[0], d);
      float dk0 = 0.f, dk1 = 0.f;
#pragma unroll
      for (int q = 0; q <= TILE_KMAX + 1; ++q) {
        if (q <= K + 1) sig[q * 32] = (float)d[q];
        if (q == K) dk0 = (float)d[q];
        if (q == K + 1) dk1 = (float)d[q];
      }
      // D_K = sigma_K, E_K = sigma_{K+1}: row 0 of buffer K & 1
      float2 *dk = (float2 *)(sm + ((K & 1) ? a.o_d1 : a.o_d0)) + lane;
      dk[0] = make_float2(dk0, dk1);
    }
    __syncthreads();
    c.S = Sb;
    c.T = a.T + pt * plane + j;
    c.H = TRAIN ? a.h + pt * plane + j : nullptr;
    for (int q = K - 1; q >= 0; --q) {
      c.Dr = (const float2 *)(sm + (((q + 1) & 1) ? a.o_d1 : a.o_d0)) + lane;
      c.Dw = (float2 *)(sm + ((q & 1) ? a.o_d1 : a.o_d0)) + lane;
      const float inv = 1.0f / (float)(q + 1);
      const float2 sg = make_float2(sig[q * 32], sig[(q + 1) * 32]);
      const int u0 = slist[(q * TWF + warp) * 2], un = slist[(q * TWF + warp) * 2 + 1];
      for (int u = u0; u < u0 + un; ++u) {
        const int4 U = sunit[u];
        switch (U.x & 0xff) {
#define F10(LL) \
  case LL: fwd_unit<TD, LL, TRAIN>(c, U, q, inv, sg); break;
          F10(1) F10(2) F10(3) F10(4) F10(5) F10(6) F10(7) F10(8)
#undef F10
          default: break;
        }
      }
      if (q > 0) __syncthreads();
    }
    buf ^= 1;
  }
  cp_wait_all();
}

// ------------------------------------------------------------ adjoint
struct Adj10Args {
  int n, na, npts, gy, gstride;
  int nunit, nrec, nfin, nscr;
  int o_b1, o_scr, o_list, o_unit, o_rec, o_flist, o_fin, o_perm, o_rowslot, o_fact, o_ifact;
  const int *list;       // [TWA][2]
  const int4 *unit;      // [nunit]: Lout | split << 8, first record, records, out row
  const uint32_t *rec;   // [nrec]: h row | Tb row << 14 | L << 28
  const int *flist;      // [TWA][2]
  const int4 *fin;       // [nfin]: Lout, out row, parts, first scratch row
  const int *perm;
  const int *rowslot;
  const float *fact, *ifact;
  const float *Tb, *h;
  float *Sb;
  double *gbias;
};

// one record: acc[a - c] += (a! Tb)_a (h / c!)_c over a in the Tb tile of
// side L and c <= a (componentwise).  tb, hh: this lane's word of the two
// tiles' first rows.  Template recursions keep every index compile-time.
// c = (C1, C2): C2 runs over 0 .. a2, C1 over 0 .. a1
template <int TD, int A, int C1, int C2, bool END = (C2 > tsecond(TD, A))>
struct AdjInner;
template <int TD, int A, int C1, int C2>
struct AdjInner<TD, A, C1, C2, false> {
  static __device__ __forceinline__ void run(float x, const float *hv, float *acc) {
    constexpr int o = tindex(TD, tfirst(TD, A) - C1, tsecond(TD, A) - C2);
    acc[o] = fmaf(x, hv[tindex(TD, C1, C2)], acc[o]);
    AdjInner<TD, A, C1, C2 + 1>::run(x, hv, acc);
  }
};
template <int TD, int A, int C1, int C2>
struct AdjInner<TD, A, C1, C2, true> {
  static __device__ __forceinline__ void run(float, const float *, float *) {}
};
template <int TD, int A, int C1, bool END = (C1 > tfirst(TD, A))>
struct AdjOuter;
template <int TD, int A, int C1>
struct AdjOuter<TD, A, C1, false> {
  static __device__ __forceinline__ void run(float x, const float *hv, float *acc) {
    AdjInner<TD, A, C1, 0>::run(x, hv, acc);
    AdjOuter<TD, A, C1 + 1>::run(x, hv, acc);
  }
};
template <int TD, int A, int C1>
struct AdjOuter<TD, A, C1, true> {
  static __device__ __forceinline__ void run(float, const float *, float *) {}
};
template <int TD, int A, int AN>
struct AdjRows {
  static __device__ __forceinline__ void run(const float *tb, const float *hv, float *acc) {
    const float x = tb[A * 32];
    AdjOuter<TD, A, 0>::run(x, hv, acc);
    AdjRows<TD, A + 1, AN>::run(tb, hv, acc);
  }
};
template <int TD, int AN>
struct AdjRows<TD, AN, AN> {
  static __device__ __forceinline__ void run(const float *, const float *, float *) {}
};

template <int TD, int LO, int L>
__device__ __forceinline__ void tile_adj(const float *tb, const float *hh,
                                         float (&acc)[tsize(TD, LO)]) {
  constexpr int NT = tsize(TD, L);
  float hv[NT];
#pragma unroll
  for (int c = 0; c < NT; ++c) hv[c] = hh[c * 32];
  AdjRows<TD, 0, NT>::run(tb, hv, acc);
}

// Every unit keeps the accumulators of the largest output tile (side LMAX),
// so that the record code is one body per record tile side, shared by all
// output tile sides: the units run their records of side LMAX, LMAX - 1,
// ..., 1 in turn, (cw >> 4 (LO - L)) & 15 of side L (the plan orders them
// so), where LO is the unit's output tile side.
constexpr int LMAX = TILE_KMAX + 1;
template <int TD, int L>
struct AdjL {
  static __device__ __forceinline__ void run(const float *tbb, const float *hb,
                                             const uint32_t *rec, int i, uint32_t cw, int lo,
                                             float (&acc)[tsize(TD, LMAX)]) {
    const int cnt = lo >= L ? (int)((cw >> (4 * (lo - L))) & 15u) : 0;
    for (int k = 0; k < cnt; ++k) {
      const uint32_t r = rec[i + k];
      tile_adj<TD, LMAX, L>(tbb + ((r >> 14) & 0x3fffu) * 32, hb + (r & 0x3fffu) * 32, acc);
    }
    AdjL<TD, L - 1>::run(tbb, hb, rec, i + cnt, cw, lo, acc);
  }
};
template <int TD>
struct AdjL<TD, 0> {
  static __device__ __forceinline__ void run(const float *, const float *, const uint32_t *, int,
                                             uint32_t, int, float (&)[tsize(TD, LMAX)]) {}
};

// the first tsize(TD, LO) accumulators of a unit: into its scratch rows
// (one part of a split output tile), or scaled by 1/b! and stored
template <int TD, int LO>
__device__ __forceinline__ void adj_store(const float (&acc)[tsize(TD, LMAX)], int4 u, float *scr,
                                          const int *rowslot, const float *ifact, float *Sb,
                                          int n, bool act, double &gb) {
  constexpr int NT = tsize(TD, LO);
  if (u.x >> 8) {
#pragma unroll
    for (int e = 0; e < NT; ++e) scr[(u.w + e) * 32] = acc[e];
  } else {
#pragma unroll
    for (int e = 0; e < NT; ++e) {
      const int row = u.w + e;
      const float v = acc[e] * ifact[row];
      if (act) Sb[(size_t)rowslot[row] * n] = v;
      if (row == 0) gb += (double)v;
    }
  }
}

// tbb, hb: this lane's word of the current buffer's Tb rows and h rows
template <int TD>
__device__ __forceinline__ void adj_unit(const float *tbb, const float *hb, const uint32_t *rec,
                                         int4 u, float *scr, const int *rowslot,
                                         const float *ifact, float *Sb, int n, bool act,
                                         double &gb) {
  float acc[tsize(TD, LMAX)];
#pragma unroll
  for (int e = 0; e < tsize(TD, LMAX); ++e) acc[e] = 0.f;
  const int lo = u.x & 0xff;
  AdjL<TD, LMAX>::run(tbb, hb, rec, u.y, (uint32_t)u.z, lo, acc);
  switch (lo) {
#define ST10(LL) \
  case LL: adj_store<TD, LL>(acc, u, scr, rowslot, ifact, Sb, n, act, gb); break;
    ST10(1) ST10(2) ST10(3) ST10(4) ST10(5) ST10(6) ST10(7) ST10(8)
#undef ST10
    default: break;
  }
}

template <int TD>
__global__ void __launch_bounds__(TWA * 32, 1) k_bell_adj10(Adj10Args a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *sm = smem_raw;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = a.n, na = a.na;
  int *slist = (int *)(sm + a.o_list);
  int4 *sunit = (int4 *)(sm + a.o_unit);
  uint32_t *srec = (uint32_t *)(sm + a.o_rec);
  int *sflist = (int *)(sm + a.o_flist);
  int4 *sfin = (int4 *)(sm + a.o_fin);
  int *sperm = (int *)(sm + a.o_perm);
  int *srowslot = (int *)(sm + a.o_rowslot);
  float *sfact = (float *)(sm + a.o_fact);
  float *sifact = (float *)(sm + a.o_ifact);
  copy_words(slist, a.list, TWA * 2);
  copy_words(sunit, a.unit, a.nunit * 4);
  copy_words(srec, a.rec, a.nrec);
  copy_words(sflist, a.flist, TWA * 2);
  copy_words(sfin, a.fin, a.nfin * 4);
  copy_words(sperm, a.perm, na);
  copy_words(srowslot, a.rowslot, na);
  copy_words(sfact, a.fact, na);
  copy_words(sifact, a.ifact, na);
  __syncthreads();
  // two sets of scratch rows: an item's split tiles are summed while the
  // next item is computed, so no barrier separates the two
  float *scr0 = (float *)(sm + a.o_scr) + lane;
  const int scr_words = a.nscr * 32;
  const size_t plane = (size_t)na * n;
  const long nitem = (long)a.npts * a.gy;
  long it0, it1;
  block_items(nitem, it0, it1);
  // buffer b: Tb rows at b * o_b1, h rows na rows further
  auto stage = [&](int b, long it) {
    const size_t o = (it % a.npts) * plane;
    const int j0 = (int)(it / a.npts) * 32;
    unsigned char *dst = sm + b * a.o_b1;
    stage_perm(dst, a.Tb + o, sperm, na, n, j0);
    stage_perm(dst + na * 128, a.h + o, sperm, na, n, j0);
  };
  if (it0 < it1) stage(0, it0);
  cp_commit();
  const int u0 = slist[warp * 2], un = slist[warp * 2 + 1];
  const int f0 = sflist[warp * 2], fn = sflist[warp * 2 + 1];
  // the bias gradient: Sb_0 of this lane's neuron summed over the block's
  // items, added once per neuron tile; gb for the units' outputs, gbp for
  // the split tiles' (summed one item later)
  double gb = 0.0, gbp = 0.0;
  int gj = -1, gjp = -1;
  auto flush = [&](double &g, int &jj, int jn) {
    if (jj != jn) {
      if (a.gbias && jj >= 0 && jj < n && g != 0.0) atomicAdd(a.gbias + (size_t)jj * a.gstride, g);
      g = 0.0;
      jj = jn;
    }
  };
  // split output tiles of item itp from scratch set sc: each element's parts
  // summed in a fixed order, the elements dealt over all warps
  auto finish = [&](long itp, const float *sc) {
    const int jp = (int)(itp / a.npts) * 32 + lane;
    flush(gbp, gjp, jp);
    float *Sbp = a.Sb + (itp % a.npts) * plane + jp;
    for (int f = f0; f < f0 + fn; ++f) {
      const int4 F = sfin[f];  // row, parts, first scratch row, part stride
      float v = 0.f;
      for (int p = 0; p < F.y; ++p) v += sc[(F.z + p * F.w) * 32];
      v *= sifact[F.x];
      if (jp < n) Sbp[(size_t)srowslot[F.x] * n] = v;
      if (F.x == 0) gbp += (double)v;
    }
  };
  int buf = 0;
  for (long it = it0; it < it1; ++it) {
    const int pt = (int)(it % a.npts);
    const int j = (int)(it / a.npts) * 32 + lane;
    const bool act = j < n;
    flush(gb, gj, j);
    cp_wait_all();
    __syncthreads();  // this item's rows are in; every warp is done with the last item
    if (it + 1 < it1) stage(buf ^ 1, it + 1);
    cp_commit();
    // Tb_a -> a! Tb_a, h_g -> h_g / g!
    float *rb = (float *)(sm + buf * a.o_b1) + lane;
    {
      unsigned char *b0 = sm + buf * a.o_b1;  // 16 bytes per thread at a time
#pragma unroll 4
      for (int c = threadIdx.x; c < 2 * na * 8; c += blockDim.x) {
        const int r = c >> 3;
        const float f = r < na ? sfact[r] : sifact[r - na];
        float4 *p = (float4 *)(b0 + c * 16);
        float4 v = *p;
        v.x *= f; v.y *= f; v.z *= f; v.w *= f;
        *p = v;
      }
    }
    __syncthreads();  // the rows are scaled; the last item's split parts are in
    if (it > it0) finish(it - 1, scr0 + ((it - 1 - it0) & 1) * scr_words);
    float *Sb = a.Sb + pt * plane + j;
    float *scr = scr0 + ((it - it0) & 1) * scr_words;
    const float *tbb = rb, *hb = rb + na * 32;  // Tb rows, then h rows
    for (int u = u0; u < u0 + un; ++u) {
      const int4 U = sunit[u];
      adj_unit<TD>(tbb, hb, srec, U, scr, srowslot, sifact, Sb, n, act, gb);
    }
    buf ^= 1;
  }
  cp_wait_all();
  __syncthreads();  // the last item's split parts are in
  if (it0 < it1) finish(it1 - 1, scr0 + ((it1 - 1 - it0) & 1) * scr_words);
  flush(gb, gj, -1);
  flush(gbp, gjp, -1);
}

int grid_for(const void *k, int threads, size_t smem, long items) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long g = (long)grid_sms() * per_sm;
  return (int)std::max(1L, std::min(g, items));
}

template <typename T>
int put_vec(T **d, const std::vector<T> &h) {
  if (h.empty()) return RC_OK;
  if (cudaMalloc(d, h.size() * sizeof(T)) != cudaSuccess) {
    set_error("device allocation failed (tile plan)");
    return RC_NOMEM;
  }
  if (cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("copy to the device failed (tile plan)");
    return RC_DEVICE;
  }
  return RC_OK;
}

#define CKT(x)                                                         \
  do {                                                                 \
    cudaError_t e_ = (x);                                              \
    if (e_ != cudaSuccess) {                                           \
      set_error(std::string("bell_tile: ") + cudaGetErrorString(e_));  \
      return RC_DEVICE;                                                \
    }                                                                  \
  } while (0)

}  // namespace

// ------------------------------------------------------------ host side
void TileDev::release() {
  for (void *p : {(void *)flist, (void *)funit, (void *)frec, (void *)alist, (void *)aunit,
                  (void *)arec, (void *)aflist, (void *)afin, (void *)perm, (void *)rowslot,
                  (void *)fact, (void *)ifact})
    if (p) cudaFree(p);
  *this = TileDev();
}

int upload_tile_plan(const TableSet &t, TileDev &d) {
  d.release();
  TilePlan P = build_tile_plan(t, TWF, TWA);
  if (!P.ok) return RC_OK;
  std::vector<float> fact(P.na), ifact(P.na);
  for (int r = 0; r < P.na; ++r) {
    const int ia = P.rowslot[r];
    double f = 1.0;
    for (int i = 0; i < t.d0; ++i)
      for (int v = 2; v <= t.alpha[(size_t)ia * t.d0 + i]; ++v) f *= v;
    fact[r] = (float)f;
    ifact[r] = (float)(1.0 / f);
  }
  int rc;
  if ((rc = put_vec(&d.flist, P.flist)) || (rc = put_vec(&d.funit, P.funit)) ||
      (rc = put_vec(&d.frec, P.frec)) || (rc = put_vec(&d.alist, P.alist)) ||
      (rc = put_vec(&d.aunit, P.aunit)) || (rc = put_vec(&d.arec, P.arec)) ||
      (rc = put_vec(&d.aflist, P.aflist)) || (rc = put_vec(&d.afin, P.afin)) ||
      (rc = put_vec(&d.perm, P.perm)) || (rc = put_vec(&d.rowslot, P.rowslot)) ||
      (rc = put_vec(&d.fact, fact)) || (rc = put_vec(&d.ifact, ifact))) {
    d.release();
    return rc;
  }
  d.td = P.td;
  d.k = P.k;
  d.na = P.na;
  d.nbuf0 = P.nbuf[0];
  d.nbuf1 = P.nbuf[1];
  d.nfunit = (int)P.funit.size() / 4;
  d.nfrec = (int)P.frec.size();
  d.naunit = (int)P.aunit.size() / 4;
  d.narec = (int)P.arec.size();
  d.nafin = (int)P.afin.size() / 4;
  d.nscratch = P.nscratch;
  // shared-memory layouts
  const int na = P.na, K = P.k;
  int o = 2 * na * 128;
  d.f_o_d0 = o;
  o += std::max(1, P.nbuf[0]) * 256;
  d.f_o_d1 = o;
  o += std::max(1, P.nbuf[1]) * 256;
  d.f_o_sig = o;
  o += (K + 2) * 128;
  d.f_o_list = o;
  o += K * TWF * 2 * 4;
  o = (o + 15) / 16 * 16;
  d.f_o_unit = o;
  o += d.nfunit * 16;
  d.f_o_rec = o;
  o += d.nfrec * 4;
  d.f_o_perm = o;
  o += na * 4;
  d.f_o_rowslot = o;
  o += na * 4;
  d.f_o_fact = o;
  o += na * 4;
  d.f_o_ifact = o;
  o += na * 4;
  d.f_smem = o;
  o = 4 * na * 128;  // two buffers of Tb and h rows
  d.a_o_scr = o;
  o += 2 * std::max(1, P.nscratch) * 128;  // two sets of scratch rows
  d.a_o_list = o;
  o += TWA * 2 * 4;
  d.a_o_flist = o;
  o += TWA * 2 * 4;
  o = (o + 15) / 16 * 16;
  d.a_o_unit = o;
  o += d.naunit * 16;
  d.a_o_fin = o;
  o += d.nafin * 16;
  d.a_o_rec = o;
  o += d.narec * 4;
  d.a_o_perm = o;
  o += na * 4;
  d.a_o_rowslot = o;
  o += na * 4;
  d.a_o_fact = o;
  o += na * 4;
  d.a_o_ifact = o;
  o += na * 4;
  d.a_smem = o;
  d.ok = true;
  return RC_OK;
}

bool tile_fwd_applies(const TileDev &d, int n) {
  return d.ok && n % 4 == 0 && d.f_smem <= 227 * 1024;
}
bool tile_adj_applies(const TileDev &d, int n) {
  return d.ok && n % 4 == 0 && d.a_smem <= 227 * 1024;
}

int bell_fwd_tile(const TileDev &d, const DevTables &t, int n, int npts, const void *S, void *T,
                  void *h, bool train, cudaStream_t st) {
  if (!tile_fwd_applies(d, n)) return RC_UNSUPPORTED;
  Fwd10Args a;
  a.n = n; a.na = d.na; a.npts = npts; a.gy = (n + 31) / 32; a.k = d.k; a.iact = t.iact;
  a.nunit = d.nfunit; a.nrec = d.nfrec;
  a.o_s1 = d.na * 128; a.o_d0 = d.f_o_d0; a.o_d1 = d.f_o_d1; a.o_sig = d.f_o_sig;
  a.o_list = d.f_o_list; a.o_unit = d.f_o_unit; a.o_rec = d.f_o_rec; a.o_perm = d.f_o_perm;
  a.o_rowslot = d.f_o_rowslot; a.o_fact = d.f_o_fact; a.o_ifact = d.f_o_ifact;
  a.tpc = t.tpc; a.list = d.flist; a.unit = (const int4 *)d.funit; a.rec = d.frec;
  a.perm = d.perm; a.rowslot = d.rowslot; a.fact = d.fact; a.ifact = d.ifact;
  a.S = (const float *)S; a.T = (float *)T; a.h = (float *)h;
  const void *k = d.td == 2 ? (train ? (const void *)k_bell_fwd10<2, true> : (const void *)k_bell_fwd10<2, false>)
                            : (train ? (const void *)k_bell_fwd10<1, true> : (const void *)k_bell_fwd10<1, false>);
  CKT(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, d.f_smem));
  const int grid = grid_for(k, TWF * 32, d.f_smem, (long)npts * a.gy);
  if (d.td == 2) {
    if (train) { LAUNCH("k_bell_fwd", st, (k_bell_fwd10<2, true><<<grid, TWF * 32, d.f_smem, st>>>(a))); }
    else { LAUNCH("k_bell_fwd", st, (k_bell_fwd10<2, false><<<grid, TWF * 32, d.f_smem, st>>>(a))); }
  } else {
    if (train) { LAUNCH("k_bell_fwd", st, (k_bell_fwd10<1, true><<<grid, TWF * 32, d.f_smem, st>>>(a))); }
    else { LAUNCH("k_bell_fwd", st, (k_bell_fwd10<1, false><<<grid, TWF * 32, d.f_smem, st>>>(a))); }
  }
  CKT(cudaGetLastError());
  return RC_OK;
}

int bell_adj_tile(const TileDev &d, int n, int npts, const void *Tb, const void *h, void *Sb,
                  double *gbias, int gstride, cudaStream_t st) {
  if (!tile_adj_applies(d, n)) return RC_UNSUPPORTED;
  Adj10Args a;
  a.n = n; a.na = d.na; a.npts = npts; a.gy = (n + 31) / 32; a.gstride = gstride;
  a.nunit = d.naunit; a.nrec = d.narec; a.nfin = d.nafin; a.nscr = std::max(1, d.nscratch);
  a.o_b1 = 2 * d.na * 128; a.o_scr = d.a_o_scr; a.o_list = d.a_o_list; a.o_unit = d.a_o_unit;
  a.o_rec = d.a_o_rec; a.o_flist = d.a_o_flist; a.o_fin = d.a_o_fin; a.o_perm = d.a_o_perm;
  a.o_rowslot = d.a_o_rowslot; a.o_fact = d.a_o_fact; a.o_ifact = d.a_o_ifact;
  a.list = d.alist; a.unit = (const int4 *)d.aunit; a.rec = d.arec; a.flist = d.aflist;
  a.fin = (const int4 *)d.afin; a.perm = d.perm; a.rowslot = d.rowslot; a.fact = d.fact;
  a.ifact = d.ifact; a.Tb = (const float *)Tb; a.h = (const float *)h; a.Sb = (float *)Sb;
  a.gbias = gbias;
  const void *k = d.td == 2 ? (const void *)k_bell_adj10<2> : (const void *)k_bell_adj10<1>;
  CKT(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, d.a_smem));
  const int grid = grid_for(k, TWA * 32, d.a_smem, (long)npts * a.gy);
  if (d.td == 2) {
    LAUNCH("k_bell_adj", st, (k_bell_adj10<2><<<grid, TWA * 32, d.a_smem, st>>>(a)));
  } else {
    LAUNCH("k_bell_adj", st, (k_bell_adj10<1><<<grid, TWA * 32, d.a_smem, st>>>(a)));
  }
  CKT(cudaGetLastError());
  return RC_OK;
}

}  // namespace dnnf90
