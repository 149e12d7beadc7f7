// tile_plan.hpp - work lists of the register-tiled Bell kernels (bell_tile.cu).
//
// Forward.  With s~ the factorial-normalised series of S without its
// value (s~_a = S_a / a!, s~_0 = 0) and sigma_q = sigma^(q)(S_0), the
// carried derivatives T_a = a! t~_a, h_a = a! h~_a of
// lib/train_module.f90:297-325 are the two Horner recurrences
//   D_K = sigma_K,      D_q = sigma_q   + (s~ * D_{q+1}) / (q + 1),
//   E_K = sigma_{K+1},  E_q = sigma_{q+1} + (s~ * E_{q+1}) / (q + 1),
// t~ = D_0, h~ = E_0, where * is the product of truncated series (the
// Cauchy product over multi-indices) and D_q is needed up to degree K - q
// only, because s~ has no constant term.  Both chains multiply by the same
// s~, so one step is one product with (D, E) pairs: K steps of
//   c_a = sum_{0 < b <= a} s~_b (D, E)_{a-b},  |a| <= K - q.
// This is the Faa di Bruno sum of the reference regrouped (sum over q of
// sigma_q B_{a,q}, B_q = s~^q / q!), evaluated innermost-first.
//
// Adjoint (lib/train_module.f90:381-403): every Sb_b is one correlation,
//   Sb_b b! = sum_{g : b + g carried} (a! Tb_a) (h_g / g!),  a = b + g.
//
// Tiling.  A dense set (every multi-index of degree <= K) is laid out as
// tiles over its first td dimensions (td = 2: triangles a1 + a2 <= L - 1;
// td = 1: lines a1 <= L - 1), one tile per outer index (the remaining
// dimensions).  Inside a tile the entries are in graded order, so the
// entries of degree <= L' - 1 are a prefix of it.  A product restricted to
// one outer index of the output, one of the first factor and one of the
// second is then a small dense product of tiles that a thread runs from
// registers: the tile of s~ (or of h~) held in registers, the tile of the
// other factor streamed from shared memory, each loaded value feeding every
// output of the tile it reaches.  A record names one such (factor tile,
// factor tile) pair; a unit is one output tile with its records.
#pragma once
#include <cstdint>
#include <vector>

#include "tables.hpp"

namespace dnnf90 {

// warps per block of the tiled forward and of the tiled adjoint (at most 128
// registers each)
constexpr int TILE_WARPS_F = 16;
constexpr int TILE_WARPS_A = 16;
constexpr int TILE_KMAX = 7;    // longest tile side is K + 1 <= 8

struct TilePlan {
  bool ok = false;
  int td = 0;                   // tile dimensions: 1 (lines) or 2 (triangles)
  int d0 = 0, k = 0, na = 0, fwarps = 0, awarps = 0;
  std::vector<int> perm;        // [na]: row of slot ia in the tile layout of the full set
  std::vector<int> rowslot;     // [na]: slot of each row (the inverse)
  std::vector<int> tbase;       // per outer index: first row of its tile (full set)
  // forward: Horner step q (q = K-1 .. 0) is phase q of the kernel
  int nbuf[2] = {0, 0};         // rows of the two (D, E) buffers; D_q sits in buffer q & 1
  std::vector<int> flist;       // [k][fwarps][2]: first unit, units of each warp in step q
  std::vector<int> funit;       // [*][4]: L | (output tile is the origin's) << 8,
                                //   first record, records, first output row
                                //   (buffer q & 1 for q > 0, the full layout for q = 0)
  std::vector<uint32_t> frec;   // s~ tile row | D tile row << 16; a unit's first
                                //   record is the one whose s~ tile holds the origin
  // adjoint: one phase of units, then one of split outputs
  std::vector<int> alist;       // [awarps][2]
  std::vector<int> aunit;       // [*][4]: Lout | split << 8, first record, record
                                //   counts (4 bits per E: records of tile side
                                //   Lout - E, in that order), first output row
                                //   (full layout) or scratch row
  std::vector<uint32_t> arec;   // h tile row | Tb tile row << 14 | L << 28
  std::vector<int> afin;        // [*][4] per element of a split output tile: its row
                                //   (full layout), parts, first scratch row, part stride
  std::vector<int> aflist;      // [awarps][2] into afin
  int nscratch = 0;             // scratch rows of the split outputs
  // work model (diagnostic): multiply-adds and shared loads per item
  long fwd_fma2 = 0, fwd_loads = 0, adj_fma = 0, adj_loads = 0;
};

// The plan of a dense table set with 1 <= K <= TILE_KMAX (ok = false
// otherwise, and the caller keeps the general kernels).
TilePlan build_tile_plan(const TableSet &t, int fwarps, int awarps);

// entries of a tile of side L
inline int tile_size(int td, int L) { return td == 2 ? L * (L + 1) / 2 : L; }

}  // namespace dnnf90
