// bell_plan.hpp - work lists of the warp-cooperative Bell kernels.
//
// The forward recurrence of lib/train_module.f90:303-325,
//   B_{a,q} = sum_{b in fq(a,q)} C(a,b)/q S_b B_{a-b,q-1},
//   T_a = sum_q sigma^(q) B_{a,q},  h_a = sum_q sigma^(q+1) B_{a,q},
// is regrouped by b: for one output a the same sub-multi-index b serves
// every level q <= p - |b| + 1, so one "group" {b, g = a - b, C(a,b),
// qmax} feeds up to K-1 register accumulators.  Multi-indices of one
// degree are independent of each other, so each degree is a phase whose
// outputs are spread over the workers (warps) of a block, balanced by work.
//
// The adjoint (:381-403) has no recurrence: every Sb_b is one sum over
// a >= b of C(a,b) Tb_a h_{a-b}; Sb_0 is the sum of Tb_a h_a.
#pragma once
#include <cstdint>
#include <vector>

#include "tables.hpp"

namespace dnnf90 {

// Adjoint v7, grouped correlation.  Outputs whose lists {g : b + g
// carried} are equal (for a dense set: every b of one degree; output 0
// pairs every a with itself) form units of up to nkmax outputs that share
// each h_g load:  acc_k += (a! Tb)_{b_k + g} (h/g!)_g  over a range of the
// group's g list.  A group whose list is long is split over several units;
// their partial sums meet in a shared scratch row per output.
struct A7Plan {
  std::vector<int> list;        // [workers][2]: start, count into unit
  std::vector<int> unit;        // [*][8]: record start (words, 4-aligned), ng,
                                //   nk | partial << 8, out start, g-list start, 0, 0, 0
  std::vector<int> out;         // output slot | scratch row << 16
  std::vector<uint32_t> glist;  // byte offsets of the h rows, per group
  std::vector<uint32_t> rec;    // per unit and g: a7_stride(nk) words of Tb row offsets
  std::vector<int> fin;         // [*][2]: output slot, scratch row (split outputs)
  int nscratch = 0;
  bool ok = false;
};

// Forward v8: the v5 recurrences with one 32-bit record per (b, g) pair,
//   x << 16 | z / 4,
// x the byte offset of the S_b/b! row inside the current S buffer and z the
// byte offset of g's first row inside its region: the S buffer for |g| = 1,
// the B region for 2 <= |g| <= K-2 (levels 1..|g| of B_{g,q}/g!, level 1 a
// copy of S_g/g!), the U/V region on the top degree.  A U/V pair is one
// 256-byte row holding (U_g/g!, V_g/g!) side by side for each lane.
// Shared memory: two S buffers of na + 1 rows (row na stays zero), the B
// region, the U/V region (with a zero pair), K+2 sigma rows, the records.
struct F8Plan {
  std::vector<int> list;       // [(k+1) * workers][2]: first target, count
  std::vector<int> hdr;        // [*][8]: ia, rstart, nrec, B run of a (or -1),
                               //   U/V pair of a (or -1), bands D=1..4, D=5..8, 0
  std::vector<uint32_t> rec;   // records; top-degree lists 4-aligned, padded
                               //   with (zero S row, zero U/V pair)
  std::vector<int> cpdst;      // [na]: B-region offset of the level-1 copy, or -1
  int srows = 0, sbase1 = 0, bbase = 0, uvbase = 0, dtbase = 0, recbase = 0;
  int zuv = 0;                 // U/V-region offset of the zero pair
  int smem = 0;                // bytes of shared memory
  bool ok = false;
};

// The tanh forward by the series identity of tanh' = 1 - tanh^2 (v9).
// With t~, u~ and s~ the factorial-normalised series of T, h = 1 - T^2 and
// S, Euler's relation gives, degree by degree,
//   |a| t~_a = sum_{0<b<=a} |b| s~_b u~_{a-b},
//   u~_a = -sum_{b+c=a} t~_b t~_c,
// and the two sums over the ordered pairs (b, c), b + c = a, b, c != 0, run
// as one packed multiply-add of (|b| s~_b, t~_b) by (u~_c, t~_c).  Shared
// memory: S rows [na+1][128 B]; P rows (|b| s~_b, t~_b) and Q rows
// (u~_c, t~_c), [na+1][256 B] each (row na zero).  Needs a downward-closed
// set (every b <= a carried).
struct F9Plan {
  std::vector<int> list;       // [(k+1) * workers][2]: first target, count
  std::vector<int> hdr;        // [*][4]: ia, first record, records (even), 0
  std::vector<uint32_t> rec;   // [*][2]: byte offsets of the P row of b and the Q row of c
  std::vector<double> sdeg;    // [na]: |a| / a!
  int pbase = 0, qbase = 0, smem = 0;
  bool ok = false;
};

struct BellPlan {
  int workers = 0, k = 0, na = 0, nslot = 0;
  F8Plan f8;
  F9Plan f9;
  // forward
  std::vector<int> fw_list;   // [(k+1) * workers][2]: start, count into fw_arec
  std::vector<int> fw_arec;   // [*][4]: ia | p << 16, gstart, gcount, bbase
  std::vector<int> fw_grec;   // [*][4]: ib, g, gbase (state slot of B_{g,2}), qmax
  std::vector<double> fw_gc;  // C(a,b) per group
  std::vector<int> bbase;     // [na]: state slot of B_{a,2} (or -1)
  // forward, v3 (top degree by the U/V convolution, banded groups, byte
  // offsets into the shared-memory state; one state row = 128 bytes)
  int nrows = 0;              // state rows: S | B | U | V | sigma
  std::vector<int> f3_list;   // [(k+1) * workers][2]
  std::vector<int> f3_arec;   // [*][8]: ia | p << 16, gstart, gcount, band_hi,
                              //         b_off, u_off, v_off, band_lo
  std::vector<int> f3_grec;   // [*][4]: s_b off, s_g off, B_g (or U_g) off, V_g off
  std::vector<double> f3_gc;  // C(a,b)
  int dt_off = 0;             // byte offset of the sigma rows
  bool f3_ok = false;         // every band fits its 8-bit count
  // forward v4: the same work lists over factorial-normalised state
  // (rows hold S_b/b!, B_{a,q}/a!, U_g/g!, V_g/g!), so no coefficient is
  // needed; one 32-bit record per group:
  //   p < K : ib | g << 10 | (first row of the B run of g) << 20
  //   p = K : ib | (U row of g) << 10         (V row = U row + nuv)
  std::vector<uint32_t> f4_grec;
  int nuv = 0;
  // forward v5: the v4 work lists with flat records of two byte offsets
  // into the shared state, no decoding in the inner loop.  Rows:
  //   [0, na)       S_b / b!                         (double-buffered)
  //   B run of g    levels 1..|g| of B_{g,q} / g!, level 1 a copy of S_g/g!
  //                 (2 <= |g| <= K-2)
  //   U/V pair of g U_g/g! and, in the next row, V_g/g!  (1 <= |g| <= K-1)
  //   sigma         K+2 rows of sigma^(q)
  // Records (uint2):
  //   p < K : (S row of b, first level row of g)  -- level l at + (l-1) rows;
  //           for |g| = 1 the level-1 row is S_g itself (S region)
  //   p = K : (S row of b, U row of g)            -- V one row further
  int nrows5 = 0, dt_off5 = 0;
  int zuv5 = 0;                    // byte offset of the zero U/V pair
  // top-degree lists (p = K) start on a 4-record boundary and are padded to a
  // multiple of 4 with (S row 0, zero U/V pair) records
  bool f5_ok = false;
  std::vector<int> f5_list;        // [(k+1) * workers][2]: start, count into f5_arec
  std::vector<int> f5_arec;        // [*][8]: ia | p << 16, rstart, rcount, band_hi,
                                   //         B run of a (or -1), U/V pair of a (or -1), 0, band_lo
  std::vector<uint32_t> f5_rec;    // [*][2]
  std::vector<int> f5_cpdst;       // [na]: byte offset of the level-1 copy of S_a, or -1
  std::vector<uint32_t> f6_rec;    // the f5 records as rows: x row | z row << 16
  // adjoint v7, grouped correlation (A7Plan): FP32 units of up to 16
  // outputs, FP64 units of up to 8 (one lane's accumulators in registers)
  A7Plan a7f, a7d;
  // adjoint, v3: Sb_b b! = sum_{a >= b} (a! Tb_a) (h_{a-b} / (a-b)!), the
  // pair coefficient C(a,b) = a!/(b!(a-b)!) folded into per-row scales
  std::vector<int> a3_orec;   // [*][4]: ib, pstart, pcount, 0
  std::vector<int> a3_pair;   // [*][2]: byte offsets of the Tb and h rows
  std::vector<uint32_t> a4_pair;  // [*]: Tb row | h row << 16
  std::vector<double> fact;   // a! per slot
  // adjoint
  std::vector<int> aj_list;   // [workers][2]
  std::vector<int> aj_orec;   // [*][4]: ib, pstart, pcount, 0
  std::vector<int> aj_pair;   // [*]: ia | id << 16
  std::vector<double> aj_c;
};

BellPlan build_bell_plan(const TableSet &t, int workers, int aj_workers);
// words per g of a v7 unit's records: nk, or nk rounded up to 4 above 2
int a7_stride(int nk);

}  // namespace dnnf90
