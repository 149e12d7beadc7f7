// The register-tiled Bell kernels' plan (TilePlan) on the CPU: the layout
// is a permutation of the slots, every unit's records point inside the
// buffers the kernel reads, and the Horner forward and the tiled
// correlation adjoint, run over the records in the kernels' own loop order
// (FP64 here), reproduce the Bell recurrence and the pair sums over the
// table set's own lists (lib/train_module.f90:297-325, 381-403) to 1e-12.
// Built and run by tests/test_tile_plan.py.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <random>
#include <vector>

#include "tables.hpp"
#include "tile_plan.hpp"
using namespace dnnf90;

static int tri_deg(int td, int e) {
  if (td == 1) return e;
  int s = 0;
  while ((s + 1) * (s + 2) / 2 <= e) ++s;
  return s;
}
static void untri(int td, int e, int &a1, int &a2) {
  if (td == 1) { a1 = e; a2 = 0; return; }
  int s = tri_deg(td, e);
  a2 = e - s * (s + 1) / 2;
  a1 = s - a2;
}
static int tri(int td, int a1, int a2) {
  if (td == 1) return a1;
  int s = a1 + a2;
  return s * (s + 1) / 2 + a2;
}

static int check(int d0, int k) {
  TableSet t;
  std::string err = build_tables(d0, k, 0, nullptr, t);
  if (!err.empty()) { printf("tables: %s\n", err.c_str()); return 1; }
  TilePlan P = build_tile_plan(t, TILE_WARPS_F, TILE_WARPS_A);
  const int na = t.na, td = P.td;
  printf("d0=%d k=%d na=%d ok=%d td=%d fwd fma2 %ld loads %ld, adj fma %ld loads %ld, "
         "units fwd %zu adj %zu, scratch %d, bufs %d %d\n",
         d0, k, na, P.ok, td, P.fwd_fma2, P.fwd_loads, P.adj_fma, P.adj_loads,
         P.funit.size() / 4, P.aunit.size() / 4, P.nscratch, P.nbuf[0], P.nbuf[1]);
  if (!P.ok) return k <= TILE_KMAX ? 1 : 0;
  std::vector<int> seen(na, 0);
  for (int ia = 0; ia < na; ++ia) {
    if (P.perm[ia] < 0 || P.perm[ia] >= na || P.rowslot[P.perm[ia]] != ia) { printf("perm\n"); return 1; }
    seen[P.perm[ia]]++;
  }
  for (int r = 0; r < na; ++r) if (seen[r] != 1) { printf("row %d\n", r); return 1; }
  std::vector<double> fact(na, 1.0);
  for (int ia = 0; ia < na; ++ia)
    for (int j = 0; j < d0; ++j)
      for (int v = 2; v <= t.alpha[ia * d0 + j]; ++v) fact[ia] *= v;

  std::mt19937_64 g(11 + d0 * 10 + k);
  std::normal_distribution<double> nd(0, 0.7);
  // ---------------- forward
  std::vector<double> S(na);
  for (auto &v : S) v = nd(g);
  const int ld = k + 3;
  double tt = std::tanh(S[0]);
  std::vector<double> sg(k + 2);
  for (int q = 0; q <= k + 1; ++q) {
    double v = t.tpc[q * ld + q + 1];
    for (int i = q; i >= 0; --i) v = v * tt + t.tpc[q * ld + i];
    sg[q] = v;
  }
  std::vector<std::vector<double>> B(na, std::vector<double>(k + 1, 0.0));
  std::vector<double> Tr(na), Hr(na);
  Tr[0] = sg[0];
  Hr[0] = sg[1];
  for (int ia = 1; ia < na; ++ia) {
    B[ia][1] = S[ia];
    for (int q = 2; q <= t.deg[ia]; ++q) {
      double s = 0;
      for (int i = t.fq_at(ia, q); i < t.fq_at(ia, q) + t.fq_len(ia, q); ++i)
        s += t.fq_c[i] * S[t.fq_ib[i]] * B[t.fq_id[i]][q - 1];
      B[ia][q] = s;
    }
    double a = 0, b = 0;
    for (int q = 1; q <= t.deg[ia]; ++q) { a += sg[q] * B[ia][q]; b += sg[q + 1] * B[ia][q]; }
    Tr[ia] = a;
    Hr[ia] = b;
  }
  std::vector<double> srow(na);
  for (int ia = 0; ia < na; ++ia) srow[P.perm[ia]] = ia ? S[ia] / fact[ia] : S[ia];
  std::vector<std::vector<double>> DB[2];
  for (int b = 0; b < 2; ++b) DB[b].assign(std::max(1, P.nbuf[b]), std::vector<double>(2, NAN));
  DB[k & 1][0] = {sg[k], sg[k + 1]};
  std::vector<double> To(na, NAN), Ho(na, NAN);
  for (int q = k - 1; q >= 0; --q) {
    const int nw = P.fwarps;
    for (int w = 0; w < nw; ++w) {
      const int u0 = P.flist[((size_t)q * nw + w) * 2], un = P.flist[((size_t)q * nw + w) * 2 + 1];
      for (int u = u0; u < u0 + un; ++u) {
        const int L = P.funit[4 * u] & 0xff, origin = P.funit[4 * u] >> 8;
        const int r0 = P.funit[4 * u + 1], rn = P.funit[4 * u + 2], out = P.funit[4 * u + 3];
        const int NT = tile_size(td, L);
        std::vector<double> ax(NT, 0.0), ay(NT, 0.0);
        for (int r = r0; r < r0 + rn; ++r) {
          const int sr = P.frec[r] & 0xffff, dr = P.frec[r] >> 16;
          const bool z = r == r0;
          const int LD = z ? L - 1 : L;
          if (sr + NT > na) { printf("s rows\n"); return 1; }
          if (LD > 0 && dr + tile_size(td, LD) > P.nbuf[(q + 1) & 1]) { printf("d rows\n"); return 1; }
          for (int c = 0; c < tile_size(td, LD); ++c) {
            const double dx = DB[(q + 1) & 1][dr + c][0], dy = DB[(q + 1) & 1][dr + c][1];
            int c1, c2;
            untri(td, c, c1, c2);
            for (int e = z ? 1 : 0; e < tile_size(td, L - tri_deg(td, c)); ++e) {
              int b1, b2;
              untri(td, e, b1, b2);
              const int o = tri(td, b1 + c1, b2 + c2);
              ax[o] += srow[sr + e] * dx;
              ay[o] += srow[sr + e] * dy;
            }
          }
        }
        for (int e = 0; e < NT; ++e) { ax[e] /= (q + 1); ay[e] /= (q + 1); }
        if (origin) { ax[0] = sg[q]; ay[0] = sg[q + 1]; }
        for (int e = 0; e < NT; ++e) {
          if (q > 0) {
            if (out + e >= P.nbuf[q & 1]) { printf("out rows\n"); return 1; }
            DB[q & 1][out + e] = {ax[e], ay[e]};
          } else {
            const int ia = P.rowslot[out + e];
            To[ia] = ax[e] * fact[ia];
            Ho[ia] = ay[e] * fact[ia];
          }
        }
      }
    }
  }
  double et = 0, mt = 0, eh = 0, mh = 0;
  for (int ia = 0; ia < na; ++ia) {
    if (std::isnan(To[ia])) { printf("slot %d not written\n", ia); return 1; }
    et = std::max(et, std::fabs(To[ia] - Tr[ia]));
    mt = std::max(mt, std::fabs(Tr[ia]));
    eh = std::max(eh, std::fabs(Ho[ia] - Hr[ia]));
    mh = std::max(mh, std::fabs(Hr[ia]));
  }
  printf("  forward: T %.2e h %.2e\n", et / mt, eh / mh);
  if (et / mt > 1e-12 || eh / mh > 1e-12) return 1;

  // ---------------- adjoint
  std::vector<double> Tb(na), h(na);
  for (auto &v : Tb) v = nd(g);
  for (auto &v : h) v = nd(g);
  std::vector<double> Sr(na, 0.0);
  for (int ia = 0; ia < na; ++ia) Sr[0] += Tb[ia] * h[ia];
  for (int ib = 1; ib < na; ++ib)
    for (int i = t.pair_start[ib]; i < t.pair_start[ib] + t.pair_num[ib]; ++i)
      Sr[ib] += t.pair_binom[i] * Tb[t.pair_ia[i]] * h[t.pair_id[i]];
  std::vector<double> tbn(na), hn(na), So(na, NAN);
  for (int ia = 0; ia < na; ++ia) {
    tbn[P.perm[ia]] = Tb[ia] * fact[ia];
    hn[P.perm[ia]] = h[ia] / fact[ia];
  }
  std::vector<double> scr((size_t)P.nscratch, NAN);
  for (int w = 0; w < P.awarps; ++w) {
    for (int u = P.alist[2 * w]; u < P.alist[2 * w] + P.alist[2 * w + 1]; ++u) {
      const int Lout = P.aunit[4 * u] & 0xff, split = P.aunit[4 * u] >> 8;
      const int r0 = P.aunit[4 * u + 1], out = P.aunit[4 * u + 3];
      const uint32_t cw = (uint32_t)P.aunit[4 * u + 2];
      const int NT = tile_size(td, Lout);
      std::vector<double> acc(NT, 0.0);
      // the kernel's order: for E = 0 .. Lout-1, the unit's records of tile side Lout - E
      int r = r0;
      for (int E = 0; E < Lout; ++E)
      for (int cnt = (cw >> (4 * E)) & 15; cnt > 0; --cnt, ++r) {
        const int hr = P.arec[r] & 0x3fff, tr = (P.arec[r] >> 14) & 0x3fff, L = P.arec[r] >> 28;
        if (L != Lout - E) { printf("adj record side\n"); return 1; }
        if (L > Lout || hr + tile_size(td, L) > na || tr + tile_size(td, L) > na) { printf("adj rec\n"); return 1; }
        for (int a = 0; a < tile_size(td, L); ++a) {
          int a1, a2;
          untri(td, a, a1, a2);
          for (int c1 = 0; c1 <= a1; ++c1)
            for (int c2 = 0; c2 <= a2; ++c2)
              acc[tri(td, a1 - c1, a2 - c2)] += tbn[tr + a] * hn[hr + tri(td, c1, c2)];
        }
      }
      for (int e = 0; e < NT; ++e) {
        if (split) {
          if (out + e >= P.nscratch) { printf("scratch\n"); return 1; }
          scr[out + e] = acc[e];
        } else {
          const int ib = P.rowslot[out + e];
          So[ib] = acc[e] / fact[ib];
        }
      }
    }
  }
  for (int w = 0; w < P.awarps; ++w)
    for (int f = P.aflist[2 * w]; f < P.aflist[2 * w] + P.aflist[2 * w + 1]; ++f) {
      const int row = P.afin[4 * f], np = P.afin[4 * f + 1], s0 = P.afin[4 * f + 2], st = P.afin[4 * f + 3];
      double v = 0;
      for (int p = 0; p < np; ++p) {
        if (s0 + p * st >= P.nscratch) { printf("fin scratch\n"); return 1; }
        v += scr[s0 + p * st];
      }
      const int ib = P.rowslot[row];
      So[ib] = v / fact[ib];
    }
  double es = 0, ms = 0;
  for (int ia = 0; ia < na; ++ia) {
    if (std::isnan(So[ia])) { printf("adjoint slot %d not written\n", ia); return 1; }
    es = std::max(es, std::fabs(So[ia] - Sr[ia]));
    ms = std::max(ms, std::fabs(Sr[ia]));
  }
  printf("  adjoint: Sb %.2e\n", es / ms);
  return es / ms > 1e-12;
}

int main() {
  int bad = 0;
  for (int d0 = 1; d0 <= 4; ++d0)
    for (int k = 1; k <= 8; ++k) bad += check(d0, k);
  if (!bad) printf("ALL OK\n");
  return bad ? 1 : 0;
}
