// The tanh series forward's plan (F9Plan) on the CPU: every multi-index
// of degree >= 1 is listed once, in its degree's work lists; every record
// points inside the P and Q row regions; and the recurrence run over the
// records, as the kernel runs it, reproduces the Bell recurrence over the
// table set's own lists (lib/train_module.f90:297-325) to 1e-12.  Built and
// run by tests/test_series_plan.py.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <random>
#include <vector>
#include "bell_plan.hpp"
#include "tables.hpp"
using namespace dnnf90;
int check(int d0, int k, int nseed, const int *seeds) {
  TableSet t;
  std::string err = build_tables(d0, k, nseed, seeds, t);
  if (!err.empty()) { printf("tables: %s\n", err.c_str()); return 1; }
  BellPlan bp = build_bell_plan(t, 32, 32);
  const F9Plan &P = bp.f9;
  const int na = t.na;
  printf("d0=%d k=%d na=%d ok=%d smem=%d records=%zu\n", d0, k, na, P.ok, P.smem, P.rec.size() / 2);
  if (!P.ok) return 0;
  std::vector<int> seen(na, 0);
  for (int p = 1; p <= k; ++p)
    for (int w = 0; w < 32; ++w) {
      int s0 = P.list[(p * 32 + w) * 2], n = P.list[(p * 32 + w) * 2 + 1];
      for (int h = s0; h < s0 + n; ++h) {
        int ia = P.hdr[h * 4], rs = P.hdr[h * 4 + 1], nr = P.hdr[h * 4 + 2];
        if (t.deg[ia] != p || rs % 2 || nr % 2) { printf("bad hdr\n"); return 1; }
        seen[ia]++;
        for (int r = rs; r < rs + nr; ++r) {
          uint32_t x = P.rec[2 * r], y = P.rec[2 * r + 1];
          if (x < (uint32_t)P.pbase || x >= (uint32_t)(P.pbase + (na + 1) * 256) || (x - P.pbase) % 256) { printf("bad x\n"); return 1; }
          if (y < (uint32_t)P.qbase || y >= (uint32_t)(P.qbase + (na + 1) * 256) || (y - P.qbase) % 256) { printf("bad y\n"); return 1; }
        }
      }
    }
  for (int ia = 1; ia < na; ++ia) if (seen[ia] != 1) { printf("slot %d seen %d\n", ia, seen[ia]); return 1; }
  // emulate: random S, tanh series by the records vs the Bell recurrence
  std::mt19937_64 g(7); std::normal_distribution<double> nd(0, 0.7);
  std::vector<double> S(na); for (auto &v : S) v = nd(g);
  // sigma^(q)
  const int ld = k + 3; double tt = std::tanh(S[0]); std::vector<double> sg(k + 2);
  for (int q = 0; q <= k + 1; ++q) { double v = t.tpc[q * ld + q + 1]; for (int i = q; i >= 0; --i) v = v * tt + t.tpc[q * ld + i]; sg[q] = v; }
  // Bell: B[a][q]
  std::vector<std::vector<double>> B(na, std::vector<double>(k + 1, 0.0));
  std::vector<double> Tb(na), Hb(na);
  Tb[0] = sg[0]; Hb[0] = sg[1];
  for (int ia = 1; ia < na; ++ia) {
    B[ia][1] = S[ia];
    for (int q = 2; q <= t.deg[ia]; ++q) {
      double s = 0; for (int i = t.fq_at(ia, q); i < t.fq_at(ia, q) + t.fq_len(ia, q); ++i) s += t.fq_c[i] * S[t.fq_ib[i]] * B[t.fq_id[i]][q - 1];
      B[ia][q] = s;
    }
    double a = 0, b = 0; for (int q = 1; q <= t.deg[ia]; ++q) { a += sg[q] * B[ia][q]; b += sg[q + 1] * B[ia][q]; }
    Tb[ia] = a; Hb[ia] = b;
  }
  // series by the plan (rows indexed by offset)
  std::vector<double> fact(na, 1.0);
  for (int ia = 0; ia < na; ++ia) for (int i = 0; i < d0; ++i) for (int v = 2; v <= t.alpha[ia * d0 + i]; ++v) fact[ia] *= v;
  std::vector<double> Px(na + 1, 0), Py(na + 1, 0), Qx(na + 1, 0), Qy(na + 1, 0);
  for (int ia = 1; ia < na; ++ia) Px[ia] = S[ia] * P.sdeg[ia];
  double t0 = sg[0], u0 = sg[1];
  std::vector<double> T9(na), H9(na); T9[0] = t0; H9[0] = u0;
  for (int p = 1; p <= k; ++p)
    for (int w = 0; w < 32; ++w) {
      int s0 = P.list[(p * 32 + w) * 2], n = P.list[(p * 32 + w) * 2 + 1];
      for (int h = s0; h < s0 + n; ++h) {
        int ia = P.hdr[h * 4], rs = P.hdr[h * 4 + 1], nr = P.hdr[h * 4 + 2];
        double aT = 0, aU = 0;
        for (int r = rs; r < rs + nr; ++r) {
          int b = (P.rec[2 * r] - P.pbase) / 256, c = (P.rec[2 * r + 1] - P.qbase) / 256;
          aT += Px[b] * Qx[c]; aU += Py[b] * Qy[c];
        }
        double tv = (aT + Px[ia] * u0) / p, uv = -(aU + 2 * t0 * tv);
        Py[ia] = tv; Qx[ia] = uv; Qy[ia] = tv;
        T9[ia] = fact[ia] * tv; H9[ia] = fact[ia] * uv;
      }
    }
  double et = 0, eh = 0, mt = 0, mh = 0;
  for (int ia = 0; ia < na; ++ia) { et = std::max(et, std::fabs(T9[ia] - Tb[ia])); eh = std::max(eh, std::fabs(H9[ia] - Hb[ia])); mt = std::max(mt, std::fabs(Tb[ia])); mh = std::max(mh, std::fabs(Hb[ia])); }
  printf("  rel err T %.3e h %.3e\n", et / mt, eh / mh);
  return et / mt > 1e-12 || eh / mh > 1e-12;
}
int main() {
  int rc = 0;
  rc |= check(4, 7, 0, nullptr);
  rc |= check(4, 3, 0, nullptr);
  rc |= check(2, 2, 0, nullptr);
  int kdv[] = {0, 1, 1, 0, 3, 0};
  rc |= check(2, 3, 3, kdv);
  int heat[] = {1, 0, 0, 0, 2, 0, 0, 0, 2};
  rc |= check(3, 2, 3, heat);
  rc |= check(4, 8, 0, nullptr);
  rc |= check(3, 1, 0, nullptr);
  printf(rc ? "FAIL\n" : "ALL OK\n");
  return rc;
}
