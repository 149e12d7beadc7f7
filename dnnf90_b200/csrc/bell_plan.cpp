// bell_plan.cpp - see bell_plan.hpp.
#include "bell_plan.hpp"

#include <algorithm>
#include <unordered_map>
#include <cmath>
#include <map>
#include <numeric>

namespace dnnf90 {

namespace {

// longest-processing-time assignment of items (by cost) to workers
std::vector<std::vector<int>> balance(const std::vector<long> &cost, int workers) {
  std::vector<int> order(cost.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<long> load(workers, 0);
  std::vector<std::vector<int>> out(workers);
  for (int i : order) {
    int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[w] += cost[i];
    out[w].push_back(i);
  }
  for (auto &v : out) std::sort(v.begin(), v.end());  // reference order inside a worker
  return out;
}

}  // namespace

int a7_stride(int nk) { return nk <= 2 ? nk : (nk + 3) / 4 * 4; }

// the v7 adjoint plan with units of at most nkmax outputs
static A7Plan build_a7(const TableSet &t, int aj_workers, int nkmax) {
  A7Plan P;
  const int na = t.na;
    const int ROW = 128;
    // g list of every output (output 0 pairs every a with itself, g = a)
    std::map<std::vector<int>, std::vector<int>> groups;
    {
      std::vector<int> all(na);
      std::iota(all.begin(), all.end(), 0);
      groups[all].push_back(0);
    }
    for (int ib = 1; ib < na; ++ib) {
      std::vector<int> gl;
      for (int ip = t.pair_start[ib]; ip < t.pair_start[ib] + t.pair_num[ib]; ++ip)
        gl.push_back(t.pair_id[ip]);
      std::sort(gl.begin(), gl.end());
      groups[gl].push_back(ib);
    }
    long total = 0;
    for (auto &kv : groups) total += (long)kv.first.size() * kv.second.size();
    const double target = std::max(8.0, (double)total / aj_workers * 0.5);
    struct Unit {
      const std::vector<int> *gl;  // the group's g list
      int gstart, g0, ng;
      std::vector<int> outs;
      bool partial;
      long cost;
    };
    std::vector<Unit> units;
    std::vector<int> scratch_of(na, -1);
    P.nscratch = 0;
    for (auto &kv : groups) {
      const std::vector<int> &gl = kv.first, &outs = kv.second;
      const int G = (int)gl.size();
      const int gstart = (int)P.glist.size();
      for (int g : gl) P.glist.push_back((uint32_t)(na + g) * ROW);
      // up to nkmax outputs per unit, evenly spread
      const int nchunk = ((int)outs.size() + nkmax - 1) / nkmax;
      for (int c = 0; c < nchunk; ++c) {
        const size_t o0 = (size_t)c * outs.size() / nchunk, o1 = (size_t)(c + 1) * outs.size() / nchunk;
        const int nk = (int)(o1 - o0);
        // the g list split so that one unit holds about `target` products
        const int nsplit = std::max(1, (int)std::lround((double)G * nk / target));
        const int parts = std::min(nsplit, G);
        for (int sp = 0; sp < parts; ++sp) {
          Unit u;
          u.gl = &gl;
          u.gstart = gstart;
          u.g0 = (int)((long)sp * G / parts);
          u.ng = (int)((long)(sp + 1) * G / parts) - u.g0;
          u.outs.assign(outs.begin() + o0, outs.begin() + o1);
          u.partial = parts > 1;
          u.cost = (long)u.ng * (2 * nk + 2) + 16;
          units.push_back(u);
        }
        if (parts > 1)
          for (size_t o = o0; o < o1; ++o) scratch_of[outs[o]] = P.nscratch++;
      }
    }
    P.fin.clear();
    for (int b = 0; b < na; ++b)
      if (scratch_of[b] >= 0) {
        P.fin.push_back(b);
        P.fin.push_back(scratch_of[b]);
      }
    std::vector<long> cost;
    for (auto &u : units) cost.push_back(u.cost);
    auto asg = balance(cost, aj_workers);
    P.list.assign((size_t)aj_workers * 2, 0);
    for (int w = 0; w < aj_workers; ++w) {
      P.list[w * 2] = (int)P.unit.size() / 8;
      P.list[w * 2 + 1] = (int)asg[w].size();
      for (int ui : asg[w]) {
        const Unit &u = units[ui];
        const int nk = (int)u.outs.size();
        const int stride = a7_stride(nk);
        while (P.rec.size() % 4) P.rec.push_back(0);
        P.unit.push_back((int)P.rec.size());
        P.unit.push_back(u.ng);
        P.unit.push_back(nk | (u.partial ? 1 << 8 : 0));
        P.unit.push_back((int)P.out.size());
        P.unit.push_back(u.gstart + u.g0);
        P.unit.push_back(0);
        P.unit.push_back(0);
        P.unit.push_back(0);
        for (int b : u.outs) P.out.push_back(b | ((u.partial ? scratch_of[b] : 0) << 16));
        for (int gi = u.g0; gi < u.g0 + u.ng; ++gi) {
          const int g = (*u.gl)[gi];
          for (int b : u.outs) {
            int a = g;  // output 0: the partner of g is g
            if (b != 0) {
              std::vector<int> v(t.d0);
              for (int i = 0; i < t.d0; ++i)
                v[i] = t.alpha[(size_t)b * t.d0 + i] + t.alpha[(size_t)g * t.d0 + i];
              a = t.find(v.data());
            }
            P.rec.push_back((uint32_t)a * ROW);
          }
          for (int e = nk; e < stride; ++e) P.rec.push_back(0);
        }
      }
    }
    for (int i = 0; i < 16; ++i) P.rec.push_back(0);
    for (int i = 0; i < 4; ++i) P.glist.push_back(0);
    P.ok = na < 65536 && P.nscratch < 65536;
    for (size_t i = 0; i < P.rec.size(); ++i)
      if (P.rec[i] >= (uint32_t)(2 * na) * ROW) P.ok = false;
  
  return P;
}

// the v9 tanh series forward plan (see F9Plan)
static F9Plan build_f9(const TableSet &t, int workers) {
  F9Plan P;
  const int na = t.na, k = t.k, d0 = t.d0;
  P.pbase = (na + 1) * 128;
  P.qbase = P.pbase + (na + 1) * 256;
  P.smem = P.qbase + (na + 1) * 256;
  if (k > 8 || na < 1) return P;
  P.sdeg.assign(na, 0.0);
  for (int ia = 0; ia < na; ++ia) {
    double f = 1.0;
    for (int i = 0; i < d0; ++i)
      for (int v = 2; v <= t.alpha[(size_t)ia * d0 + i]; ++v) f *= v;
    P.sdeg[ia] = t.deg[ia] / f;
  }
  const uint32_t zp = (uint32_t)(P.pbase + na * 256), zq = (uint32_t)(P.qbase + na * 256);
  // slots by multi-index (digits base k + 1)
  std::unordered_map<long long, int> slot;
  auto key = [&](const int *a) {
    long long v = 0;
    for (int i = d0 - 1; i >= 0; --i) v = v * (k + 1) + a[i];
    return v;
  };
  for (int ia = 0; ia < na; ++ia) slot[key(&t.alpha[(size_t)ia * d0])] = ia;
  auto find = [&](const int *a) {
    auto f = slot.find(key(a));
    return f == slot.end() ? -1 : f->second;
  };
  // every ordered pair (b, a - b) with b != 0, a - b != 0; the set must hold both
  std::vector<std::vector<uint32_t>> recs(na);
  std::vector<int> b(d0), c(d0);
  for (int ia = 1; ia < na; ++ia) {
    if (t.deg[ia] < 2) continue;
    const int *a = &t.alpha[(size_t)ia * d0];
    // odometer over b <= a
    std::fill(b.begin(), b.end(), 0);
    while (true) {
      int i = 0;
      while (i < d0 && b[i] == a[i]) b[i++] = 0;
      if (i == d0) break;
      ++b[i];
      int db = 0;
      for (int m = 0; m < d0; ++m) {
        c[m] = a[m] - b[m];
        db += b[m];
      }
      if (db == t.deg[ia]) continue;  // c = 0
      const int ib = find(b.data()), ic = find(c.data());
      if (ib < 0 || ic < 0) return P;  // not downward closed
      recs[ia].push_back((uint32_t)(P.pbase + ib * 256));
      recs[ia].push_back((uint32_t)(P.qbase + ic * 256));
    }
    if ((recs[ia].size() / 2) % 2) {  // an even count: two records per 16-byte load
      recs[ia].push_back(zp);
      recs[ia].push_back(zq);
    }
  }
  P.list.assign((size_t)(k + 1) * workers * 2, 0);
  for (int p = 1; p <= k; ++p) {
    std::vector<int> items;
    std::vector<long> cost;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] == p) {
        items.push_back(ia);
        cost.push_back(12 + (long)recs[ia].size() / 2);
      }
    auto asg = balance(cost, workers);
    for (int w = 0; w < workers; ++w) {
      P.list[((size_t)p * workers + w) * 2] = (int)P.hdr.size() / 4;
      P.list[((size_t)p * workers + w) * 2 + 1] = (int)asg[w].size();
      for (int it : asg[w]) {
        const int ia = items[it];
        P.hdr.push_back(ia);
        P.hdr.push_back((int)P.rec.size() / 2);
        P.hdr.push_back((int)recs[ia].size() / 2);
        P.hdr.push_back(0);
        P.rec.insert(P.rec.end(), recs[ia].begin(), recs[ia].end());
      }
    }
  }
  P.ok = P.smem <= 227 * 1024;
  return P;
}

// the v8 forward plan (see F8Plan)
static F8Plan build_f8(const TableSet &t, int workers) {
  F8Plan P;
  const int na = t.na, k = t.k, ROW = 128;
  P.srows = na + 1;
  std::vector<int> b1(na, -1), uv(na, -1);
  int brow = 0, uvrow = 0;
  for (int ia = 1; ia < na; ++ia)
    if (t.deg[ia] >= 2 && t.deg[ia] <= k - 2) {
      b1[ia] = brow * ROW;
      brow += t.deg[ia];
    }
  // U/V pairs interleaved per lane: one 256-byte row per pair
  for (int ia = 1; ia < na; ++ia)
    if (t.deg[ia] <= k - 1) {
      uv[ia] = uvrow * ROW;
      uvrow += 2;
    }
  P.zuv = uvrow * ROW;
  uvrow += 2;
  P.sbase1 = P.srows * ROW;
  P.bbase = 2 * P.srows * ROW;
  P.uvbase = P.bbase + brow * ROW;
  P.dtbase = P.uvbase + uvrow * ROW;
  P.recbase = P.dtbase + (k + 2) * ROW;
  P.cpdst = b1;
  // x: a 16-bit byte offset in the S buffer; z: a 16-bit offset in 4-byte
  // units inside its region
  bool ok = k <= 8 && (long)P.srows * ROW <= 65536 && (long)brow * ROW <= 4 * 65536 &&
            (long)uvrow * ROW <= 4 * 65536;
  const uint32_t zrec = ((uint32_t)(na * ROW) << 16) | (uint32_t)(P.zuv / 4);
  P.list.assign((size_t)(k + 1) * workers * 2, 0);
  for (int p = 1; p <= k && ok; ++p) {
    std::vector<int> items;
    std::vector<long> cost;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] == p) {
        items.push_back(ia);
        long c = 24;
        const int st = p >= 2 ? t.fq_at(ia, 2) : 0, nn = p >= 2 ? t.fq_len(ia, 2) : 0;
        for (int i = st; i < st + nn; ++i) c += p == k ? 9 : 6 + 2 * t.deg[t.fq_id[i]];
        cost.push_back(c);
      }
    auto asg = balance(cost, workers);
    for (int w = 0; w < workers; ++w) {
      P.list[((size_t)p * workers + w) * 2] = (int)P.hdr.size() / 8;
      P.list[((size_t)p * workers + w) * 2 + 1] = (int)asg[w].size();
      for (int it : asg[w]) {
        const int ia = items[it];
        if (p == k)
          while (P.rec.size() % 4) P.rec.push_back(zrec);
        const int rstart = (int)P.rec.size();
        int cnt[9] = {0};
        if (p >= 2) {
          const int st = t.fq_at(ia, 2), nn = t.fq_len(ia, 2);
          std::vector<int> idx;
          for (int i = st; i < st + nn; ++i) idx.push_back(i);
          if (p < k)  // bands of |g| = D, longest first, slot order inside
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
              return t.deg[t.fq_id[a]] > t.deg[t.fq_id[b]];
            });
          for (int i : idx) {
            const int ib = t.fq_ib[i], g = t.fq_id[i];
            const int z = p == k ? uv[g] : (t.deg[g] >= 2 ? b1[g] : g * ROW);
            P.rec.push_back(((uint32_t)(ib * ROW) << 16) | (uint32_t)(z / 4));
            if (p < k) cnt[t.deg[g]]++;
          }
        }
        if (p == k)
          while ((P.rec.size() - rstart) % 4) P.rec.push_back(zrec);
        uint32_t blo = 0, bhi = 0;
        for (int d = 1; d <= 8; ++d) {
          if (cnt[d] > 255) ok = false;
          if (d <= 4)
            blo |= (uint32_t)(cnt[d] & 0xff) << (8 * (d - 1));
          else
            bhi |= (uint32_t)(cnt[d] & 0xff) << (8 * (d - 5));
        }
        P.hdr.push_back(ia);
        P.hdr.push_back(rstart);
        P.hdr.push_back((int)P.rec.size() - rstart);
        P.hdr.push_back(p <= k - 2 ? b1[ia] : -1);
        P.hdr.push_back(p <= k - 1 ? uv[ia] : -1);
        P.hdr.push_back((int)blo);
        P.hdr.push_back((int)bhi);
        P.hdr.push_back(0);
      }
    }
  }
  for (int i = 0; i < 4; ++i) P.rec.push_back(0);
  while (P.rec.size() % 4) P.rec.push_back(0);  // whole 16-byte pieces
  P.smem = P.recbase + (int)P.rec.size() * 4;
  P.ok = ok && P.smem <= 227 * 1024;
  return P;
}

BellPlan build_bell_plan(const TableSet &t, int workers, int aj_workers) {
  BellPlan P;
  P.workers = workers;
  P.k = t.k;
  P.na = t.na;
  const int na = t.na, k = t.k;
  // state slots: B_{a,q}, q = 2..deg(a), kept for the multi-indices that
  // later degrees reread (deg < k), contiguous in q
  P.bbase.assign(na, -1);
  int ns = 0;
  for (int ia = 1; ia < na; ++ia)
    if (t.deg[ia] < k && t.deg[ia] >= 2) {
      P.bbase[ia] = ns;
      ns += t.deg[ia] - 1;
    }
  P.nslot = ns;

  // groups of one output a: the b of fq(a, 2) (every b with b <= a, b != 0,
  // b != a), each with the highest level it reaches
  P.fw_list.assign((size_t)(k + 1) * workers * 2, 0);
  for (int p = 1; p <= k; ++p) {
    std::vector<int> items;
    std::vector<long> cost;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] == p) {
        items.push_back(ia);
        long c = 4;
        for (int q = 2; q <= p; ++q) c += t.fq_len(ia, q);
        cost.push_back(c);
      }
    auto asg = balance(cost, workers);
    for (int w = 0; w < workers; ++w) {
      P.fw_list[((size_t)p * workers + w) * 2] = (int)P.fw_arec.size() / 4;
      P.fw_list[((size_t)p * workers + w) * 2 + 1] = (int)asg[w].size();
      for (int it : asg[w]) {
        const int ia = items[it];
        const int gstart = (int)P.fw_grec.size() / 4;
        int gcount = 0;
        if (p >= 2) {
          // fq(a, 2) lists every admissible b in increasing slot order;
          // the level limit of b is q <= p - deg(b) + 1
          const int st = t.fq_at(ia, 2), nn = t.fq_len(ia, 2);
          for (int i = st; i < st + nn; ++i) {
            const int ib = t.fq_ib[i], g = t.fq_id[i];
            const int qmax = std::min(p, p - t.deg[ib] + 1);
            P.fw_grec.push_back(ib);
            P.fw_grec.push_back(g);
            P.fw_grec.push_back(P.bbase[g]);
            P.fw_grec.push_back(qmax);
            P.fw_gc.push_back(t.fq_c[i] * 2.0);  // fq_c at q = 2 is C(a,b)/2
            ++gcount;
          }
        }
        P.fw_arec.push_back(ia | (p << 16));
        P.fw_arec.push_back(gstart);
        P.fw_arec.push_back(gcount);
        P.fw_arec.push_back(P.bbase[ia]);
      }
    }
  }

  // ---- forward v3.  T_a = sum_q s^(q) B_{a,q} regrouped by b (0 < b < a):
  //   T_a = s' S_a + sum_b C(a,b) S_b U_{a-b},  h_a = s'' S_a + sum_b C(a,b) S_b V_{a-b},
  //   U_g = sum_{q=1}^{|g|} s^(q+1)/(q+1) B_{g,q},  V_g = sum s^(q+2)/(q+1) B_{g,q}
  // (the q >= 2 terms of lib/train_module.f90:308-322 with the level index
  // shifted).  The top degree uses it directly, so no Bell value of degree
  // K-1 is kept; lower degrees run the recurrence, whose group of b reads
  // every level of g = a - b (qmax = |g| + 1), so groups are banded by |g|.
  {
    const int ROW = 128;  // bytes per state row (NPB lanes x sizeof(R))
    std::vector<int> b_off(na, -1), u_off(na, -1), v_off(na, -1);
    int row = na;  // rows 0..na-1: S
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] >= 2 && t.deg[ia] <= k - 2) {
        b_off[ia] = row * ROW;
        row += t.deg[ia] - 1;
      }
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] <= k - 1) u_off[ia] = (row++) * ROW;
    P.nuv = 0;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] <= k - 1) {
        v_off[ia] = (row++) * ROW;
        P.nuv++;
      }
    P.dt_off = row * ROW;
    P.nrows = row + k + 2;
    P.f3_list.assign((size_t)(k + 1) * workers * 2, 0);
    for (int p = 1; p <= k; ++p) {
      std::vector<int> items;
      std::vector<long> cost;
      for (int ia = 1; ia < na; ++ia)
        if (t.deg[ia] == p) {
          items.push_back(ia);
          long c = 6;
          const int st = p >= 2 ? t.fq_at(ia, 2) : 0, nn = p >= 2 ? t.fq_len(ia, 2) : 0;
          for (int i = st; i < st + nn; ++i) c += p == k ? 3 : 2 + (p - t.deg[t.fq_ib[i]]);
          cost.push_back(c);
        }
      auto asg = balance(cost, workers);
      for (int w = 0; w < workers; ++w) {
        P.f3_list[((size_t)p * workers + w) * 2] = (int)P.f3_arec.size() / 8;
        P.f3_list[((size_t)p * workers + w) * 2 + 1] = (int)asg[w].size();
        for (int it : asg[w]) {
          const int ia = items[it];
          const int gstart = (int)P.f3_grec.size() / 4;
          uint64_t bands = 0;
          if (p >= 2) {
            const int st = t.fq_at(ia, 2), nn = t.fq_len(ia, 2);
            std::vector<int> idx;
            for (int i = st; i < st + nn; ++i) idx.push_back(i);
            if (p < k)  // bands of |g| = d, longest first, slot order inside
              std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
                return t.deg[t.fq_id[a]] > t.deg[t.fq_id[b]];
              });
            for (int i : idx) {
              const int ib = t.fq_ib[i], g = t.fq_id[i];
              P.f3_grec.push_back(ib * ROW);
              P.f3_grec.push_back(g * ROW);
              P.f3_grec.push_back(p == k ? u_off[g] : b_off[g]);
              P.f3_grec.push_back(p == k ? v_off[g] : 0);
              if (p == k)
                P.f4_grec.push_back((uint32_t)ib | ((uint32_t)(u_off[g] / ROW) << 10));
              else
                P.f4_grec.push_back((uint32_t)ib | ((uint32_t)g << 10) |
                                    ((uint32_t)(b_off[g] > 0 ? b_off[g] / ROW : 0) << 20));
              P.f3_gc.push_back(t.fq_c[i] * 2.0);  // C(a,b)
              if (p < k) bands += 1ull << (8 * (t.deg[g] - 1));
            }
          }
          P.f3_arec.push_back(ia | (p << 16));
          P.f3_arec.push_back(gstart);
          P.f3_arec.push_back((int)P.f3_grec.size() / 4 - gstart);
          P.f3_arec.push_back((int)(bands >> 32));
          P.f3_arec.push_back(b_off[ia]);
          P.f3_arec.push_back(u_off[ia]);
          P.f3_arec.push_back(v_off[ia]);
          P.f3_arec.push_back((int)(bands & 0xffffffffu));
        }
      }
    }
    P.f3_ok = k <= 8 && na <= 1023 && P.nrows <= 4095;
    for (size_t r = 0; r < P.f3_arec.size(); r += 8) {
      const int p = P.f3_arec[r] >> 16;
      if (p < k && P.f3_arec[r + 2] > 0) {
        // a band count above 255 would have carried into the next field
        int total = 0;
        const uint64_t b = ((uint64_t)(uint32_t)P.f3_arec[r + 3] << 32) | (uint32_t)P.f3_arec[r + 7];
        for (int d = 1; d < p; ++d) total += (int)((b >> (8 * (d - 1))) & 0xff);
        if (total != P.f3_arec[r + 2]) P.f3_ok = false;
      }
    }
  }

  // ---- forward v5 (flat records; see bell_plan.hpp)
  {
    const int ROW = 128;
    std::vector<int> b1(na, -1), uv(na, -1);
    int row = na;
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] >= 2 && t.deg[ia] <= k - 2) {
        b1[ia] = row * ROW;
        row += t.deg[ia];
      }
    for (int ia = 1; ia < na; ++ia)
      if (t.deg[ia] <= k - 1) {
        uv[ia] = row * ROW;
        row += 2;
      }
    P.zuv5 = row * ROW;  // a U/V pair of zeros, target of the padding records
    row += 2;
    P.dt_off5 = row * ROW;
    P.nrows5 = row + k + 2;
    P.f5_cpdst = b1;
    P.f5_list.assign((size_t)(k + 1) * workers * 2, 0);
    bool bands_ok = true;
    for (int p = 1; p <= k; ++p) {
      std::vector<int> items;
      std::vector<long> cost;
      for (int ia = 1; ia < na; ++ia)
        if (t.deg[ia] == p) {
          items.push_back(ia);
          long c = 6;
          const int st = p >= 2 ? t.fq_at(ia, 2) : 0, nn = p >= 2 ? t.fq_len(ia, 2) : 0;
          for (int i = st; i < st + nn; ++i) c += p == k ? 4 : 3 + t.deg[t.fq_id[i]];
          cost.push_back(c);
        }
      auto asg = balance(cost, workers);
      for (int w = 0; w < workers; ++w) {
        P.f5_list[((size_t)p * workers + w) * 2] = (int)P.f5_arec.size() / 8;
        P.f5_list[((size_t)p * workers + w) * 2 + 1] = (int)asg[w].size();
        for (int it : asg[w]) {
          const int ia = items[it];
          if (p == k)  // top-degree lists start on a 4-record boundary
            while ((P.f5_rec.size() / 2) % 4) {
              P.f5_rec.push_back(0);
              P.f5_rec.push_back((uint32_t)P.zuv5);
            }
          const int rstart = (int)P.f5_rec.size() / 2;
          uint64_t bands = 0;
          int cnt[9] = {0};
          if (p >= 2) {
            const int st = t.fq_at(ia, 2), nn = t.fq_len(ia, 2);
            std::vector<int> idx;
            for (int i = st; i < st + nn; ++i) idx.push_back(i);
            if (p < k)  // bands of |g| = d, longest first
              std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
                return t.deg[t.fq_id[a]] > t.deg[t.fq_id[b]];
              });
            for (int i : idx) {
              const int ib = t.fq_ib[i], g = t.fq_id[i];
              P.f5_rec.push_back((uint32_t)(ib * ROW));
              if (p == k)
                P.f5_rec.push_back((uint32_t)uv[g]);
              else
                P.f5_rec.push_back((uint32_t)(t.deg[g] >= 2 ? b1[g] : g * ROW));
              if (p < k) cnt[t.deg[g]]++;
            }
          }
          if (p == k)  // and hold a multiple of 4: padding adds S_0 x 0
            while ((P.f5_rec.size() / 2 - rstart) % 4) {
              P.f5_rec.push_back(0);
              P.f5_rec.push_back((uint32_t)P.zuv5);
            }
          for (int d = 1; d <= 8; ++d) {
            if (cnt[d] > 255) bands_ok = false;
            bands += (uint64_t)(cnt[d] & 0xff) << (8 * (d - 1));
          }
          P.f5_arec.push_back(ia | (p << 16));
          P.f5_arec.push_back(rstart);
          P.f5_arec.push_back((int)P.f5_rec.size() / 2 - rstart);
          P.f5_arec.push_back((int)(bands >> 32));
          P.f5_arec.push_back(b1[ia]);
          P.f5_arec.push_back(uv[ia]);
          P.f5_arec.push_back(0);
          P.f5_arec.push_back((int)(bands & 0xffffffffu));
        }
      }
    }
    // the kernels read two records ahead of the one they use
    for (int i = 0; i < 8; ++i) P.f5_rec.push_back(0);
    for (size_t i = 0; i < P.f5_rec.size(); i += 2)
      P.f6_rec.push_back((P.f5_rec[i] / ROW) | ((P.f5_rec[i + 1] / ROW) << 16));
    while (P.f6_rec.size() % 4) P.f6_rec.push_back(0);  // whole 16-byte pieces
    P.f5_ok = bands_ok && k <= 8 && (size_t)(P.nrows5 + na) * ROW <= 227 * 1024;
  }

  // padding: the kernels prefetch the record after the last one of a list
  for (int i = 0; i < 4; ++i) {
    for (int c = 0; c < 4; ++c) P.f3_grec.push_back(0);
    P.f3_gc.push_back(0.0);
    P.f4_grec.push_back(0);
  }

  // ---- factorial scales of the adjoint v3 (records built with the lists below)
  {
    P.fact.assign(na, 1.0);
    for (int ia = 0; ia < na; ++ia)
      for (int i = 0; i < t.d0; ++i)
        for (int v = 2; v <= t.alpha[(size_t)ia * t.d0 + i]; ++v) P.fact[ia] *= v;
  }

  P.a7f = build_a7(t, aj_workers, 16);
  P.a7d = build_a7(t, aj_workers, 8);
  P.f8 = build_f8(t, workers);
  P.f9 = build_f9(t, workers);

  // adjoint outputs: Sb_0 (pairs (a, a) for every a) and every Sb_b, b >= 1
  std::vector<long> cost;
  std::vector<std::vector<std::pair<uint32_t, double>>> lists(na);
  for (int ia = 0; ia < na; ++ia) lists[0].push_back({(uint32_t)ia | ((uint32_t)ia << 16), 1.0});
  for (int ib = 1; ib < na; ++ib)
    for (int ip = t.pair_start[ib]; ip < t.pair_start[ib] + t.pair_num[ib]; ++ip)
      lists[ib].push_back({(uint32_t)t.pair_ia[ip] | ((uint32_t)t.pair_id[ip] << 16),
                           t.pair_binom[ip]});
  for (int ib = 0; ib < na; ++ib) cost.push_back(4 + (long)lists[ib].size());
  auto asg = balance(cost, aj_workers);
  P.aj_list.assign((size_t)aj_workers * 2, 0);
  for (int w = 0; w < aj_workers; ++w) {
    P.aj_list[w * 2] = (int)P.aj_orec.size() / 4;
    P.aj_list[w * 2 + 1] = (int)asg[w].size();
    for (int ib : asg[w]) {
      P.aj_orec.push_back(ib);
      P.aj_orec.push_back((int)P.aj_pair.size());
      P.aj_orec.push_back((int)lists[ib].size());
      P.aj_orec.push_back(0);
      P.a3_orec.push_back(ib);
      P.a3_orec.push_back((int)P.a3_pair.size() / 2);
      P.a3_orec.push_back((int)lists[ib].size());
      P.a3_orec.push_back(0);
      for (auto &pr : lists[ib]) {
        P.aj_pair.push_back((int)pr.first);
        P.aj_c.push_back(pr.second);
        // rows 0..na-1 hold a! Tb_a, rows na..2na-1 hold h_g / g!
        P.a3_pair.push_back((int)(pr.first & 0xffffu) * 128);
        P.a3_pair.push_back((na + (int)(pr.first >> 16)) * 128);
        P.a4_pair.push_back((pr.first & 0xffffu) | ((uint32_t)(na + (pr.first >> 16)) << 16));
      }
    }
  }
  return P;
}

}  // namespace dnnf90
