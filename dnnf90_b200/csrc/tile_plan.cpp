// tile_plan.cpp - work lists of the register-tiled Bell kernels (see
// tile_plan.hpp for the recurrences and the tiling).
#include "tile_plan.hpp"

#include <algorithm>
#include <map>
#include <numeric>

namespace dnnf90 {

namespace {

long binom(int n, int r) {
  if (r < 0 || r > n) return 0;
  long v = 1;
  for (int i = 1; i <= r; ++i) v = v * (n - r + i) / i;
  return v;
}

// multiply-adds of one tile product: pairs (b, c) of td-dimensional
// indices with |b| + |c| <= L - 1
long tile_pairs(int td, int L) { return binom(L - 1 + 2 * td, 2 * td); }

// outer indices: every tuple of dout nonnegative integers of sum <= k, by
// degree, then lexicographically
std::vector<std::vector<int>> outer_indices(int dout, int k) {
  std::vector<std::vector<int>> out;
  std::vector<int> cur(dout, 0);
  std::vector<std::vector<int>> all;
  if (dout == 0) return {{}};
  // enumerate all tuples with sum <= k
  std::vector<int> a(dout, 0);
  while (true) {
    int s = std::accumulate(a.begin(), a.end(), 0);
    if (s <= k) all.push_back(a);
    int i = dout - 1;
    while (i >= 0) {
      if (++a[i] <= k) break;
      a[i] = 0;
      --i;
    }
    if (i < 0) break;
  }
  std::stable_sort(all.begin(), all.end(), [](const std::vector<int> &x, const std::vector<int> &y) {
    return std::accumulate(x.begin(), x.end(), 0) < std::accumulate(y.begin(), y.end(), 0);
  });
  return all;
}

int deg_of(const std::vector<int> &g) { return std::accumulate(g.begin(), g.end(), 0); }

bool leq(const std::vector<int> &a, const std::vector<int> &b) {
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i] > b[i]) return false;
  return true;
}

// longest-processing-time assignment of costs to w workers; returns the
// worker of each item
std::vector<int> lpt(const std::vector<long> &cost, int w) {
  std::vector<int> idx(cost.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<long> load(w, 0);
  std::vector<int> owner(cost.size(), 0);
  for (int i : idx) {
    int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    owner[i] = b;
    load[b] += cost[i];
  }
  return owner;
}

}  // namespace

// fixed cost of a unit in the load balance, beside its multiply-adds and
// loads (its accumulators, its record loop, its output stores)
static const long ADJ_UNIT_COST = 1000;
static const long FWD_UNIT_COST = 500;

TilePlan build_tile_plan(const TableSet &t, int fwarps, int awarps) {
  TilePlan P;
  const int d = t.d0, K = t.k;
  if (d < 1 || K < 1 || K > TILE_KMAX || fwarps < 1 || awarps < 1) return P;
  if ((long)t.na != binom(K + d, d)) return P;  // not the dense set
  for (int ia = 0; ia < t.na; ++ia)
    if (t.deg[ia] > K) return P;
  const int td = d >= 3 ? 2 : 1, dout = d - td;
  P.td = td;
  P.d0 = d;
  P.k = K;
  P.na = t.na;
  P.fwarps = fwarps;
  P.awarps = awarps;

  // ---- the tile layout of the full set
  const auto outer = outer_indices(dout, K);
  std::map<std::vector<int>, int> oidx;
  for (size_t i = 0; i < outer.size(); ++i) oidx[outer[i]] = (int)i;
  auto inner = [td](int e, int *a) {  // graded entry e of a tile -> inner index
    if (td == 1) {
      a[0] = e;
      return;
    }
    int s = 0;
    while ((s + 1) * (s + 2) / 2 <= e) ++s;
    a[1] = e - s * (s + 1) / 2;
    a[0] = s - a[1];
  };
  P.perm.assign(t.na, -1);
  P.rowslot.assign(t.na, -1);
  P.tbase.resize(outer.size());
  int row = 0;
  for (size_t o = 0; o < outer.size(); ++o) {
    P.tbase[o] = row;
    const int L = K - deg_of(outer[o]) + 1;
    for (int e = 0; e < tile_size(td, L); ++e) {
      int a[8] = {0};
      inner(e, a);
      for (int i = 0; i < dout; ++i) a[td + i] = outer[o][i];
      const int ia = t.find(a);
      if (ia < 0 || P.perm[ia] >= 0) return TilePlan();
      P.perm[ia] = row;
      P.rowslot[row] = ia;
      ++row;
    }
  }
  if (row != t.na) return TilePlan();

  // ---- forward: D_q over degrees <= K - q, tiles of side m - |g| + 1
  // dbase[q][o]: first row of outer index o's tile of D_q (q = 1..K)
  std::vector<std::vector<int>> dbase(K + 1, std::vector<int>(outer.size(), -1));
  for (int q = K; q >= 1; --q) {
    const int m = K - q;
    int r = 0;
    for (size_t o = 0; o < outer.size(); ++o) {
      const int g = deg_of(outer[o]);
      if (g > m) continue;
      dbase[q][o] = r;
      r += tile_size(td, m - g + 1);
    }
    P.nbuf[q & 1] = std::max(P.nbuf[q & 1], r);
  }
  P.flist.assign((size_t)K * fwarps * 2, 0);
  for (int q = K - 1; q >= 0; --q) {
    const int m = K - q;
    struct U {
      int L, origin, out;
      std::vector<uint32_t> rec;
      long cost;
    };
    std::vector<U> us;
    for (size_t o = 0; o < outer.size(); ++o) {
      const auto &gam = outer[o];
      const int g = deg_of(gam);
      if (g > m) continue;
      U u;
      u.L = m - g + 1;
      u.origin = g == 0;
      u.out = q > 0 ? dbase[q][o] : P.tbase[o];
      u.cost = 0;
      // the record of delta = 0 first, then every other delta <= gamma
      std::vector<std::vector<int>> dels;
      dels.push_back(std::vector<int>(dout, 0));
      for (size_t o2 = 0; o2 < outer.size(); ++o2)
        if (deg_of(outer[o2]) > 0 && leq(outer[o2], gam)) dels.push_back(outer[o2]);
      for (size_t i = 0; i < dels.size(); ++i) {
        std::vector<int> eps(dout);
        for (int j = 0; j < dout; ++j) eps[j] = gam[j] - dels[i][j];
        const int so = oidx.at(dels[i]), eo = oidx.at(eps);
        const bool z = i == 0;
        const int LD = z ? u.L - 1 : u.L;
        // a delta = 0 record of a one-entry tile reads no D row
        const int srow = P.tbase[so], drow = LD > 0 ? dbase[q + 1][eo] : 0;
        if (drow < 0) return TilePlan();
        u.rec.push_back((uint32_t)srow | (uint32_t)drow << 16);
        long f = tile_pairs(td, u.L);
        if (z) f -= tile_size(td, u.L);  // b = 0 is left out
        if (z && LD == 0) f = 0;
        const long ld = tile_size(td, u.L) - (z ? 1 : 0) + tile_size(td, LD);
        P.fwd_fma2 += f;
        P.fwd_loads += ld;
        u.cost += f + ld + 8;
      }
      u.cost += 3 * tile_size(td, u.L);
      us.push_back(std::move(u));
    }
    std::vector<long> cost;
    for (auto &u : us) cost.push_back(u.cost + FWD_UNIT_COST);
    const auto own = lpt(cost, fwarps);
    for (int w = 0; w < fwarps; ++w) {
      P.flist[((size_t)q * fwarps + w) * 2] = (int)P.funit.size() / 4;
      int cnt = 0;
      for (size_t i = 0; i < us.size(); ++i) {
        if (own[i] != w) continue;
        P.funit.push_back(us[i].L | us[i].origin << 8);
        P.funit.push_back((int)P.frec.size());
        P.funit.push_back((int)us[i].rec.size());
        P.funit.push_back(us[i].out);
        P.frec.insert(P.frec.end(), us[i].rec.begin(), us[i].rec.end());
        ++cnt;
      }
      P.flist[((size_t)q * fwarps + w) * 2 + 1] = cnt;
    }
  }

  // ---- adjoint: output tile delta, records eps with |delta| + |eps| <= K
  struct A {
    int Lout, out;
    std::vector<uint32_t> rec;
    std::vector<long> rcost;
    long cost;
  };
  std::vector<A> as;
  long total = 0;
  for (size_t o = 0; o < outer.size(); ++o) {
    const auto &del = outer[o];
    const int gd = deg_of(del);
    A a;
    a.Lout = K - gd + 1;
    a.out = P.tbase[o];
    a.cost = 0;
    for (size_t o2 = 0; o2 < outer.size(); ++o2) {
      const auto &eps = outer[o2];
      if (gd + deg_of(eps) > K) continue;
      std::vector<int> sum(dout);
      for (int j = 0; j < dout; ++j) sum[j] = del[j] + eps[j];
      const int L = K - gd - deg_of(eps) + 1;
      const int hrow = P.tbase[o2], tbrow = P.tbase[oidx.at(sum)];
      a.rec.push_back((uint32_t)hrow | (uint32_t)tbrow << 14 | (uint32_t)L << 28);
      const long c = tile_pairs(td, L) + 2 * tile_size(td, L) + 40;
      a.rcost.push_back(c);
      a.cost += c;
      P.adj_fma += tile_pairs(td, L);
      P.adj_loads += 2 * tile_size(td, L);
    }
    total += a.cost;
    as.push_back(std::move(a));
  }
  long maxrec = 0;
  for (auto &a : as) maxrec = std::max(maxrec, *std::max_element(a.rcost.begin(), a.rcost.end()));
  // split an output tile when it holds more than a twelfth of the work (at
  // most: more splits would need more scratch rows than fit beside the two
  // item buffers)
  const int ways = std::min(awarps, 12);
  const long cap = std::max(maxrec, (total + ways - 1) / ways);
  struct Part {
    int Lout, split, rec0, nrec, out;
    long cost;
  };
  std::vector<Part> parts;
  std::vector<uint32_t> recs;
  int scratch = 0;
  for (auto &a : as) {
    const int rec0 = (int)recs.size();
    recs.insert(recs.end(), a.rec.begin(), a.rec.end());
    if (a.cost <= cap) {
      parts.push_back({a.Lout, 0, rec0, (int)a.rec.size(), a.out, a.cost});
      continue;
    }
    // split into np parts of about equal cost, records kept in order
    const int np = (int)((a.cost + cap - 1) / cap);
    const long share = (a.cost + np - 1) / np;
    const int first_scr = scratch;
    int start = 0, made = 0;
    long acc = 0;
    for (size_t i = 0; i < a.rec.size(); ++i) {
      acc += a.rcost[i];
      const bool last = i + 1 == a.rec.size();
      if (last || (acc >= share && made < np - 1)) {
        parts.push_back({a.Lout, 1, rec0 + start, (int)i + 1 - start, scratch, acc});
        scratch += tile_size(td, a.Lout);
        start = (int)i + 1;
        acc = 0;
        ++made;
      }
    }
    P.afin.push_back(a.Lout);
    P.afin.push_back(a.out);
    P.afin.push_back(made);
    P.afin.push_back(first_scr);
  }
  P.arec = recs;
  P.nscratch = scratch;
  {
    // a unit's fixed cost: measured per-warp times at C3 fit about 1000
    // cycles a unit better than its multiply-adds, which overlap across warps
    std::vector<long> cost;
    for (auto &p : parts) cost.push_back(p.cost + ADJ_UNIT_COST);
    const auto own = lpt(cost, awarps);
    P.alist.assign((size_t)awarps * 2, 0);
    for (int w = 0; w < awarps; ++w) {
      P.alist[w * 2] = (int)P.aunit.size() / 4;
      int cnt = 0;
      for (size_t i = 0; i < parts.size(); ++i) {
        if (own[i] != w) continue;
        // records per degree of eps (tile side Lout - E): 4 bits each
        uint32_t cw = 0;
        for (int r = parts[i].rec0; r < parts[i].rec0 + parts[i].nrec; ++r) {
          const int E = parts[i].Lout - (int)(P.arec[r] >> 28);
          if (E < 0 || E > 7 || ((cw >> (4 * E)) & 15u) == 15u) return TilePlan();
          cw += 1u << (4 * E);
        }
        P.aunit.push_back(parts[i].Lout | parts[i].split << 8);
        P.aunit.push_back(parts[i].rec0);
        P.aunit.push_back((int)cw);
        P.aunit.push_back(parts[i].out);
        ++cnt;
      }
      P.alist[w * 2 + 1] = cnt;
    }
    // finishing phase: every element of a split output tile is one entry
    // (its row, parts, first scratch row, part stride), dealt round robin, so
    // that all warps share the sums
    std::vector<int> elems;
    const int ntiles = (int)P.afin.size() / 4;
    for (int f = 0; f < ntiles; ++f) {
      const int lo = P.afin[4 * f], out = P.afin[4 * f + 1], np = P.afin[4 * f + 2];
      const int s0 = P.afin[4 * f + 3], nt = tile_size(td, lo);
      for (int e = 0; e < nt; ++e) {
        elems.push_back(out + e);
        elems.push_back(np);
        elems.push_back(s0 + e);
        elems.push_back(nt);
      }
    }
    P.aflist.assign((size_t)awarps * 2, 0);
    std::vector<int> fin;
    const int nfin = (int)elems.size() / 4;
    for (int w = 0; w < awarps; ++w) {
      P.aflist[w * 2] = (int)fin.size() / 4;
      int cnt = 0;
      for (int f = w; f < nfin; f += awarps) {
        fin.insert(fin.end(), elems.begin() + 4 * f, elems.begin() + 4 * f + 4);
        ++cnt;
      }
      P.aflist[w * 2 + 1] = cnt;
    }
    P.afin = fin;
  }
  P.ok = true;
  return P;
}

}  // namespace dnnf90
