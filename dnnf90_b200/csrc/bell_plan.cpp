// bell_plan.cpp - see bell_plan.hpp.
#include "bell_plan.hpp"

#include <algorithm>
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
      for (auto &pr : lists[ib]) {
        P.aj_pair.push_back((int)pr.first);
        P.aj_c.push_back(pr.second);
      }
    }
  }
  return P;
}

}  // namespace dnnf90
