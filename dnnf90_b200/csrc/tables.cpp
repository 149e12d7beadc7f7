// tables.cpp - build of a multi-index table set; see tables.hpp.
#include "tables.hpp"

#include <algorithm>
#include <functional>
#include <unordered_map>

namespace dnnf90 {

namespace {

struct VecHash {
  size_t operator()(const std::vector<int> &v) const {
    size_t h = 1469598103934665603ull;
    for (int x : v) h = (h ^ (size_t)(x + 1)) * 1099511628211ull;
    return h;
  }
};

// number of multi-indices with |alpha| <= k (n_multi_indices,
// lib/multi_index_bell_module.f90:551-572), 64-bit with a range check
long long count_dense(int d0, int k) {
  long long tot = 0;
  for (int p = 0; p <= k; ++p) {
    long long c = 1;
    for (int i = 1; i <= p; ++i) {
      c = c * (long long)(d0 - 1 + i) / i;
      if (c > (1ll << 40)) return -1;
    }
    tot += c;
  }
  return tot;
}

}  // namespace

int TableSet::find(const int *a) const {
  // binary search is not needed at the sizes a kernel can carry; a linear
  // scan keeps the builder free of auxiliary state
  for (int ia = 0; ia < na; ++ia) {
    bool eq = true;
    for (int i = 0; i < d0; ++i)
      if (alpha[(size_t)ia * d0 + i] != a[i]) { eq = false; break; }
    if (eq) return ia;
  }
  return -1;
}

std::string build_tables(int d0, int k, int nseed, const int *seeds,
                         TableSet &t) {
  // argument contract of table_args_ok (lib/c_api_module.f90:72-84)
  if (d0 < 1 || k < 1 || k > 15 || nseed < 0) return "bad d0, k or nseed";
  for (int i = 0; i < d0 * nseed; ++i)
    if (seeds[i] < 0 || seeds[i] > k) return "seed component out of range";
  long long nfull = count_dense(d0, k);
  if (nfull < 0 || nfull > 2000000) return "carried set too large";

  // graded CWR enumeration (gen_cwr, :576-615)
  std::vector<int> afull;
  afull.reserve((size_t)nfull * d0);
  std::vector<int> slots(k + 1), cur(d0);
  afull.insert(afull.end(), d0, 0);
  for (int p = 1; p <= k; ++p) {
    std::function<void(int, int)> rec = [&](int depth, int vmin) {
      for (int v = vmin; v < d0; ++v) {
        slots[depth] = v;
        if (depth == p - 1) {
          std::fill(cur.begin(), cur.end(), 0);
          for (int i = 0; i < p; ++i) cur[slots[i]]++;
          afull.insert(afull.end(), cur.begin(), cur.end());
        } else {
          rec(depth + 1, v);
        }
      }
    };
    rec(0, 0);
  }

  // downward closure of the seeds (:164-179)
  std::vector<char> incl((size_t)nfull, nseed > 0 ? 0 : 1);
  for (int s = 0; s < nseed; ++s) {
    const int *sa = seeds + (size_t)s * d0;
    int ssum = 0;
    for (int i = 0; i < d0; ++i) ssum += sa[i];
    if (ssum > k) return "seed multi-index exceeds K";
    for (long long ia = 0; ia < nfull; ++ia) {
      bool ok = true;
      for (int i = 0; i < d0; ++i)
        if (afull[(size_t)ia * d0 + i] > sa[i]) { ok = false; break; }
      if (ok) incl[(size_t)ia] = 1;
    }
  }

  t = TableSet();
  t.d0 = d0;
  t.k = k;
  for (long long ia = 0; ia < nfull; ++ia) {
    if (!incl[(size_t)ia]) continue;
    int s = 0;
    for (int i = 0; i < d0; ++i) {
      t.alpha.push_back(afull[(size_t)ia * d0 + i]);
      s += afull[(size_t)ia * d0 + i];
    }
    t.deg.push_back(s);
  }
  t.na = (int)t.deg.size();
  if (t.na < 1 || t.deg[0] != 0) return "empty closure";
  const int na = t.na;

  std::unordered_map<std::vector<int>, int, VecHash> index;
  index.reserve(na * 2);
  for (int ia = 0; ia < na; ++ia)
    index[std::vector<int>(t.alpha.begin() + (size_t)ia * d0,
                           t.alpha.begin() + (size_t)(ia + 1) * d0)] = ia;

  t.ind_e1.assign(d0, -1);
  for (int ia = 0; ia < na; ++ia)
    if (t.deg[ia] == 1)
      for (int i = 0; i < d0; ++i)
        if (t.alpha[(size_t)ia * d0 + i] == 1) t.ind_e1[i] = ia;

  double fact[17];
  fact[0] = 1.0;
  for (int i = 1; i <= 16; ++i) fact[i] = fact[i - 1] * (double)i;

  // sub-multi-index relation: for each ia, the ib <= ia with the index of
  // ia - ib and the multi-binomial C(alpha_ia, alpha_ib) (:219-234)
  struct Sub { int ib, id; double c; };
  std::vector<std::vector<Sub>> subs(na);
  std::vector<int> diff(d0);
  for (int ia = 0; ia < na; ++ia) {
    const int *a = &t.alpha[(size_t)ia * d0];
    for (int ib = 0; ib < na; ++ib) {
      const int *b = &t.alpha[(size_t)ib * d0];
      bool le = true;
      for (int i = 0; i < d0; ++i)
        if (b[i] > a[i]) { le = false; break; }
      if (!le) continue;
      for (int i = 0; i < d0; ++i) diff[i] = a[i] - b[i];
      auto it = index.find(diff);
      int id = it == index.end() ? -1 : it->second;
      double r = 1.0;
      for (int i = 0; i < d0; ++i)
        r = r * fact[a[i]] / (fact[b[i]] * fact[a[i] - b[i]]);
      subs[ia].push_back({ib, id, r});
    }
  }

  // Bell term count (bell_enum, :243-264, :356-403)
  {
    std::vector<int> rem(d0);
    std::function<void(int, int, int, const int *)> enumr =
        [&](int q, int depth, int id_min, const int *rm) {
          int remsum = 0;
          for (int i = 0; i < d0; ++i) remsum += rm[i];
          std::vector<int> rn(d0);
          for (int id = id_min; id < na; ++id) {
            if (t.deg[id] < 1) continue;
            if (t.deg[id] > remsum - (q - depth)) continue;
            const int *aid = &t.alpha[(size_t)id * d0];
            bool bad = false;
            for (int i = 0; i < d0; ++i)
              if (aid[i] > rm[i]) { bad = true; break; }
            if (bad) continue;
            for (int i = 0; i < d0; ++i) rn[i] = rm[i] - aid[i];
            if (depth == q) {
              bool z = true;
              for (int i = 0; i < d0; ++i)
                if (rn[i]) { z = false; break; }
              if (z) t.nbell++;
            } else {
              enumr(q, depth + 1, id, rn.data());
            }
          }
        };
    if ((long long)na * na <= 4000000)
      for (int ia = 1; ia < na; ++ia)
        for (int q = 1; q <= t.deg[ia]; ++q)
          enumr(q, 1, 1, &t.alpha[(size_t)ia * d0]);
  }

  // adjoint pair lists (:267-297): for ib = 2..na, every ia = 2..na with
  // ib <= ia, in increasing ia
  t.pair_start.assign(na, 0);
  t.pair_num.assign(na, 0);
  {
    std::vector<std::vector<Sub>> by_ib(na);
    for (int ia = 1; ia < na; ++ia)
      for (const Sub &s : subs[ia])
        if (s.ib >= 1 && s.id >= 0) by_ib[s.ib].push_back({ia, s.id, s.c});
    for (int ib = 1; ib < na; ++ib) {
      t.pair_start[ib] = (int)t.pair_ia.size();
      t.pair_num[ib] = (int)by_ib[ib].size();
      for (const Sub &s : by_ib[ib]) {
        t.pair_ia.push_back(s.ib);  // the ia of the pair
        t.pair_id.push_back(s.id);
        t.pair_binom.push_back(s.c);
      }
    }
  }

  // forward convolution lists (:299-332): for ia = 2..na, q = 2..deg(ia),
  // every ib = 2..na with ib <= ia and deg(ia) - deg(ib) >= q - 1;
  // coefficient C(alpha,beta)/q
  t.fq_start.assign((size_t)na * (k + 1), 0);
  t.fq_num.assign((size_t)na * (k + 1), 0);
  for (int ia = 1; ia < na; ++ia) {
    int p = t.deg[ia];
    for (int q = 2; q <= p; ++q) {
      t.fq_start[(size_t)ia * (k + 1) + q] = (int)t.fq_ib.size();
      for (const Sub &s : subs[ia]) {
        if (s.ib < 1 || s.id < 0) continue;
        if (p - t.deg[s.ib] >= q - 1) {
          t.fq_ib.push_back(s.ib);
          t.fq_id.push_back(s.id);
          t.fq_c.push_back(s.c / (double)q);
        }
      }
      t.fq_num[(size_t)ia * (k + 1) + q] =
          (int)t.fq_ib.size() - t.fq_start[(size_t)ia * (k + 1) + q];
    }
  }

  // tanh derivative polynomials P_0 = t, P_{q+1} = (1 - t^2) P_q'
  // (build_tanh_poly, :406-429), q = 0..k+1
  {
    int qmax = k + 1, ld = k + 3;
    t.tpc.assign((size_t)ld * (qmax + 1), 0.0);
    std::vector<double> dc(ld);
    t.tpc[0 * ld + 1] = 1.0;
    for (int q = 0; q < qmax; ++q) {
      std::fill(dc.begin(), dc.end(), 0.0);
      for (int i = 0; i <= qmax; ++i) dc[i] = (double)(i + 1) * t.tpc[q * ld + i + 1];
      for (int i = 0; i <= qmax + 1; ++i) {
        double v = dc[i];
        if (i >= 2) v = v - dc[i - 2];
        t.tpc[(q + 1) * ld + i] = v;
      }
    }
  }

  // state slots of the Bell kernels: B_{ia,q} (q >= 2) is reread by later
  // multi-indices only when deg(ia) < k
  t.bslot.assign((size_t)na * (k + 1), -1);
  t.nslot = 0;
  for (int ia = 1; ia < na; ++ia)
    if (t.deg[ia] < k)
      for (int q = 2; q <= t.deg[ia]; ++q) t.bslot[(size_t)ia * (k + 1) + q] = t.nslot++;
  return "";
}

}  // namespace dnnf90
