/* oracle.c - CPU FP64 restatement of the DNNF90 hot path.  TEST
 * INFRASTRUCTURE ONLY (see oracle.h): it is the checker for the CUDA
 * path, never the thing measured or shipped.
 *
 * Build with -ffp-contract=off: the reference's default build
 * (gfortran -O3, x86-64 baseline, Makefile:30-33) issues no FMA, and the
 * operation order below is the reference's, so the results agree bitwise.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_tables {
  int d0, k, na;
  int iact;  /* activation: 0 tanh, 1 sin, 2 erf, 3 J0, 4 J1 (the tabset's iact) */
  int *alpha;   /* [na][d0] */
  int *deg;     /* [na] */
  int *ind_e1;  /* [d0], 1-based slot or 0 */
  int *fq_start, *fq_num; /* [na][kq], kq = max(K,2)-1, q = 2.. */
  int kq;
  int nfq;
  int *fq_ib, *fq_id;
  double *fq_c;
  int *pair_start, *pair_num;
  int npair;
  int *pair_ia, *pair_id;
  double *pair_binom;
  int nbell;
  double *tpc; /* tpc(i,q), i = 0..K+2, q = 0..K+1, at q*(K+3)+i */
};

static double fact_tab[17];

/* ---- enumeration (gen_cwr / cwr_rec, lib/multi_index_bell_module.f90:
 * 576-615): degree-p multi-indices in combinations-with-replacement order */
static void cwr_rec(int d0, int p, int depth, int vmin, int *slots,
                    int *list, int *icount) {
  for (int v = vmin; v <= d0; ++v) {
    slots[depth - 1] = v;
    if (depth == p) {
      int *a = list + (size_t)(*icount) * d0;
      memset(a, 0, sizeof(int) * d0);
      for (int i = 0; i < p; ++i) a[slots[i] - 1] += 1;
      (*icount)++;
    } else {
      cwr_rec(d0, p, depth + 1, v, slots, list, icount);
    }
  }
}

/* n_multi_indices (:551-572) */
static long long n_multi(int d0, int k) {
  long long tot = 0;
  for (int p = 0; p <= k; ++p) {
    long long c = 1;
    for (int i = 1; i <= p; ++i) c = c * (long long)(d0 - 1 + i) / i;
    tot += c;
  }
  return tot;
}

/* lookup of a multi-index by value (find_alpha, :520-538); a linear scan
 * is enough for a checker */
static int find_alpha(const orc_tables *t, const int *a) {
  for (int ia = 0; ia < t->na; ++ia) {
    if (memcmp(t->alpha + (size_t)ia * t->d0, a, sizeof(int) * t->d0) == 0)
      return ia + 1;
  }
  return 0;
}

/* bell_enum (:356-403), counting only: the explicit partition tables are
 * diagnostic in the reference (no kernel reads them) */
static void bell_count(const orc_tables *t, int q, int depth, int id_min,
                       const int *rem, int *nterm) {
  int d0 = t->d0;
  int remsum = 0;
  for (int i = 0; i < d0; ++i) remsum += rem[i];
  int *rem_new = (int *)malloc(sizeof(int) * d0);
  for (int id = id_min; id <= t->na; ++id) {
    const int *aid = t->alpha + (size_t)(id - 1) * d0;
    if (t->deg[id - 1] < 1) continue;
    if (t->deg[id - 1] > remsum - (q - depth)) continue;
    int bad = 0;
    for (int i = 0; i < d0; ++i)
      if (aid[i] > rem[i]) { bad = 1; break; }
    if (bad) continue;
    for (int i = 0; i < d0; ++i) rem_new[i] = rem[i] - aid[i];
    if (depth == q) {
      int zero = 1;
      for (int i = 0; i < d0; ++i)
        if (rem_new[i] != 0) { zero = 0; break; }
      if (zero) (*nterm)++;
    } else {
      bell_count(t, q, depth + 1, id, rem_new, nterm);
    }
  }
  free(rem_new);
}

orc_tables *orc_tables_build(int d0, int k, int nseed, const int *seeds) {
  if (d0 < 1 || k < 1 || k > 15 || nseed < 0) return NULL;
  fact_tab[0] = 1.0;
  for (int i = 1; i <= 16; ++i) fact_tab[i] = fact_tab[i - 1] * (double)i;

  long long nfull_ll = n_multi(d0, k);
  if (nfull_ll > (1 << 24)) return NULL;
  int nfull = (int)nfull_ll;
  int *afull = (int *)malloc(sizeof(int) * (size_t)nfull * d0);
  int icount = 0;
  int *slots = (int *)malloc(sizeof(int) * (k + 1));
  for (int p = 0; p <= k; ++p) {
    if (p == 0) {
      memset(afull, 0, sizeof(int) * d0);
      icount = 1;
    } else {
      cwr_rec(d0, p, 1, 1, slots, afull, &icount);
    }
  }
  free(slots);

  /* downward closure of the seeds (:164-179) */
  char *incl = (char *)malloc(nfull);
  if (nseed > 0) {
    memset(incl, 0, nfull);
    for (int is = 0; is < nseed; ++is) {
      const int *s = seeds + (size_t)is * d0;
      int ssum = 0;
      for (int i = 0; i < d0; ++i) {
        if (s[i] < 0) { free(afull); free(incl); return NULL; }
        ssum += s[i];
      }
      if (ssum > k) { free(afull); free(incl); return NULL; }
      for (int ia = 0; ia < nfull; ++ia) {
        int ok = 1;
        for (int i = 0; i < d0; ++i)
          if (afull[(size_t)ia * d0 + i] > s[i]) { ok = 0; break; }
        if (ok) incl[ia] = 1;
      }
    }
  } else {
    memset(incl, 1, nfull);
  }

  orc_tables *t = (orc_tables *)calloc(1, sizeof(orc_tables));
  t->d0 = d0;
  t->k = k;
  int na = 0;
  for (int ia = 0; ia < nfull; ++ia) na += incl[ia];
  t->na = na;
  t->alpha = (int *)malloc(sizeof(int) * (size_t)na * d0);
  t->deg = (int *)malloc(sizeof(int) * na);
  int c = 0;
  for (int ia = 0; ia < nfull; ++ia) {
    if (!incl[ia]) continue;
    int s = 0;
    for (int i = 0; i < d0; ++i) {
      t->alpha[(size_t)c * d0 + i] = afull[(size_t)ia * d0 + i];
      s += afull[(size_t)ia * d0 + i];
    }
    t->deg[c] = s;
    c++;
  }
  free(afull);
  free(incl);
  if (na < 1 || t->deg[0] != 0) { orc_tables_free(t); return NULL; }

  /* unit multi-indices (:209-217) */
  t->ind_e1 = (int *)calloc(d0, sizeof(int));
  for (int ia = 0; ia < na; ++ia) {
    if (t->deg[ia] == 1) {
      for (int iv = 0; iv < d0; ++iv)
        if (t->alpha[(size_t)ia * d0 + iv] == 1) t->ind_e1[iv] = ia + 1;
    }
  }

  /* ind_diff and multi-binomials (:219-234) */
  int *ind_diff = (int *)calloc((size_t)na * na, sizeof(int));
  double *binom = (double *)calloc((size_t)na * na, sizeof(double));
  int *diff = (int *)malloc(sizeof(int) * d0);
  for (int ia = 0; ia < na; ++ia) {
    const int *a = t->alpha + (size_t)ia * d0;
    for (int ib = 0; ib < na; ++ib) {
      const int *b = t->alpha + (size_t)ib * d0;
      int le = 1;
      for (int i = 0; i < d0; ++i)
        if (b[i] > a[i]) { le = 0; break; }
      if (!le) continue;
      for (int i = 0; i < d0; ++i) diff[i] = a[i] - b[i];
      ind_diff[(size_t)ia * na + ib] = find_alpha(t, diff);
      double rtmp = 1.0;
      for (int iv = 0; iv < d0; ++iv)
        rtmp = rtmp * fact_tab[a[iv]] /
               (fact_tab[b[iv]] * fact_tab[a[iv] - b[iv]]);
      binom[(size_t)ia * na + ib] = rtmp;
    }
  }
  free(diff);

  /* Bell term count (:243-264) */
  t->nbell = 0;
  for (int ia = 2; ia <= na; ++ia) {
    int p = t->deg[ia - 1];
    for (int q = 1; q <= p; ++q)
      bell_count(t, q, 1, 2, t->alpha + (size_t)(ia - 1) * d0, &t->nbell);
  }

  /* adjoint pair tables (:267-297) */
  t->pair_start = (int *)calloc(na, sizeof(int));
  t->pair_num = (int *)calloc(na, sizeof(int));
  for (int ib = 2; ib <= na; ++ib)
    for (int ia = 2; ia <= na; ++ia)
      if (ind_diff[(size_t)(ia - 1) * na + (ib - 1)] > 0)
        t->pair_num[ib - 1]++;
  t->pair_start[0] = 1;
  if (na >= 2) t->pair_start[1] = 1;
  for (int ib = 3; ib <= na; ++ib)
    t->pair_start[ib - 1] = t->pair_start[ib - 2] + t->pair_num[ib - 2];
  int np = 0;
  for (int ib = 0; ib < na; ++ib) np += t->pair_num[ib];
  t->npair = np;
  t->pair_ia = (int *)malloc(sizeof(int) * (np > 0 ? np : 1));
  t->pair_id = (int *)malloc(sizeof(int) * (np > 0 ? np : 1));
  t->pair_binom = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  int iv = 0;
  for (int ib = 2; ib <= na; ++ib)
    for (int ia = 2; ia <= na; ++ia) {
      int id = ind_diff[(size_t)(ia - 1) * na + (ib - 1)];
      if (id > 0) {
        t->pair_ia[iv] = ia;
        t->pair_id[iv] = id;
        t->pair_binom[iv] = binom[(size_t)(ia - 1) * na + (ib - 1)];
        iv++;
      }
    }

  /* forward convolution tables (:299-332) */
  int kq = (k > 2 ? k : 2) - 1;
  t->kq = kq;
  t->fq_start = (int *)malloc(sizeof(int) * (size_t)na * kq);
  t->fq_num = (int *)calloc((size_t)na * kq, sizeof(int));
  for (int i = 0; i < na * kq; ++i) t->fq_start[i] = 1;
  int nfq = 0;
  for (int ia = 2; ia <= na; ++ia) {
    int p = t->deg[ia - 1];
    for (int q = 2; q <= p; ++q)
      for (int ib = 2; ib <= na; ++ib)
        if (ind_diff[(size_t)(ia - 1) * na + (ib - 1)] > 0 &&
            p - t->deg[ib - 1] >= q - 1)
          nfq++;
  }
  t->nfq = nfq;
  t->fq_ib = (int *)malloc(sizeof(int) * (nfq > 0 ? nfq : 1));
  t->fq_id = (int *)malloc(sizeof(int) * (nfq > 0 ? nfq : 1));
  t->fq_c = (double *)malloc(sizeof(double) * (nfq > 0 ? nfq : 1));
  iv = 0;
  for (int ia = 2; ia <= na; ++ia) {
    int p = t->deg[ia - 1];
    for (int q = 2; q <= p; ++q) {
      t->fq_start[(size_t)(ia - 1) * kq + (q - 2)] = iv + 1;
      for (int ib = 2; ib <= na; ++ib) {
        int id = ind_diff[(size_t)(ia - 1) * na + (ib - 1)];
        if (id > 0 && p - t->deg[ib - 1] >= q - 1) {
          t->fq_ib[iv] = ib;
          t->fq_id[iv] = id;
          t->fq_c[iv] = binom[(size_t)(ia - 1) * na + (ib - 1)] / (double)q;
          iv++;
        }
      }
      t->fq_num[(size_t)(ia - 1) * kq + (q - 2)] =
          iv - t->fq_start[(size_t)(ia - 1) * kq + (q - 2)] + 1;
    }
  }
  free(ind_diff);
  free(binom);

  /* tanh derivative polynomials (build_tanh_poly, :406-429), qmax = K+1 */
  int qmax = k + 1;
  int ld = qmax + 2; /* rows i = 0..qmax+1 */
  t->tpc = (double *)calloc((size_t)ld * (qmax + 1), sizeof(double));
  double *dc = (double *)malloc(sizeof(double) * ld);
  t->tpc[0 * ld + 1] = 1.0;
  for (int q = 0; q <= qmax - 1; ++q) {
    for (int i = 0; i < ld; ++i) dc[i] = 0.0;
    for (int i = 0; i <= qmax; ++i) dc[i] = (double)(i + 1) * t->tpc[q * ld + i + 1];
    for (int i = 0; i <= qmax + 1; ++i) {
      t->tpc[(q + 1) * ld + i] = dc[i];
      if (i >= 2) t->tpc[(q + 1) * ld + i] = t->tpc[(q + 1) * ld + i] - dc[i - 2];
    }
  }
  free(dc);
  return t;
}

void orc_tables_free(orc_tables *t) {
  if (!t) return;
  free(t->alpha); free(t->deg); free(t->ind_e1);
  free(t->fq_start); free(t->fq_num); free(t->fq_ib); free(t->fq_id);
  free(t->fq_c); free(t->pair_start); free(t->pair_num); free(t->pair_ia);
  free(t->pair_id); free(t->pair_binom); free(t->tpc);
  free(t);
}

void orc_tables_sizes(const orc_tables *t, int *na, int *nfq, int *npair,
                      int *nbell) {
  if (na) *na = t->na;
  if (nfq) *nfq = t->nfq;
  if (npair) *npair = t->npair;
  if (nbell) *nbell = t->nbell;
}

void orc_tables_copy(const orc_tables *t, int *alpha, int *deg, int *ind_e1,
                     int *fq_start, int *fq_num, int *fq_ib, int *fq_id,
                     double *fq_c, int *pair_start, int *pair_num,
                     int *pair_ia, int *pair_id, double *pair_binom,
                     double *tpc) {
  int na = t->na, d0 = t->d0, kq = t->kq;
  if (alpha) memcpy(alpha, t->alpha, sizeof(int) * (size_t)na * d0);
  if (deg) memcpy(deg, t->deg, sizeof(int) * na);
  if (ind_e1) memcpy(ind_e1, t->ind_e1, sizeof(int) * d0);
  /* fq_start / fq_num as [na][K-1] (q = 2..K); kq may exceed K-1 at K=1 */
  int kk = t->k - 1;
  for (int ia = 0; ia < na; ++ia)
    for (int c = 0; c < kk; ++c) {
      if (fq_start) fq_start[ia * kk + c] = t->fq_start[ia * kq + c];
      if (fq_num) fq_num[ia * kk + c] = t->fq_num[ia * kq + c];
    }
  if (fq_ib) memcpy(fq_ib, t->fq_ib, sizeof(int) * t->nfq);
  if (fq_id) memcpy(fq_id, t->fq_id, sizeof(int) * t->nfq);
  if (fq_c) memcpy(fq_c, t->fq_c, sizeof(double) * t->nfq);
  if (pair_start) memcpy(pair_start, t->pair_start, sizeof(int) * na);
  if (pair_num) memcpy(pair_num, t->pair_num, sizeof(int) * na);
  if (pair_ia) memcpy(pair_ia, t->pair_ia, sizeof(int) * t->npair);
  if (pair_id) memcpy(pair_id, t->pair_id, sizeof(int) * t->npair);
  if (pair_binom) memcpy(pair_binom, t->pair_binom, sizeof(double) * t->npair);
  if (tpc) memcpy(tpc, t->tpc, sizeof(double) * (size_t)(t->k + 3) * (t->k + 2));
}

/* tanh_derivs_ts (:852-867): Horner in t = tanh(a) */
void orc_tanh_derivs(const orc_tables *t, double a, int nq, double *d) {
  int ld = t->k + 3;
  double tt = tanh(a);
  for (int q = 0; q <= nq; ++q) {
    double v = t->tpc[q * ld + q + 1];
    for (int i = q; i >= 0; --i) v = v * tt + t->tpc[q * ld + i];
    d[q] = v;
  }
}

/* sin_derivs (lib/multi_index_bell_module.f90:745-755): every derivative is
 * a phase shift, sigma^(q)(a) = sin(a + q pi/2) */
static void sin_derivs(double a, int nq, double *d) {
  const double pio2 = 1.57079632679489661923;
  for (int q = 0; q <= nq; ++q) d[q] = sin(a + (double)q * pio2);
}

/* erf_derivs (:831-850): sigma' = (2/sqrt(pi)) exp(-a^2) and the higher
 * derivatives through the Hermite-function recurrence
 * psi_{n+1} = 2 a psi_n - 2 n psi_{n-1}, psi_0 = exp(-a^2).  The value
 * itself is libm's erf (the reference carries its own series / continued
 * fraction; both are correctly rounded to a few ulps). */
static void erf_derivs(double a, int nq, double *d) {
  const double c2spi = 1.12837916709551257390;
  d[0] = erf(a);
  if (nq < 1) return;
  double psi[64];
  psi[0] = exp(-a * a);
  psi[1] = 2.0 * a * psi[0];
  for (int n = 1; n <= nq - 2 && n + 1 < 64; ++n)
    psi[n + 1] = 2.0 * a * psi[n] - 2.0 * (double)n * psi[n - 1];
  for (int q = 1; q <= nq; ++q) d[q] = c2spi * ((q - 1) % 2 ? -1.0 : 1.0) * psi[q - 1];
}

/* J_0(x) .. J_n(x) (n <= 62): for |x| < 1e-5 two terms of the power
 * series, otherwise Miller's backward recurrence
 *   J_{k-1}(x) = (2k / x) J_k(x) - J_{k+1}(x)
 * started at an even index well above max(n, |x|) and normalised by
 *   J_0(x) + 2 sum_{k >= 1} J_{2k}(x) = 1
 * (Abramowitz & Stegun 9.1.27, 9.1.46; the method of 9.12), with a
 * rescale whenever the unnormalised values grow past 1e200.  Negative
 * arguments by J_n(-x) = (-1)^n J_n(x), as the reference's besj_series
 * wrapper does (lib/bessel_module.f90:50-72).  The reference computes the
 * values with Zhang and Jin's jyna; this is an independent method, pinned
 * against scipy in the tests. */
void orc_besj_all(int n, double x, double *bj) {
  const double ax = fabs(x);
  if (ax < 1e-5) {
    // two terms of the power series, (x/2)^k / k! (1 - (x/2)^2 / (k + 1));
    // the next term is below 1e-21 of the first
    const double h = 0.5 * x;
    double p = 1.0;
    for (int k = 0; k <= n; ++k) {
      bj[k] = p * (1.0 - h * h / (double)(k + 1));
      p = p * h / (double)(k + 1);
    }
    return;
  }
  const double top = ax > n ? ax : (double)n;
  int m = (int)top + 30 + (int)(3.0 * sqrt(top));
  m += m & 1;
  double jp1 = 0.0, j = 1.0, sum = 0.0;
  for (int k = m; k >= 1; --k) {
    const double jm1 = (2.0 * k / ax) * j - jp1;
    jp1 = j;
    j = jm1; /* J_{k-1} */
    if (k - 1 <= n) bj[k - 1] = j;
    if (k - 1 >= 2 && !((k - 1) & 1)) sum += 2.0 * j;
    if (fabs(j) > 1e200) {
      j *= 1e-200;
      jp1 *= 1e-200;
      sum *= 1e-200;
      for (int i = k - 1; i <= n; ++i) bj[i] *= 1e-200;
    }
  }
  sum += j;
  for (int i = 0; i <= n; ++i) bj[i] /= sum;
  if (x < 0.0)
    for (int i = 1; i <= n; i += 2) bj[i] = -bj[i];
}

/* besj0_derivs / besj1_derivs (lib/multi_index_bell_module.f90:757-826):
 *   J_0^(q) = ((-1)^q / 2^q) sum_k (-1)^k C(q,k) J_{q-2k},
 *   J_1^(q) = ((-1)^q / 2^q) sum_k (-1)^k C(q,k) J_{1+q-2k},
 * J_{-n} = (-1)^n J_n, the binomials built as C(q,k+1) = C(q,k)(q-k)/(k+1) */
static void besj_derivs(int shift, double a, int nq, double *d) {
  double bj[64];
  orc_besj_all(nq + shift, a, bj);
  for (int q = 0; q <= nq; ++q) {
    double term = 0.0, c = 1.0;
    for (int k = 0; k <= q; ++k) {
      const int m = shift + q - 2 * k;
      const double sk = (k & 1) ? -1.0 : 1.0;
      if (m >= 0) term = term + sk * c * bj[m];
      else term = term + sk * c * ((-m) & 1 ? -1.0 : 1.0) * bj[-m];
      c = c * (double)(q - k) / (double)(k + 1);
    }
    d[q] = (q & 1 ? -1.0 : 1.0) * term / ldexp(1.0, q);
  }
}

/* act_derivs_ts (:723-741): the activation contract, sigma^(q), q = 0..nq */
void orc_act_derivs(const orc_tables *t, double a, int nq, double *d) {
  if (t->iact == 1) sin_derivs(a, nq, d);
  else if (t->iact == 2) erf_derivs(a, nq, d);
  else if (t->iact == 3) besj_derivs(0, a, nq, d);
  else if (t->iact == 4) besj_derivs(1, a, nq, d);
  else orc_tanh_derivs(t, a, nq, d);
}

int orc_tables_set_activation(orc_tables *t, int iact) {
  if (iact < 0 || iact > 4) return -1;
  t->iact = iact;
  return 0;
}

int orc_weight_count(int nlayer, const int *dims) {
  int n = 0;
  for (int l = 1; l < nlayer; ++l) n += dims[l] * (dims[l - 1] + 1);
  return n;
}

/* ------------------------------------------------------------------ */
/* Per-point work space, laid out like twork_t (lib/train_module.f90:74-90):
 * T(0:ndmax, na, nlayer) with the neuron index fastest, h(1:ndmax, na,
 * nlayer), and one plane each for S, Tb, Sb plus the Bell scratch
 * bqv(ndmax, na, K). */
typedef struct {
  int ndmax, na, nlayer, k;
  double *T, *h, *S, *Tb, *Sb, *bqv, *dt, *acc;
  double *ttv, *htv, *bsv;
} work;

static void work_init(work *wk, const orc_tables *t, int nlayer,
                      const int *dims) {
  int ndmax = 0;
  for (int l = 0; l < nlayer; ++l) if (dims[l] > ndmax) ndmax = dims[l];
  wk->ndmax = ndmax;
  wk->na = t->na;
  wk->nlayer = nlayer;
  wk->k = t->k;
  size_t plane0 = (size_t)(ndmax + 1) * t->na;
  size_t plane = (size_t)ndmax * t->na;
  wk->T = (double *)calloc(plane0 * nlayer, sizeof(double));
  wk->h = (double *)calloc(plane * nlayer, sizeof(double));
  wk->S = (double *)calloc(plane, sizeof(double));
  wk->Tb = (double *)calloc(plane, sizeof(double));
  wk->Sb = (double *)calloc(plane, sizeof(double));
  wk->bqv = (double *)calloc(plane * (t->k > 1 ? t->k : 1), sizeof(double));
  wk->dt = (double *)calloc((size_t)ndmax * (t->k + 2), sizeof(double));
  wk->acc = (double *)calloc((size_t)ndmax * (ndmax + 1), sizeof(double));
  wk->ttv = (double *)calloc(ndmax, sizeof(double));
  wk->htv = (double *)calloc(ndmax, sizeof(double));
  wk->bsv = (double *)calloc(ndmax, sizeof(double));
  for (int l = 0; l < nlayer; ++l) wk->T[plane0 * l] = 1.0; /* bias channel */
}

static void work_free(work *wk) {
  free(wk->T); free(wk->h); free(wk->S); free(wk->Tb); free(wk->Sb);
  free(wk->bqv); free(wk->dt); free(wk->acc); free(wk->ttv); free(wk->htv);
  free(wk->bsv);
}

#define TT(wk, i, ia, l) \
  (wk)->T[(size_t)(i) + ((size_t)(wk)->ndmax + 1) * ((size_t)(ia) + (size_t)(wk)->na * (l))]
#define HH(wk, j, ia, l) \
  (wk)->h[(size_t)(j) + (size_t)(wk)->ndmax * ((size_t)(ia) + (size_t)(wk)->na * (l))]
#define PL(arr, wk, j, ia) (arr)[(size_t)(j) + (size_t)(wk)->ndmax * (size_t)(ia)]
#define BQ(wk, j, ia, q) \
  (wk)->bqv[(size_t)(j) + (size_t)(wk)->ndmax * ((size_t)(ia) + (size_t)(wk)->na * (q))]
#define DT(wk, j, q) (wk)->dt[(size_t)(j) + (size_t)(wk)->ndmax * (size_t)(q)]

static const double *layer_w(const double *w, const int *dims, int l) {
  /* l is 1-based in the reference's sense (2..nlayer) */
  const double *p = w;
  for (int ll = 2; ll < l; ++ll) p += (size_t)dims[ll - 1] * (dims[ll - 2] + 1);
  return p;
}

/* forward_core (lib/train_module.f90:241-335); store_h = 0 gives the
 * net_eval_hod arithmetic (lib/net_module.f90:295-375), which is the same
 * sequence minus the h cache. */
static void forward_core(const orc_tables *t, work *wk, const int *dims,
                         const double *w, const double *x, int store_h) {
  int na = t->na, kq = t->kq, nlayer = wk->nlayer;
  double dsc[32];
  for (int j = 1; j <= dims[0]; ++j) {
    TT(wk, j, 0, 0) = x[j - 1];
    for (int ia = 1; ia < na; ++ia) TT(wk, j, ia, 0) = 0.0;
    if (t->ind_e1[j - 1] > 0) TT(wk, j, t->ind_e1[j - 1] - 1, 0) = 1.0;
  }
  for (int l = 2; l <= nlayer; ++l) {
    int nd = dims[l - 1], ndm = dims[l - 2];
    const double *wl = layer_w(w, dims, l); /* wl[j][i], i = 0 bias */
    int lc = l - 1, lp = l - 2;             /* 0-based layer planes */
    for (int ia = 0; ia < na; ++ia) {
      for (int j = 0; j < nd; ++j)
        PL(wk->S, wk, j, ia) = wl[(size_t)j * (ndm + 1) + 0] * TT(wk, 0, ia, lp);
      for (int i = 1; i <= ndm; ++i)
        for (int j = 0; j < nd; ++j)
          PL(wk->S, wk, j, ia) = PL(wk->S, wk, j, ia) +
                                 wl[(size_t)j * (ndm + 1) + i] * TT(wk, i, ia, lp);
    }
    if (l < nlayer) {
      for (int j = 0; j < nd; ++j) {
        orc_act_derivs(t, PL(wk->S, wk, j, 0), t->k + 1, dsc);
        for (int q = 0; q <= t->k + 1; ++q) DT(wk, j, q) = dsc[q];
      }
      for (int j = 0; j < nd; ++j) {
        TT(wk, j + 1, 0, lc) = DT(wk, j, 0);
        if (store_h) HH(wk, j, 0, lc) = DT(wk, j, 1);
      }
      for (int ia = 2; ia <= na; ++ia) {
        int p = t->deg[ia - 1];
        for (int j = 0; j < nd; ++j) {
          BQ(wk, j, ia - 1, 0) = PL(wk->S, wk, j, ia - 1);
          wk->ttv[j] = DT(wk, j, 1) * PL(wk->S, wk, j, ia - 1);
          wk->htv[j] = DT(wk, j, 2) * PL(wk->S, wk, j, ia - 1);
        }
        for (int q = 2; q <= p; ++q) {
          for (int j = 0; j < nd; ++j) wk->bsv[j] = 0.0;
          int st = t->fq_start[(size_t)(ia - 1) * kq + (q - 2)];
          int nn = t->fq_num[(size_t)(ia - 1) * kq + (q - 2)];
          for (int it = st; it <= st + nn - 1; ++it) {
            double c = t->fq_c[it - 1];
            int ib = t->fq_ib[it - 1] - 1, id = t->fq_id[it - 1] - 1;
            for (int j = 0; j < nd; ++j)
              wk->bsv[j] = wk->bsv[j] + c * PL(wk->S, wk, j, ib) * BQ(wk, j, id, q - 2);
          }
          for (int j = 0; j < nd; ++j) {
            BQ(wk, j, ia - 1, q - 1) = wk->bsv[j];
            wk->ttv[j] = wk->ttv[j] + DT(wk, j, q) * wk->bsv[j];
            wk->htv[j] = wk->htv[j] + DT(wk, j, q + 1) * wk->bsv[j];
          }
        }
        for (int j = 0; j < nd; ++j) {
          TT(wk, j + 1, ia - 1, lc) = wk->ttv[j];
          if (store_h) HH(wk, j, ia - 1, lc) = wk->htv[j];
        }
      }
    } else {
      for (int ia = 0; ia < na; ++ia)
        for (int j = 0; j < nd; ++j) TT(wk, j + 1, ia, lc) = PL(wk->S, wk, j, ia);
    }
  }
}

/* backward_core (lib/train_module.f90:360-450) after the seeding of
 * net_backward_point_multi (:459-475) */
static void backward_core(const orc_tables *t, work *wk, const int *dims,
                          const double *w, const double *seedm, double *grad) {
  int na = t->na, nlayer = wk->nlayer;
  int nout = dims[nlayer - 1];
  for (int ia = 0; ia < na; ++ia)
    for (int j = 0; j < nout; ++j)
      PL(wk->Tb, wk, j, ia) = seedm[(size_t)j * na + ia];
  for (int l = nlayer; l >= 2; --l) {
    int nd = dims[l - 1], ndm = dims[l - 2];
    int lc = l - 1, lp = l - 2;
    if (l == nlayer) {
      for (int ia = 0; ia < na; ++ia)
        for (int j = 0; j < nd; ++j) PL(wk->Sb, wk, j, ia) = PL(wk->Tb, wk, j, ia);
    } else {
      for (int j = 0; j < nd; ++j)
        wk->bsv[j] = PL(wk->Tb, wk, j, 0) * HH(wk, j, 0, lc);
      for (int ia = 1; ia < na; ++ia)
        for (int j = 0; j < nd; ++j)
          wk->bsv[j] = wk->bsv[j] + PL(wk->Tb, wk, j, ia) * HH(wk, j, ia, lc);
      for (int j = 0; j < nd; ++j) PL(wk->Sb, wk, j, 0) = wk->bsv[j];
      for (int ib = 2; ib <= na; ++ib) {
        for (int j = 0; j < nd; ++j) wk->bsv[j] = 0.0;
        int st = t->pair_start[ib - 1], nn = t->pair_num[ib - 1];
        for (int ip = st; ip <= st + nn - 1; ++ip) {
          double c = t->pair_binom[ip - 1];
          int ia = t->pair_ia[ip - 1] - 1, id = t->pair_id[ip - 1] - 1;
          for (int j = 0; j < nd; ++j)
            wk->bsv[j] = wk->bsv[j] + c * PL(wk->Tb, wk, j, ia) * HH(wk, j, id, lc);
        }
        for (int j = 0; j < nd; ++j) PL(wk->Sb, wk, j, ib - 1) = wk->bsv[j];
      }
    }
    /* gradient block: acc(1:nd,0:ndm) = sum_ia Sb(:,ia) T(0:ndm,ia,l-1) */
    double *acc = wk->acc; /* acc[i][j], j fastest, like acc(1:nd, 0:ndm) */
    for (int i = 0; i <= ndm; ++i)
      for (int j = 0; j < nd; ++j) acc[(size_t)i * wk->ndmax + j] = 0.0;
    for (int ia = 0; ia < na; ++ia)
      for (int i = 0; i <= ndm; ++i)
        for (int j = 0; j < nd; ++j)
          acc[(size_t)i * wk->ndmax + j] = acc[(size_t)i * wk->ndmax + j] +
                                           PL(wk->Sb, wk, j, ia) * TT(wk, i, ia, lp);
    double *gl = (double *)layer_w(grad, dims, l);
    for (int j = 0; j < nd; ++j)
      for (int i = 0; i <= ndm; ++i)
        gl[(size_t)j * (ndm + 1) + i] = gl[(size_t)j * (ndm + 1) + i] +
                                        acc[(size_t)i * wk->ndmax + j];
    if (l > 2) {
      const double *wl = layer_w(w, dims, l);
      for (int ia = 0; ia < na; ++ia)
        for (int i = 1; i <= ndm; ++i) {
          double s = 0.0;
          for (int j = 0; j < nd; ++j)
            s = s + wl[(size_t)j * (ndm + 1) + i] * PL(wk->Sb, wk, j, ia);
          PL(wk->Tb, wk, i - 1, ia) = s;
        }
    }
  }
}

int orc_eval_point(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, const double *x, double *tout,
                   double *tall) {
  if (nlayer < 2 || dims[0] != t->d0) return -1;
  work wk;
  work_init(&wk, t, nlayer, dims);
  forward_core(t, &wk, dims, w, x, 0);
  for (int ia = 0; ia < t->na; ++ia) tout[ia] = TT(&wk, 1, ia, nlayer - 1);
  if (tall)
    for (int j = 0; j < dims[nlayer - 1]; ++j)
      for (int ia = 0; ia < t->na; ++ia)
        tall[(size_t)j * t->na + ia] = TT(&wk, j + 1, ia, nlayer - 1);
  work_free(&wk);
  return 0;
}

int orc_grad_point(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, const double *x, const double *seedm,
                   double *grad, double *tout) {
  if (nlayer < 2 || dims[0] != t->d0) return -1;
  work wk;
  work_init(&wk, t, nlayer, dims);
  forward_core(t, &wk, dims, w, x, 1);
  if (tout)
    for (int ia = 0; ia < t->na; ++ia) tout[ia] = TT(&wk, 1, ia, nlayer - 1);
  backward_core(t, &wk, dims, w, seedm, grad);
  work_free(&wk);
  return 0;
}

double orc_pinn_residual(const orc_seed_rule *r, const double *t) {
  double R = 0.0;
  for (int k = 0; k < r->nterm; ++k) {
    if (r->nonlin[k])
      R = R + r->coeff[k] * t[0] * t[r->ind[k] - 1];
    else
      R = R + r->coeff[k] * t[r->ind[k] - 1];
  }
  return R;
}

void orc_pinn_seed(const orc_seed_rule *r, const double *t, double R,
                   double fac, double *seed, int na) {
  for (int i = 0; i < na; ++i) seed[i] = 0.0;
  for (int k = 0; k < r->nterm; ++k) {
    int ind = r->ind[k] - 1;
    if (r->nonlin[k]) {
      seed[ind] = seed[ind] + fac * R * r->coeff[k] * t[0];
      seed[0] = seed[0] + fac * R * r->coeff[k] * t[ind];
    } else {
      seed[ind] = seed[ind] + fac * R * r->coeff[k];
    }
  }
}

int orc_grad_batch(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, int npts, const double *X,
                   const orc_seed_rule *rule, const double *seeds,
                   double *grad, double *rows, double *tout, double *loss,
                   int nthreads) {
  if (nlayer < 2 || dims[0] != t->d0 || dims[nlayer - 1] < 1) return -1;
  int na = t->na, d0 = t->d0;
  int nw = orc_weight_count(nlayer, dims);
  int nout = dims[nlayer - 1];
  if (rule->kind == ORC_SEED_JROW && !rows) return -1;
  if (grad) memset(grad, 0, sizeof(double) * nw);
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  double total = 0.0;
  int nthr = nthreads;
  double *gthr = (double *)calloc((size_t)nthr * nw, sizeof(double));
  double *lthr = (double *)calloc(nthr, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel num_threads(nthr)
#endif
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    work wk;
    work_init(&wk, t, nlayer, dims);
    double *tv = (double *)malloc(sizeof(double) * na);
    double *sd = (double *)calloc((size_t)nout * na, sizeof(double));
    double *g = gthr + (size_t)tid * nw;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int n = 0; n < npts; ++n) {
      forward_core(t, &wk, dims, w, X + (size_t)n * d0, 1);
      for (int ia = 0; ia < na; ++ia) tv[ia] = TT(&wk, 1, ia, nlayer - 1);
      if (tout) memcpy(tout + (size_t)n * na, tv, sizeof(double) * na);
      memset(sd, 0, sizeof(double) * (size_t)nout * na);
      double *gdst = g;
      if (rule->kind == ORC_SEED_GIVEN) {
        memcpy(sd, seeds + (size_t)n * na, sizeof(double) * na);
      } else if (rule->kind == ORC_SEED_HALFSQ) {
        double l = 0.0;
        for (int ia = 0; ia < na; ++ia) { sd[ia] = tv[ia]; l += tv[ia] * tv[ia]; }
        lthr[tid] += 0.5 * l;
      } else if (rule->kind == ORC_SEED_PINN) {
        double R = orc_pinn_residual(rule, tv);
        orc_pinn_seed(rule, tv, R, rule->fac, sd, na);
        lthr[tid] += 0.5 * rule->fac * R * R;
      } else { /* ORC_SEED_JROW */
        orc_pinn_seed(rule, tv, 1.0, 1.0, sd, na);
        gdst = rows + (size_t)n * nw;
        memset(gdst, 0, sizeof(double) * nw);
      }
      backward_core(t, &wk, dims, w, sd, gdst);
    }
    free(tv);
    free(sd);
    work_free(&wk);
  }
  if (grad)
    for (int th = 0; th < nthr; ++th)
      for (int i = 0; i < nw; ++i) grad[i] += gthr[(size_t)th * nw + i];
  for (int th = 0; th < nthr; ++th) total += lthr[th];
  if (loss) *loss = total;
  free(gthr);
  free(lthr);
  return 0;
}

void orc_sys_residual(const orc_sys_rule *r, const double *tm, int na, const double *src,
                      double *R) {
  for (int ir = 0; ir < r->nres; ++ir) R[ir] = src ? -src[ir] : 0.0;
  int f = 0;
  for (int k = 0; k < r->nterm; ++k) {
    double prod = r->coeff[k];
    for (int m = 0; m < r->nfac[k]; ++m)
      prod = prod * tm[(size_t)(r->comp[f + m] - 1) * na + r->slot[f + m] - 1];
    R[r->res[k] - 1] = R[r->res[k] - 1] + prod;
    f += r->nfac[k];
  }
}

void orc_sys_seed(const orc_sys_rule *r, const double *tm, int na, int nout, const double *R,
                  double *seedm) {
  for (int i = 0; i < nout * na; ++i) seedm[i] = 0.0;
  int f = 0;
  for (int k = 0; k < r->nterm; ++k) {
    const int ir = r->res[k] - 1;
    const double wr = r->wres ? r->wres[ir] : 1.0;
    for (int m = 0; m < r->nfac[k]; ++m) {
      double other = r->fac * wr * R[ir] * r->coeff[k];
      for (int mm = 0; mm < r->nfac[k]; ++mm) {
        if (mm == m) continue;
        other = other * tm[(size_t)(r->comp[f + mm] - 1) * na + r->slot[f + mm] - 1];
      }
      const size_t at = (size_t)(r->comp[f + m] - 1) * na + r->slot[f + m] - 1;
      seedm[at] = seedm[at] + other;
    }
    f += r->nfac[k];
  }
}

int orc_grad_sys_batch(const orc_tables *t, int nlayer, const int *dims, const double *w,
                       int npts, const double *X, const orc_sys_rule *rule,
                       const double *src, double *grad, double *tout, double *loss,
                       int nthreads) {
  if (nlayer < 2 || dims[0] != t->d0 || !rule || rule->nres < 1 || rule->nterm < 1) return -1;
  const int na = t->na, d0 = t->d0, nout = dims[nlayer - 1], nres = rule->nres;
  {
    int f = 0;
    for (int k = 0; k < rule->nterm; ++k) {
      if (rule->res[k] < 1 || rule->res[k] > nres || rule->nfac[k] < 1) return -1;
      for (int m = 0; m < rule->nfac[k]; ++m, ++f)
        if (rule->comp[f] < 1 || rule->comp[f] > nout || rule->slot[f] < 1 || rule->slot[f] > na)
          return -1;
    }
  }
  const int nw = orc_weight_count(nlayer, dims);
  if (grad) memset(grad, 0, sizeof(double) * nw);
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  const int nthr = nthreads;
  double *gthr = (double *)calloc((size_t)nthr * nw, sizeof(double));
  double *lthr = (double *)calloc(nthr, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel num_threads(nthr)
#endif
  {
#ifdef _OPENMP
    int tid = omp_get_thread_num();
#else
    int tid = 0;
#endif
    work wk;
    work_init(&wk, t, nlayer, dims);
    double *tm = (double *)malloc(sizeof(double) * (size_t)nout * na);
    double *sd = (double *)malloc(sizeof(double) * (size_t)nout * na);
    double *R = (double *)malloc(sizeof(double) * nres);
    double *g = gthr + (size_t)tid * nw;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int n = 0; n < npts; ++n) {
      forward_core(t, &wk, dims, w, X + (size_t)n * d0, 1);
      for (int o = 0; o < nout; ++o)
        for (int ia = 0; ia < na; ++ia) tm[(size_t)o * na + ia] = TT(&wk, o + 1, ia, nlayer - 1);
      if (tout) memcpy(tout + (size_t)n * nout * na, tm, sizeof(double) * (size_t)nout * na);
      orc_sys_residual(rule, tm, na, src ? src + (size_t)n * nres : NULL, R);
      double l = 0.0;
      for (int ir = 0; ir < nres; ++ir) l += (rule->wres ? rule->wres[ir] : 1.0) * R[ir] * R[ir];
      lthr[tid] += 0.5 * rule->fac * l;
      orc_sys_seed(rule, tm, na, nout, R, sd);
      backward_core(t, &wk, dims, w, sd, g);
    }
    free(tm);
    free(sd);
    free(R);
    work_free(&wk);
  }
  if (grad)
    for (int th = 0; th < nthr; ++th)
      for (int i = 0; i < nw; ++i) grad[i] += gthr[(size_t)th * nw + i];
  double total = 0.0;
  for (int th = 0; th < nthr; ++th) total += lthr[th];
  if (loss) *loss = total;
  free(gthr);
  free(lthr);
  return 0;
}

static void kf_downdate(int nw, double *P, int nblk, const int *bsz, const int *boff,
                        const double *kv, const double *pj, double lm, double q);
static void kf_pj(int nw, const double *P, int nblk, const int *bsz, const int *boff,
                  const double *jf, double *pj);

int orc_kf_update(int nw, double *w, double *P, int nblk, const int *bsz, const int *boff,
                  const double *jrow, double xi_in, double scale, double *lam, double lam0,
                  double q, double gate, int *ngated) {
  double *jf = (double *)calloc(nw > 0 ? nw : 1, sizeof(double));
  double *pj = (double *)malloc(sizeof(double) * nw);
  double *kv = (double *)malloc(sizeof(double) * nw);
  double xi = scale * xi_in;
  for (int m = 0; m < nw; ++m) jf[m] = scale * jrow[m];
  kf_pj(nw, P, nblk, bsz, boff, jf, pj);
  double dot = 0.0;
  for (int m = 0; m < nw; ++m) dot += jf[m] * pj[m];
  double denom = *lam + dot;
  if (!(denom > 0.0)) {
    free(jf); free(pj); free(kv);
    return -1;
  }
  if (gate > 0.0) {
    const double jpj = denom - *lam;
    if (xi * xi > gate * gate * denom) {
      const double s2 = gate * gate * *lam / (xi * xi - gate * gate * jpj);
      const double sq = sqrt(s2);
      xi = sq * xi;
      for (int m = 0; m < nw; ++m) pj[m] = sq * pj[m];
      denom = *lam + s2 * jpj;
      ++*ngated;
    }
  }
  for (int m = 0; m < nw; ++m) kv[m] = pj[m] / denom;
  for (int m = 0; m < nw; ++m) w[m] = w[m] + kv[m] * xi;
  kf_downdate(nw, P, nblk, bsz, boff, kv, pj, *lam, q);
  *lam = lam0 * *lam + 1.0 - lam0;
  free(jf); free(pj); free(kv);
  return 0;
}

/* P j per block (dense: nblk = 0) */
static void kf_pj(int nw, const double *P, int nblk, const int *bsz, const int *boff,
                  const double *jf, double *pj) {
  if (nblk > 0) {
    const double *Pb = P;
    for (int b = 0; b < nblk; ++b) {
      const int n = bsz[b], o = boff[b];
      for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int r = 0; r < n; ++r) s += Pb[(size_t)r * n + i] * jf[o + r];
        pj[o + i] = s;
      }
      Pb += (size_t)n * n;
    }
  } else {
    for (int i = 0; i < nw; ++i) {
      double s = 0.0;
      for (int r = 0; r < nw; ++r) s += P[(size_t)r * nw + i] * jf[r];
      pj[i] = s;
    }
  }
}

int orc_kf_iekf_iter(int nw, double *w, const double *wprior, double *P, int nblk,
                     const int *bsz, const int *boff, const double *jrow, double resid,
                     double rnoise, double *lam, double lam0, double q, int final) {
  if (!(rnoise > 0.0)) return -1;
  const double scale = 1.0 / sqrt(rnoise);
  double *jf = (double *)calloc(nw > 0 ? nw : 1, sizeof(double));
  double *pj = (double *)malloc(sizeof(double) * nw);
  double *kv = (double *)malloc(sizeof(double) * nw);
  for (int m = 0; m < nw; ++m) jf[m] = scale * jrow[m];
  kf_pj(nw, P, nblk, bsz, boff, jf, pj);
  double dot = 0.0;
  for (int m = 0; m < nw; ++m) dot += jf[m] * pj[m];
  const double denom = *lam + dot;
  if (!(denom > 0.0)) {
    free(jf); free(pj); free(kv);
    return -1;
  }
  for (int m = 0; m < nw; ++m) kv[m] = pj[m] / denom;
  double corr = 0.0;
  for (int m = 0; m < nw; ++m) corr += jf[m] * (wprior[m] - w[m]);
  const double xi = -scale * resid - corr;
  for (int m = 0; m < nw; ++m) w[m] = wprior[m] + kv[m] * xi;
  if (final) {
    kf_downdate(nw, P, nblk, bsz, boff, kv, pj, *lam, q);
    *lam = lam0 * *lam + 1.0 - lam0;
  }
  free(jf); free(pj); free(kv);
  return 0;
}

/* (P - kv pj^T) / lambda, the average with the transpose and the process
 * noise on the diagonal, per block (kf_update_grad :449-489) */
static void kf_downdate(int nw, double *P, int nblk, const int *bsz, const int *boff,
                        const double *kv, const double *pj, double lm, double q) {
  if (nblk > 0) {
    double *Pb = P;
    for (int b = 0; b < nblk; ++b) {
      const int n = bsz[b], o = boff[b];
      for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r)
          Pb[(size_t)r * n + c] = (Pb[(size_t)r * n + c] - kv[o + r] * pj[o + c]) / lm;
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
          const double a = 0.5 * (Pb[(size_t)i * n + j] + Pb[(size_t)j * n + i]);
          Pb[(size_t)i * n + j] = a;
          Pb[(size_t)j * n + i] = a;
        }
      if (q > 0.0)
        for (int i = 0; i < n; ++i) Pb[(size_t)i * n + i] += q;
      Pb += (size_t)n * n;
    }
  } else {
    for (int c = 0; c < nw; ++c)
      for (int r = 0; r < nw; ++r)
        P[(size_t)r * nw + c] = (P[(size_t)r * nw + c] - kv[r] * pj[c]) / lm;
    for (int i = 0; i < nw; ++i)
      for (int j = i + 1; j < nw; ++j) {
        const double a = 0.5 * (P[(size_t)i * nw + j] + P[(size_t)j * nw + i]);
        P[(size_t)i * nw + j] = a;
        P[(size_t)j * nw + i] = a;
      }
    if (q > 0.0)
      for (int i = 0; i < nw; ++i) P[(size_t)i * nw + i] += q;
  }
}

int orc_eval_batch(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, int npts, const double *X, double *tout,
                   int nthreads) {
  if (nlayer < 2 || dims[0] != t->d0) return -1;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
  {
    work wk;
    work_init(&wk, t, nlayer, dims);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int n = 0; n < npts; ++n) {
      forward_core(t, &wk, dims, w, X + (size_t)n * t->d0, 0);
      for (int ia = 0; ia < t->na; ++ia)
        tout[(size_t)n * t->na + ia] = TT(&wk, 1, ia, nlayer - 1);
    }
    work_free(&wk);
  }
  return 0;
}

void orc_adam_step(int nw, double *w, const double *grad, double *m,
                   double *v, double eta, double beta1, double beta2,
                   double eps, int nbatch, int istep) {
  int s = istep > 1 ? istep : 1;
  /* real**integer is evaluated by binary powering in gfortran */
  double p1 = 1.0, p2 = 1.0, x1 = beta1, x2 = beta2;
  for (unsigned u = (unsigned)s;;) {
    if (u & 1u) { p1 *= x1; p2 *= x2; }
    u >>= 1;
    if (!u) break;
    x1 *= x1;
    x2 *= x2;
  }
  double bc1 = 1.0 - p1;
  double bc2 = 1.0 - p2;
  for (int i = 0; i < nw; ++i) {
    double gval = grad[i] / (double)nbatch;
    m[i] = beta1 * m[i] + (1.0 - beta1) * gval;
    v[i] = beta2 * v[i] + (1.0 - beta2) * (gval * gval);
    w[i] = w[i] - eta * (m[i] / bc1) / (sqrt(v[i] / bc2) + eps);
  }
}

/* The metric build of ngd_apply_inv alone (app/optimizer_module.f90:
 * 310-321): G(i,j) += jr(ib,i) jr(ib,j) row by row, in the reference's loop
 * order; G[nw][nw] is overwritten.  The CPU baseline times it. */
void orc_ngd_metric(int nw, int nrow, const double *rows, double *G) {
  memset(G, 0, sizeof(double) * (size_t)nw * nw);
  for (int ib = 0; ib < nrow; ++ib) {
    const double *r = rows + (size_t)ib * nw;
    for (int j = 0; j < nw; ++j)
      for (int i = 0; i < nw; ++i)
        G[(size_t)j * nw + i] = G[(size_t)j * nw + i] + r[i] * r[j];
  }
}

int orc_ngd_step(int nw, int nrow, const double *rows, const double *b,
                 int nb, double mu, double *u) {
  double *G = (double *)calloc((size_t)nw * nw, sizeof(double));
  /* Gm(i,j) += jr(ib,i) jr(ib,j), row by row (:310-321) */
  for (int ib = 0; ib < nrow; ++ib) {
    const double *r = rows + (size_t)ib * nw;
    for (int j = 0; j < nw; ++j)
      for (int i = 0; i < nw; ++i)
        G[(size_t)j * nw + i] = G[(size_t)j * nw + i] + r[i] * r[j];
  }
  for (size_t i = 0; i < (size_t)nw * nw; ++i) G[i] = G[i] / (double)nb;
  for (int i = 0; i < nw; ++i) u[i] = b[i] / (double)nb;
  for (int i = 0; i < nw; ++i) G[(size_t)i * nw + i] = G[(size_t)i * nw + i] + mu;
  /* gauss_solve (:472-522); G is symmetric, A(i,j) = G[j*nw+i] */
#define A(i, j) G[(size_t)(j) * nw + (i)]
  double anorm = 0.0;
  for (size_t i = 0; i < (size_t)nw * nw; ++i)
    if (fabs(G[i]) > anorm) anorm = fabs(G[i]);
  double ptol = 1e-13 * anorm;
  for (int k = 0; k < nw - 1; ++k) {
    int ip = k;
    double pmax = fabs(A(k, k));
    for (int i = k + 1; i < nw; ++i)
      if (fabs(A(i, k)) > pmax) { pmax = fabs(A(i, k)); ip = i; }
    if (pmax <= ptol) { free(G); return -1; }
    if (ip != k) {
      for (int j = k; j < nw; ++j) { double r = A(k, j); A(k, j) = A(ip, j); A(ip, j) = r; }
      double r = u[k]; u[k] = u[ip]; u[ip] = r;
    }
    for (int i = k + 1; i < nw; ++i) {
      double fac = A(i, k) / A(k, k);
      for (int j = k; j < nw; ++j) A(i, j) = A(i, j) - fac * A(k, j);
      u[i] = u[i] - fac * u[k];
    }
  }
  for (int i = nw - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = i + 1; j < nw; ++j) s = s + A(i, j) * u[j];
    u[i] = (u[i] - s) / A(i, i);
  }
#undef A
  free(G);
  return 0;
}
