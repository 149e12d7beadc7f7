/* oracle.h - CPU FP64 restatement of DNNF90's derivative-carrying forward
 * pass and its adjoint.  TEST INFRASTRUCTURE ONLY: the checker that the
 * tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg run beside
 * the CUDA path.  Nothing in the product library links or calls it.
 *
 * Every routine follows the reference's arithmetic in the reference's loop
 * and summation order (no FMA contraction: build with -ffp-contract=off),
 * so that on x86-64 it reproduces the default gfortran -O3 build of the
 * reference bit for bit.  Citations are path:line into the reference tree.
 *
 * Pinning: tests/test_oracle_golden.py checks this code against the
 * reference's shipped golden vectors (zwork/hod_4d_k3, hod_4d_k7,
 * hod_4d_k7_active hod_golden.dat), against the reference's independent
 * Taylor-jet tool (tools/make_hod_golden.py) on further shapes, against the
 * table counts in its logs, and against the directional known-answer table
 * of bench/cpp/README.md:97-105 (weights bench/julia/wx_ref.txt).
 */
#ifndef DNNF90_ORACLE_H
#define DNNF90_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tables orc_tables;

/* init_hod_tables (lib/multi_index_bell_module.f90:128-351).  nseed = 0
 * builds the dense set; otherwise seeds holds nseed multi-indices of d0
 * ints each.  Returns NULL on bad arguments (the reference stops). */
orc_tables *orc_tables_build(int d0, int k, int nseed, const int *seeds);
void orc_tables_free(orc_tables *t);

/* sizes: na, number of fq terms, number of pair terms, Bell terms
 * (bell_enum count, printed as "Bell table terms" by the reference) */
void orc_tables_sizes(const orc_tables *t, int *na, int *nfq, int *npair,
                      int *nbell);
/* Copies of the tables, 1-based indices exactly as the reference stores
 * them.  alpha: [na][d0]; deg: [na]; ind_e1: [d0];
 * fq_start/fq_num: [na][K-1] for q = 2..K (column q-2);
 * fq_ib/fq_id/fq_c: [nfq]; pair_start/pair_num: [na];
 * pair_ia/pair_id/pair_binom: [npair]; tpc: [(K+3)*(K+2)] = tpc(i,q) at
 * q*(K+3)+i. Any pointer may be NULL. */
void orc_tables_copy(const orc_tables *t, int *alpha, int *deg, int *ind_e1,
                     int *fq_start, int *fq_num, int *fq_ib, int *fq_id,
                     double *fq_c, int *pair_start, int *pair_num,
                     int *pair_ia, int *pair_id, double *pair_binom,
                     double *tpc);

/* sigma^(q)(a), q = 0..nq, tanh (tanh_derivs_ts,
 * lib/multi_index_bell_module.f90:852-867) */
void orc_tanh_derivs(const orc_tables *t, double a, int nq, double *d);
/* sigma^(q)(a) for the table set's activation (act_derivs_ts, :723-741):
 * 0 tanh, 1 sin (:745-755), 2 erf (:831-850), 3 J0 and 4 J1 (:757-826) */
void orc_act_derivs(const orc_tables *t, double a, int nq, double *d);
/* select the activation of a table set (dnnf90_tabset_activation); 0 on
 * success, -1 for codes outside 0..4 */
int orc_tables_set_activation(orc_tables *t, int iact);
/* J_0(x) .. J_n(x), n <= 62, into bj[0..n] (Miller's backward recurrence) */
void orc_besj_all(int n, double x, double *bj);

/* Network weights: layers l = 2..nlayer concatenated, each a row-major
 * [dims[l-1]][dims[l-2]+1] block whose row j is the bias followed by the
 * incoming weights (dnnf90_net_set_layer row layout,
 * lib/c_api_module.f90:185-205).  Gradients use the same layout. */
int orc_weight_count(int nlayer, const int *dims);

/* net_eval_hod (lib/net_module.f90:295-375): t[na] of output 1;
 * tall[nout*na] (may be NULL) receives every output, [output][slot]. */
int orc_eval_point(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, const double *x, double *tout,
                   double *tall);

/* net_forward_point + net_backward_point_multi
 * (lib/train_module.f90:210-218, 241-335, 341-450, 459-475): forward, then
 * the adjoint seeded with seedm[nout][na] (row 0 = the scalar seed), adding
 * dL/dw into grad.  tout[na] receives output 1 (may be NULL). */
int orc_grad_point(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, const double *x, const double *seedm,
                   double *grad, double *tout);

/* Seed rules, the losses the batched driver forms from each point's
 * output derivatives T (app/pinn_module.f90:32-65):
 *   ORC_SEED_GIVEN   seeds[npts][na] supplied by the caller
 *   ORC_SEED_HALFSQ  L = sum_a T_a^2 / 2, seed = T
 *   ORC_SEED_PINN    R = sum_k c_k T_{ind_k} (times T_1 if nonlin_k);
 *                    L = fac R^2 / 2, seed = fac R dR/dT (set_pinn_seed)
 *   ORC_SEED_JROW    seed = dR/dT (R = 1, fac = 1), one Jacobian row per
 *                    point written to rows[npts][nw] instead of summed */
enum { ORC_SEED_GIVEN = 0, ORC_SEED_HALFSQ = 1, ORC_SEED_PINN = 2,
       ORC_SEED_JROW = 3 };

typedef struct {
  int kind;
  int nterm;
  const double *coeff; /* [nterm] */
  const int *ind;      /* [nterm], 1-based slot */
  const int *nonlin;   /* [nterm], 1 = multiplies T_1 */
  double fac;
} orc_seed_rule;

/* Residual of one point (calc_pinn_residual, app/pinn_module.f90:32-47,
 * without a source term) and its seed (set_pinn_seed, :50-65). */
double orc_pinn_residual(const orc_seed_rule *r, const double *t);
void orc_pinn_seed(const orc_seed_rule *r, const double *t, double R,
                   double fac, double *seed, int na);

/* Batched driver: per point, forward, seed by rule, adjoint; gradients
 * summed over points into grad (zeroed first) with one accumulator per
 * thread (tools/example_train.f90:139-153).  tout[npts][na] and
 * loss (sum over points) may be NULL.  seeds used for ORC_SEED_GIVEN,
 * rows for ORC_SEED_JROW.  nthreads <= 0 uses every core. */
int orc_grad_batch(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, int npts, const double *X,
                   const orc_seed_rule *rule, const double *seeds,
                   double *grad, double *rows, double *tout, double *loss,
                   int nthreads);

/* System seed rule (calc_sys_residual / set_sys_seed, app/pinn_module.f90:
 * 86-162): residual r of a point is
 *   R_r = -src_r + sum over the terms k of residual r of
 *         coeff_k * prod_{m < nfac_k} T(comp_{k,m}, slot_{k,m}),
 * the loss L = fac/2 sum_r w_r R_r^2 and the seed
 *   dL/dT(c, a) = fac sum_r w_r R_r dR_r/dT(c, a),
 * each factor of a term seeded with the product of the term's other
 * factors (accumulated, so a repeated factor counts twice).  res, comp,
 * slot are 1-based; the factors of term k follow those of terms < k in
 * comp/slot; wres may be NULL (all 1). */
typedef struct {
  int nres, nterm;
  const int *res;       /* [nterm] */
  const double *coeff;  /* [nterm] */
  const int *nfac;      /* [nterm] */
  const int *comp;      /* [sum nfac] */
  const int *slot;      /* [sum nfac] */
  const double *wres;   /* [nres] or NULL */
  double fac;
} orc_sys_rule;

/* tm[nout][na] of one point; src[nres] may be NULL (zero) */
void orc_sys_residual(const orc_sys_rule *r, const double *tm, int na, const double *src,
                      double *R);
/* seedm[nout][na], overwritten */
void orc_sys_seed(const orc_sys_rule *r, const double *tm, int na, int nout, const double *R,
                  double *seedm);
/* Batched driver for a system rule: per point forward (all outputs), seed,
 * adjoint; grad (zeroed first) summed over points, loss summed over points
 * (may be NULL), tout[npts][nout][na] (may be NULL), src[npts][nres] (may
 * be NULL).  Returns -1 on bad arguments. */
int orc_grad_sys_batch(const orc_tables *t, int nlayer, const int *dims, const double *w,
                       int npts, const double *X, const orc_sys_rule *rule,
                       const double *src, double *grad, double *tout, double *loss,
                       int nthreads);

/* Extended Kalman filter, rank-one update of kf_update_grad
 * (lib/kalman_module.f90:353-490) from one observation row jrow[nw]
 * (dy/dw in the flat layer order) with innovation xi and scale s (row and
 * innovation both scaled by s).  P is dense [nw][nw], or, decoupled,
 * nblk diagonal blocks [bsz][bsz] stored one after another (bsz[b] at
 * offset boff[b] of the flat weights); the denominator lambda + j.Pj is
 * global.  Optional innovation gate (gate > 0) and process noise q.
 * Updates w, P, *lam (lambda <- lam0 lambda + 1 - lam0) and *ngated.
 * Returns -1 if the denominator is not positive. */
int orc_kf_update(int nw, double *w, double *P, int nblk, const int *bsz, const int *boff,
                  const double *jrow, double xi_in, double scale, double *lam, double lam0,
                  double q, double gate, int *ngated);

/* One relinearisation of the iterated EKF, kf_iekf_iter
 * (lib/kalman_module.f90:534-640): jrow = dR/dw at the current weights w,
 * resid = R there, scale = 1/sqrt(rnoise).  w <- wprior + kv xi with
 * xi = -scale resid - (scale jrow).(wprior - w); the covariance and lambda
 * change only when final != 0.  No innovation gate.  -1 on rnoise <= 0 or a
 * nonpositive denominator. */
int orc_kf_iekf_iter(int nw, double *w, const double *wprior, double *P, int nblk,
                     const int *bsz, const int *boff, const double *jrow, double resid,
                     double rnoise, double *lam, double lam0, double q, int final);

/* Forward only over a batch (net_eval_hod per point). */
int orc_eval_batch(const orc_tables *t, int nlayer, const int *dims,
                   const double *w, int npts, const double *X, double *tout,
                   int nthreads);

/* opt_adam_step (lib/train_module.f90:656-683) on the flat weight layout;
 * m and v are the moments (zero on the first call). */
void orc_adam_step(int nw, double *w, const double *grad, double *m,
                   double *v, double eta, double beta1, double beta2,
                   double eps, int nbatch, int istep);

/* Primal natural-gradient step of app/optimizer_module.f90:221-469 with
 * the ABS damping: u = (J^T J / nb + mu I)^{-1} (b / nb), rows[nrow][nw],
 * solved by gauss_solve (:472-522, Gaussian elimination with partial
 * pivoting).  The flat layout here is the weight layout above; the
 * reference's flatten order only permutes the unknowns. Returns 0, or -1
 * on a singular pivot. */
void orc_ngd_metric(int nw, int nrow, const double *rows, double *G);
int orc_ngd_step(int nw, int nrow, const double *rows, const double *b,
                 int nb, double mu, double *u);

#ifdef __cplusplus
}
#endif
#endif
