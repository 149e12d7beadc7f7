/* dnnf90_b200.h - entry points of the B200 device path beyond the 24 of
 * dnnf90.h.  The reference evaluates one point per call
 * (lib/train_module.f90:198-209); these take whole batches, either in host
 * memory (copies to and from the device inside the call) or already on the
 * device with a caller stream (the torch.autograd.Function path).
 *
 * Layouts: x[npts][d0]; t[npts][na] (output 1, slot order of dnnf90_alpha);
 * tm[npts][nout][na]; seed[npts][na] (output 1) or seedm[npts][nout][na];
 * weights and gradients in the flat layer layout: layers 2..nlayer
 * concatenated, each dims[l-1] rows of dims[l-2]+1 doubles, bias first
 * (the dnnf90_net_set_layer row layout, lib/c_api_module.f90:185-205).
 * Return codes as in dnnf90.h.
 */
#ifndef DNNF90_B200_H
#define DNNF90_B200_H
#include "dnnf90.h"
#ifdef __cplusplus
extern "C" {
#endif

/* precision of a network's device path.  0 = plain FP64 (every kernel in
 * FP64; agrees with the reference to rounding).  1 = split: FP32 planes and
 * Bell arithmetic, sigma^(q) in FP64, layer GEMMs as 3-term split-BF16
 * products with FP32 accumulation on the tensor cores, FP64 gradient
 * reductions.  New; the reference is FP64 only. */
int dnnf90_net_set_precision(int nid, int prec);
/* release a table-set handle (the reference keeps every set until exit;
 * there are 64 handles).  Networks created on the set keep working: each
 * holds its own copy.  new */
int dnnf90_tabset_free(int tid);
/* number of weights of a network (flat layout); new */
int dnnf90_nweights(int nid);
/* read layer l back in the dnnf90_net_set_layer row layout; new */
int dnnf90_net_get_layer(int nid, int l, double *wrow);
/* write a network in nn_weight.dat format; counterpart of net_save,
 * lib/net_module.f90:219-243 */
int dnnf90_net_save(int nid, const char *filename);

/* net_eval_hod over a batch (lib/net_module.f90:295-375 per point) */
int dnnf90_eval_batch(int nid, int wid, int npts, const double *x, double *t);
/* net_eval_hod_multi over a batch (lib/net_module.f90:389-408) */
int dnnf90_eval_batch_multi(int nid, int wid, int npts, const double *x,
                            double *tm);
/* net_grad_point over a batch with caller seeds (lib/train_module.f90:
 * 478-489 per point), added to accumulator gid */
int dnnf90_grad_batch(int nid, int tid, int npts, const double *x,
                      const double *seed, int gid);

/* A seed rule: the loss seed formed on the device from each point's output
 * derivatives (app/pinn_module.f90:32-65).  kind 1: L = sum_a T_a^2/2,
 * seed = T.  kind 2: R = sum_k coeff_k T_{slot_k} (times T_1 when
 * nonlin_k), L = fac R^2/2, seed = fac R dR/dT (set_pinn_seed).  kind 3:
 * seed = dR/dT, one Jacobian row per point (app/lib_net_module.f90:
 * 314-330).  slot is 1-based.  Returns a rule handle. */
int dnnf90_seed_rule_create(int kind, int nterm, const double *coeff,
                            const int *slot, const int *nonlin, double fac);
int dnnf90_seed_rule_free(int rid);
/* A system seed rule (calc_sys_residual / set_sys_seed, app/pinn_module.f90:
 * 86-162): several residuals over several output components.  Term k adds
 *   coeff[k] * T(comp, slot) * ...   (nfac[k] factors, 1 <= nfac[k] <= 4)
 * to residual res[k]; its factors follow those of terms < k in comp[] and
 * slot[].  R_r = -src_r + (sum of its terms), L = fac/2 sum_r wres[r] R_r^2,
 * seed = fac sum_r wres[r] R_r dR_r/dT, each factor of a term seeded with
 * the product of the term's other factors.  res, comp and slot are 1-based;
 * 1 <= nres <= 8; wres may be NULL (all 1).  Usable with
 * dnnf90_grad_rule_batch / _dev (sources zero) and dnnf90_grad_sys_batch;
 * the Jacobian-row entries refuse it.  Returns a rule handle. */
int dnnf90_seed_rule_sys(int nres, int nterm, const int *res, const double *coeff,
                         const int *nfac, const int *comp, const int *slot,
                         const double *wres, double fac);
/* forward -> device seed -> adjoint over a batch, added to gid; loss (sum
 * over points) and t (output 1) may be NULL */
int dnnf90_grad_rule_batch(int nid, int tid, int npts, const double *x,
                           int rid, int gid, double *loss, double *t);
/* forward -> system seed with sources src[npts][nres] (NULL: zero) ->
 * adjoint over a batch, added to gid; loss (sum over points) and
 * tm[npts][nout][na] (every output component) may be NULL.  The batched
 * form of the reference's per-point calc_sys_residual / set_sys_seed /
 * net_backward_point_multi loop (app/pinn_module.f90:86-162,
 * lib/train_module.f90:459-475); new */
int dnnf90_grad_sys_batch(int nid, int tid, int npts, const double *x, const double *src,
                          int rid, int gid, double *loss, double *tm);
/* the value-only fit of net_grad_batch (lib/train_module.f90:525-631) over
 * a batch: L = coef/2 sum_n (N(x_n) - y_n)^2 for a single-output network,
 * dL/dw added to gid, loss (may be NULL) = L.  Only the value slot enters;
 * a network on the table set that carries the value alone (the closure of
 * {0}) evaluates no derivative. */
int dnnf90_grad_value_batch(int nid, int tid, int npts, const double *x, const double *y,
                            double coef, int gid, double *loss);
/* Jacobian rows of a rule's residual, rows[npts][nweights]; resid[npts]
 * (the residual R per point) and t may be NULL */
int dnnf90_jrow_batch(int nid, int tid, int npts, const double *x, int rid,
                      double *rows, double *resid, double *t);
/* flush the points queued for gid and copy the accumulator out */
int dnnf90_grad_read(int gid, double *g);
/* damped Gauss-Newton step of app/optimizer_module.f90:221-469 with the ABS
 * damping: u = (J^T J / nb + mu I)^{-1} (b / nb), rows[nrow][nw], b[nw].
 * prec 1 forms the metric as split-precision tensor-core products, prec 0
 * in FP64; the solve is an FP64 Cholesky factorization. */
int dnnf90_ngd_step(int nid, int nrow, const double *rows, const double *b,
                    int nb, double mu, int prec, double *u);
/* the same step by the dual (Gram-space) route of app/optimizer_module.f90:
 * 408-446: K = mu I + J J^T / nb (nrow x nrow), y = K^{-1} J (b / nb),
 * u = (b / nb - J^T y / nb) / mu.  The nw x nw metric is never formed, so
 * it is the route for nrow < nw; the step equals the primal one to
 * roundoff.  K is formed in FP64 whatever prec says: the final division
 * by mu after a cancellation would magnify split-product rounding.
 * mu > 0. */
int dnnf90_ngd_step_dual(int nid, int nrow, const double *rows, const double *b,
                         int nb, double mu, int prec, double *u);

/* the primal step in two halves on device arrays, for rows spread over
 * ranks (app/optimizer_module.f90:310-321): G_dev[nw][nw] = J^T J of this
 * rank's rows (lower triangle; prec as in dnnf90_ngd_step), then, after the
 * caller has summed G and b over the ranks, u_dev = (G / nb + mu I)^{-1}
 * (b / nb) with nb the total row count.  The solve overwrites G_dev with
 * its Cholesky factor. */
int dnnf90_ngd_gram_dev(int nrow, int nw, const double *rows_dev, int prec, double *G_dev,
                        void *stream);
int dnnf90_ngd_solve_dev(int nw, double *G_dev, const double *b_dev, int nb, double mu,
                         double *u_dev, void *stream);
/* the dual route of dnnf90_ngd_step_dual on device arrays (rows gathered
 * from every rank, app/optimizer_module.f90:303-307) */
int dnnf90_ngd_step_dual_dev(int nrow, int nw, const double *rows_dev, const double *b_dev,
                             int nb, double mu, double *u_dev, void *stream);

/* ---- extended Kalman filter (lib/kalman_module.f90; new at the C boundary,
 * the reference reaches it from its trainer, app/lib_net_module.f90:455-570) */
/* kf_init (:107-170) on network nid: P = p0 I, lambda = lam_ini, forgetting
 * schedule lambda <- lam0 lambda + 1 - lam0.  decoupled != 0 keeps one
 * covariance block per neuron over (bias, fan-in) instead of the dense
 * nw x nw matrix.  q >= 0 is added to the diagonal after every update and
 * gate >= 0 bounds the normalised innovation (0 = off for both).  p0 > 0 and
 * lam_ini, lam0 in (0, 1], else -1.  Returns the filter handle (> 0). */
int dnnf90_kf_create(int nid, double p0, double lam_ini, double lam0, int decoupled,
                     double q, double gate);
int dnnf90_kf_free(int kid);
/* nobs rank-one updates, in order, of kf_update_grad (:353-490): rows[k][nw]
 * = dy/dw of observation k in the flat layout, xi[k] = target - prediction,
 * scale[k] (NULL = 1) multiplying both (1/sqrt of an observation noise).
 * The network's weights are updated.  A denominator lambda + j.Pj that is
 * not positive stops the sequence there with -1 (the observations before it
 * stay applied); the reference stops the process instead. */
int dnnf90_kf_update_rows(int kid, int nobs, const double *rows, const double *xi,
                          const double *scale);
/* the same on device arrays; w_dev[nw] (flat layout) is updated in place
 * and the network's own weights are left alone.  Returns after the work on
 * stream has finished, with the filter's status checked; while the stream
 * is being captured into a graph it returns without waiting, and
 * dnnf90_kf_status tells after a replay whether an update failed. */
int dnnf90_kf_update_rows_dev(int kid, int nobs, const double *rows_dev,
                              const double *xi_dev, const double *scale_dev,
                              double *w_dev, void *stream);
/* a filter pass over npts points x[npts][d0] with a Jacobian-row rule:
 * for each point in order, its row dR/dw and residual R at the network's
 * current weights, then the update with xi = -R and scale 1/sqrt(rnoise)
 * (kf_update_resid / kf_update_resid_multi, :252-300, as the trainer's
 * lnet_kalman_resid calls them per point).  Everything stays on the device
 * between points.  tid: a training work space of the filter's network,
 * which must run in FP64 (else -5).  -1 for rnoise <= 0 or at a nonpositive
 * denominator (the points before it stay applied). */
int dnnf90_kf_pass(int kid, int tid, int npts, const double *x, int rid, double rnoise);
/* the same pass with the iterated update: for each point the current
 * weights become the prior and niter >= 1 relinearisations follow, each from
 * the row and residual at the weights the last one left; the last downdates
 * the covariance (kf_iekf_begin / kf_iekf_iter, :509-640).  niter = 1 is the
 * plain pass. */
int dnnf90_kf_pass_iekf(int kid, int tid, int npts, const double *x, int rid, double rnoise,
                        int niter);
/* the filter pass over a system of residuals (a rule of
 * dnnf90_seed_rule_sys), as the trainer presents one (app/sgd_batch_module.f90:
 * 497-545): for each point and each residual r in turn, at the network's
 * current weights, R_r (with src[npts][nres], NULL for none) and its row
 * dR_r/dw (seeded unweighted with dR_r/dT), then the update of
 * kf_update_resid_multi with xi = -R_r and scale 1/sqrt(rnoise[r])
 * (rnoise NULL: 1).  niter >= 1 takes the iterated update with niter
 * relinearisations per residual; 0 the plain one.  FP64 networks only. */
int dnnf90_kf_pass_sys(int kid, int tid, int npts, const double *x, const double *src,
                       int rid, const double *rnoise, int niter);
/* iterated EKF (kf_iekf_begin / kf_iekf_iter, :509-640): begin stores the
 * network's current weights as the prior w-.  Each iteration takes
 * row = dR/dw and resid = R evaluated by the caller at the network's current
 * weights w_i, and sets the weights to w- + K_i (-s R - s row.(w- - w_i)),
 * s = 1/sqrt(rnoise), with the gain from the unchanged prior covariance.
 * final != 0 also downdates the covariance and advances lambda, so one
 * observation costs one covariance update however many iterations it
 * takes; one final iteration is the plain update.  The gate does not
 * apply.  -1 without a prior, for rnoise <= 0 or a nonpositive
 * denominator. */
int dnnf90_kf_iekf_begin(int kid);
int dnnf90_kf_iekf_iter(int kid, const double *row, double resid, double rnoise, int final);
/* filter state: lambda, the count of gated updates, and (P not NULL) the
 * covariance, dense [nw][nw] or the decoupled blocks [n_b][n_b] one after
 * another in the weight order */
int dnnf90_kf_read(int kid, double *lam, int *ngated, double *P);
/* the filter's status after its last call: 0, or 1 + the observation at
 * which a denominator was not positive (the updates from there on were not
 * applied); -3 if a device wait gave up; -1 for a bad handle */
int dnnf90_kf_status(int kid);

/* ---- device-pointer entry points (pointers to device memory; stream is
 * a cudaStream_t, NULL for the legacy default stream).  On the split path
 * the compute entries return after the work on stream has finished, having
 * checked the tensor-core GEMMs' error flag (-3 if one gave up); while the
 * stream is being captured into a graph they return without waiting. ---- */
/* weights from a device array in the flat layout */
int dnnf90_set_weights_dev(int nid, const double *w_dev, void *stream);
/* forward of npts points: tm_dev[npts][na][nout] (may be NULL).  keep = 1
 * keeps every plane on work space tid for dnnf90_backward_dev. */
int dnnf90_forward_dev(int nid, int tid, int npts, const double *x_dev,
                       double *tm_dev, int keep, void *stream);
/* *fits = 1 when a keep=1 forward of npts points fits work space tid: every
 * layer's planes for all the points (their size follows from |A|, that is
 * from D0 and K, and the widths) within the work space's budget, the
 * smaller of 48 GiB and half of the free device memory, and within its
 * chunk (dnnf90_twork_set_chunk); 0 otherwise, when the backward recomputes
 * the forward chunk by chunk instead. */
int dnnf90_keep_fits(int nid, int tid, int npts, int *fits);
/* adjoint from seedm_dev[npts][nout][na], added to grad_dev[nweights].  Uses
 * the planes kept by the last keep=1 forward of the same points and
 * weights on tid; otherwise recomputes the forward first. */
int dnnf90_backward_dev(int nid, int tid, int npts, const double *x_dev,
                        const double *seedm_dev, double *grad_dev,
                        void *stream);
/* forward -> rule seed -> adjoint, grad_dev += dL/dw, loss_dev[0] += L;
 * tm_dev (may be NULL) receives the output derivatives [npts][na][nout] */
int dnnf90_grad_rule_dev(int nid, int tid, int npts, const double *x_dev,
                         int rid, double *grad_dev, double *loss_dev,
                         double *tm_dev, void *stream);
/* Jacobian rows rows_dev[npts][nweights] of a rule's residual */
int dnnf90_jrow_dev(int nid, int tid, int npts, const double *x_dev, int rid,
                    double *rows_dev, double *tm_dev, void *stream);
/* points per device chunk of a training work space (0 = automatic) */
int dnnf90_twork_set_chunk(int tid, int npts);

/* One training step of nnet independent networks (a committee) of any
 * widths, depths, table sets, point counts and precisions: for member i,
 * grad_dev[i] = dL_i/dw_i and loss_dev[i] = L_i (both overwritten) from
 * rule rids[i] over npts[i] points x_dev[i][npts][d0], on work space
 * tids[i] (distinct per member).  The members run as concurrent branches of
 * one CUDA graph, each member's kernels sized to a share of the SMs.  The
 * first call with a given set of members and buffers builds the graph: it
 * sizes every member's work chunk under one memory budget, runs one untimed
 * step, captures one graph per SM-sharing policy (by work, by its square
 * root, none) and keeps the fastest replay; later calls replay it (weights
 * changed in between are re-uploaded in place first).  Returns after the
 * step has finished on stream.  Members replace the reference's per-network
 * loop over net_grad_point (lib/train_module.f90:478-489); new. */
int dnnf90_committee_step(int nnet, const int *nids, const int *tids, const int *rids,
                          const int *npts, const double *const *x_dev,
                          double *const *grad_dev, double *loss_dev, void *stream);
/* the Bell kernels' autotuner: one line per tuned launch shape, "kernel d0
 * k na width precision chosen-variant ms-of-each-variant" (the table set's
 * D0, K and |A|); returns the length (buf may be NULL); new */
int dnnf90_tune_report(char *buf, int len);
/* pin the variant of the Bell forward (which 0: 0 records in global memory,
 * 1 records in shared memory, 2 per-degree loops over 16-bit offset records)
 * or adjoint (which 1: 0 pairs in global memory, 1 in shared memory,
 * 2 grouped correlation) kernels for every later launch; variant -1 hands
 * the choice back to the autotuner, and a variant a launch shape cannot use
 * runs its default.  which 2 switches the tanh forward by the series
 * identity tanh' = 1 - tanh^2 (for tanh on sets closed under b <= a whose
 * state fits shared memory): 1 on, 0 or -1 off (the default; the Bell
 * recurrence measured faster).  The two forwards agree to rounding.  which 3
 * picks the Kalman update path: 0 two launches per update, 1 one
 * cooperative launch per call, -1 by size (the default: one launch for
 * small filters); the two give identical bits.  For reproducible timing and
 * for tests; new */
int dnnf90_tune_force(int which, int variant);
/* policy (0 work, 1 square root, 2 none) and timed replay ms of the graph
 * the last committee step used; new */
int dnnf90_committee_info(int *policy, float *graph_ms);

/* dnnf90_ngd_step (plain FP64 route) on device buffers rows_dev[nrow][nw],
 * b_dev[nw], u_dev[nw], for callers that cannot allocate device memory
 * while they run: a host whose device memory is all handed out up front by
 * its own allocator or pool, or a caller under a fixed device-memory
 * budget.  No counterpart in the reference (its gauss_solve works on host
 * arrays).  The call allocates nothing: the nw x nw metric sits in a fixed
 * 8 MiB area inside the library that every GPU loading the library keeps
 * until the process exits, so nw <= 1024; larger nw is refused (-1) with a
 * message in dnnf90_last_error(); mu <= 0 is refused (-1) as well.  The
 * first call on a device looks up the area's device address and, under
 * CUDA's lazy module loading, loads the library's module on that device,
 * which is when the 8 MiB area is taken from device memory: make one call
 * before the host pools its device memory.  The address is kept for the
 * life of the process and does not survive cudaDeviceReset.  Every call
 * shares the area: calls that overlap on the GPU (other threads, other
 * streams) race and must be serialised by the caller.  The call waits for
 * stream (NULL: the legacy default stream) and reads a status back, so it
 * cannot be captured into a CUDA graph: on a capturing stream it returns -5
 * without doing anything. */
int dnnf90_ngd_step_noalloc(int nrow, int nw, const double *rows_dev,
                            const double *b_dev, int nb, double mu,
                            double *u_dev, void *stream);

/* text of the last error on this thread; 1 if a CUDA device is usable */
const char *dnnf90_last_error(void);
int dnnf90_device_available(void);
/* number of kernels this library has launched in the process */
long long dnnf90_launch_count(void);
/* per-kernel device timing: while enabled every launch is bracketed by CUDA
 * events on its stream; read writes "name launches total_ms" lines into buf
 * (returns the length needed) and clears the record */
int dnnf90_profile_enable(int on);
int dnnf90_profile_read(char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif
