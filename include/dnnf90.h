/* dnnf90.h - C interface of the B200 device path of DNNF90's
 * derivative-carrying evaluation and its adjoint.
 *
 * Drop-in for the reference's lib/dnnf90.h: the same 24 entry points with
 * the same signatures, argument meaning and return codes (handles > 0,
 * errors < 0, 0 = success; lib/dnnf90.h:4-8, lib/c_api_module.f90:17-23).
 * Each declaration names the reference function it replaces.  Link against
 * libdnnf90_b200.so.  Further codes of this library: -3 device error or no
 * GPU, -4 device memory exhausted, -5 valid for the reference but outside
 * the device path (dnnf90_last_error() gives the reason).
 *
 * Batched and device-pointer entry points are in dnnf90_b200.h.
 */
#ifndef DNNF90_H
#define DNNF90_H
#ifdef __cplusplus
extern "C" {
#endif

/* shared read-only tables (call one of these once, first) */
/* replaces dnnf90_tables_init_dense, lib/c_api_module.f90:100-108 */
int dnnf90_tables_init_dense(int d0, int k);
/* replaces dnnf90_tables_init_closure, lib/c_api_module.f90:113-125;
 * seeds: d0*nseed ints, seed s at seeds[s*d0 .. s*d0+d0-1] */
int dnnf90_tables_init_closure(int d0, int k, int nseed, const int *seeds);
/* replaces dnnf90_nderiv, lib/c_api_module.f90:128-130 */
int dnnf90_nderiv(void);
/* replaces dnnf90_alpha, lib/c_api_module.f90:133-141 (ia is 1-based) */
int dnnf90_alpha(int ia, int *a);

/* independent table sets (per-species descriptor count and order) */
/* replaces dnnf90_tabset_dense, lib/c_api_module.f90:407-421 */
int dnnf90_tabset_dense(int d0, int k);
/* replaces dnnf90_tabset_closure, lib/c_api_module.f90:423-441 */
int dnnf90_tabset_closure(int d0, int k, int nseed, const int *seeds);
/* replaces dnnf90_tabset_nderiv, lib/c_api_module.f90:443-452 */
int dnnf90_tabset_nderiv(int tid);
/* replaces dnnf90_net_create_ts, lib/c_api_module.f90:454-474 */
int dnnf90_net_create_ts(int tid, int nlayer, const int *dims);

/* networks */
/* replaces dnnf90_net_load, lib/c_api_module.f90:145-166 (nn_weight.dat) */
int dnnf90_net_load(const char *filename);
/* replaces dnnf90_tabset_activation, lib/c_api_module.f90:480-493.
 * Codes: 0 TANH, 1 SIN, 2 ERF, 3 BESSEL (J_0), 4 BESSEL1 (J_1); the device
 * path evaluates all five. */
int dnnf90_tabset_activation(int tid, int iact);
/* replaces dnnf90_net_load_ts, lib/c_api_module.f90:500-528 */
int dnnf90_net_load_ts(int tid, const char *filename);
/* replaces dnnf90_net_create, lib/c_api_module.f90:169-183 */
int dnnf90_net_create(int nlayer, const int *dims);
/* replaces dnnf90_net_set_layer, lib/c_api_module.f90:189-205: dims[l-1]
 * rows of dims[l-2]+1 doubles, each the bias then the incoming weights */
int dnnf90_net_set_layer(int nid, int l, const double *wrow);
/* replaces dnnf90_net_free, lib/c_api_module.f90:207-218 */
int dnnf90_net_free(int nid);

/* evaluation (value and all carried mixed derivatives) */
/* replaces dnnf90_work_create, lib/c_api_module.f90:221-236 */
int dnnf90_work_create(int nid);
/* replaces dnnf90_work_free, lib/c_api_module.f90:238-249 */
int dnnf90_work_free(int wid);
/* replaces dnnf90_eval, lib/c_api_module.f90:253-278 (synchronous) */
int dnnf90_eval(int nid, int wid, const double *x, double *t);

/* training (gradient accumulation and Adam) */
/* replaces dnnf90_twork_create, lib/c_api_module.f90:282-297 */
int dnnf90_twork_create(int nid);
/* replaces dnnf90_twork_free, lib/c_api_module.f90:299-310 */
int dnnf90_twork_free(int tid);
/* replaces dnnf90_grad_create, lib/c_api_module.f90:312-327 */
int dnnf90_grad_create(int nid);
/* replaces dnnf90_grad_free, lib/c_api_module.f90:329-340 */
int dnnf90_grad_free(int gid);
/* replaces dnnf90_grad_zero, lib/c_api_module.f90:342-352 */
int dnnf90_grad_zero(int gid);
/* replaces dnnf90_grad_point, lib/c_api_module.f90:358-380.  The point is
 * queued on the training work space and computed in a batch when the
 * accumulator is next used (adam_step, grad_zero, grad_free, grad_read),
 * when the weights change, or when the queue is full: no entry of the
 * reference interface can observe an accumulator before then. */
int dnnf90_grad_point(int nid, int tid, const double *x,
                      const double *seed, int gid);
/* replaces dnnf90_adam_step, lib/c_api_module.f90:384-400 */
int dnnf90_adam_step(int nid, int gid, double eta, double beta1,
                     double beta2, double eps, int nbatch, int istep);

#ifdef __cplusplus
}
#endif
#endif
