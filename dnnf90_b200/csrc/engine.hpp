// engine.hpp - the device side of the derivative-carrying evaluation and its
// adjoint: device copies of table sets and weights, per-work-space plane
// buffers, and the batched forward / seed / adjoint driver.
//
// Layout in HBM (one chunk of P points at a time):
//   T_l, h_l  [P][na][n_l]   carried derivatives and the h cache of hidden
//                            layer l (neuron index fastest, so a warp reads
//                            one 128-byte line per multi-index)
//   S, Sb, Tb [P][na][nmax]  one layer at a time
//   out       [P][na][nout]  output derivatives (identity read-out)
//   seed      [P][nout][na]  dL/dT at the output
// The reference keeps the same per-point planes with the point axis absent
// (twork_t, lib/train_module.f90:74-90).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "bell.hpp"
#include "tables.hpp"

namespace dnnf90 {

enum Precision : int {
  PREC_F64 = 0,    // plain path: FP64 everywhere
  PREC_SPLIT = 1,  // FP32 planes and Bell arithmetic, sigma^(q) in FP64,
                   // layer GEMMs as 3-term split-BF16 products with FP32
                   // accumulation, FP64 gradient reductions
};

// error codes at the C boundary (the reference's are 0, -1, -2)
enum : int {
  RC_OK = 0,
  RC_BAD_ARG = -1,
  RC_BAD_FILE = -2,
  RC_DEVICE = -3,      // CUDA error or no usable GPU
  RC_NOMEM = -4,       // device allocation failed
  RC_UNSUPPORTED = -5  // valid for the reference, outside this device path
};

// seed rules evaluated on the device at the output layer
enum SeedKind : int {
  SEED_GIVEN = 0,   // caller supplied dL/dT per point
  SEED_HALFSQ = 1,  // L = sum_a T_a^2 / 2, seed = T
  SEED_PINN = 2,    // L = fac R^2 / 2 with R a linear / u*T_a term list
  SEED_JROW = 3,    // seed = dR/dT, per-point gradient rows
  SEED_SYS = 4      // system: R_r from products of several outputs' slots,
                    // L = fac/2 sum_r w_r R_r^2 (app/pinn_module.f90:86-162)
};

struct SeedRuleHost {
  int kind = SEED_HALFSQ;
  std::vector<double> coeff;
  std::vector<int> ind;     // 0-based slots
  std::vector<int> nonlin;  // 1: term is coeff * T_0 * T_ind
  double fac = 1.0;
  // SEED_SYS: term k adds coeff[k] * prod of its factors to residual
  // sys[3k]; its sys[3k + 1] factors start at sys[3k + 2] in sfac, pairs
  // (component, slot), 0-based; wres[nres] the residual weights
  int nres = 0;
  std::vector<int> sys, sfac;
  std::vector<double> wres;
};
constexpr int SYS_MAXRES = 8;   // residuals of a system rule
constexpr int SYS_MAXFAC = 4;   // factors of one term

// device copy of one table set
struct DevTables {
  int d0 = 0, k = 0, na = 0, nslot = 0, nfq = 0, npair = 0;
  int *deg = nullptr;        // [na]
  int *alpha = nullptr;      // [na][d0]
  int *ind_e1 = nullptr;     // [d0]
  int *seg = nullptr;        // [na][k+1][3] = {start, num, store slot}
  uint32_t *fq_pk = nullptr; // ib | operand << 16 (operand: S slot if q==2
                             // else state slot of B_{id,q-1})
  double *fq_c64 = nullptr;
  float *fq_c32 = nullptr;
  int *pseg = nullptr;       // [na][2] = {start, num}
  uint32_t *pair_pk = nullptr;  // ia | id << 16
  double *pair_c64 = nullptr;
  float *pair_c32 = nullptr;
  double *tpc = nullptr;     // [(k+2)][(k+3)]
  int iact = 0;
  // first-hidden-layer tables of the streaming kernels
  int *l2par = nullptr;      // [na]: slot of a - e_i | i << 16, i the first
                             // nonzero dimension of a (0 for a = 0)
  int *l2up = nullptr;       // [na][d0]: slot of g + e_i | (g_i + 1) << 16, or -1
  bool graded = false;       // slots ordered by degree
  std::vector<int> dstart;   // [k+2]: first slot of each degree
  DevBellPlan bp;            // work lists of the warp-cooperative kernels
  void release();
};

int upload_tables(const TableSet &t, DevTables &d);

// device copy of a network's weights
struct DevNet {
  int nlayer = 0, nw = 0;
  std::vector<int> dims;
  std::vector<size_t> woff;  // offset of layer l (index l-1) in the flat array
  double *w64 = nullptr;     // flat [layer][j][0..m]
  double *wpk = nullptr;     // 2 * nw: per layer (at 2 * woff) the plain path's GEMM
                             // operands without the bias column, [n][m] then [m][n],
                             // rewritten before each use (gemm_f64.cu)
  float *w32 = nullptr;      // FP32 copy for the split path
  void *tc = nullptr;        // pre-split tensor-core weight operands
  uint64_t uploaded = 0;     // host weight version on the device
  void release();
};

// per work-space device buffers, sized for a chunk of points
struct Planes {
  int cap_pts = 0;           // points per chunk
  int prec = -1;
  size_t bytes = 0;
  void *base = nullptr;      // one allocation, carved below
  std::vector<void *> T, h;  // per layer (index l-1), hidden layers only
  void *S = nullptr, *Sb = nullptr, *Tb = nullptr, *seed = nullptr;
  void *sig = nullptr;       // [P][k + 2][n_1]: s^(q)(S^0) of the first hidden layer
  void *scratch = nullptr;   // Bell state spill when it does not fit smem
  size_t scratch_bytes = 0;
  double *X = nullptr;       // [P][d0] staged inputs
  double *out = nullptr;     // [P][na][nout]
  double *loss = nullptr;    // [1]
  void release();
};

struct Stream {
  cudaStream_t s = nullptr;
};

// Batched driver over npts points already resident on the device.
//   X      [npts][d0]
//   out    [npts][na][nout] (may be null)
//   seeds  [npts][nout][na] for SEED_GIVEN
//   grad   flat FP64 weight layout, accumulated into (may be null: eval)
//   rows   [npts][nw] for SEED_JROW
//   loss   one double, accumulated into (may be null)
struct BatchArgs {
  int npts = 0;
  const double *X = nullptr;
  const double *src = nullptr;  // SEED_SYS sources [npts][nres] (may be null)
  double *out = nullptr;
  const double *seeds = nullptr;
  double *grad = nullptr;
  double *rows = nullptr;
  double *loss = nullptr;
  bool train = false;
  int prec = PREC_F64;
};

// device-side seed rule
struct DevRule {
  int kind = SEED_HALFSQ;
  int nterm = 0;
  double fac = 1.0;
  double *coeff = nullptr;
  int *ind = nullptr;
  int *nonlin = nullptr;
  int nres = 0;              // SEED_SYS (see SeedRuleHost)
  int *sys = nullptr, *sfac = nullptr;
  double *wres = nullptr;
  void release();
};
int upload_rule(const SeedRuleHost &r, DevRule &d);

int ensure_planes(const DevTables &t, const DevNet &n, int prec, int cap_pts,
                  Planes &p);
int run_batch(const DevTables &t, const DevNet &n, const DevRule &rule,
              Planes &p, const BatchArgs &a, cudaStream_t st);

// Forward of npts <= p.cap_pts points that keeps every plane, and the
// adjoint from a caller seed [npts][nout][na] on those planes (the
// store-and-reuse mode of the autograd backward).
int forward_keep(const DevTables &t, const DevNet &n, Planes &p, int prec,
                 int npts, const double *X, double *out, cudaStream_t st);
int adjoint_kept(const DevTables &t, const DevNet &n, Planes &p, int prec,
                 int npts, const double *X, const double *seed, double *grad,
                 cudaStream_t st);

// Adam update on the device (opt_adam_step, lib/train_module.f90:656-683);
// m and v are allocated by the caller and zero on the first call
int adam_device(double *w, const double *g, double *m, double *v, int nw,
                double eta, double b1, double b2, double eps, int nbatch,
                int istep, cudaStream_t st);

// Damped Gauss-Newton step of app/optimizer_module.f90:221-469 (ABS
// damping): u = (J^T J / nb + mu I)^{-1} (b / nb), J = rows[nrow][nw].
// The metric is formed on the tensor cores (split-precision) or in FP64
// (prec), then Cholesky-factored and solved in FP64.
int ngd_device(const double *rows, int nrow, int nw, const double *b, int nb,
               double mu, double *u, int prec, cudaStream_t st);
// The primal step in two halves: G = J^T J (lower triangle, FP64; prec as
// above) and the damped solve u = (G / nb + mu I)^{-1} (b / nb), which
// overwrites G with its factor
int ngd_gram_device(const double *rows, int nrow, int nw, double *G, int prec, cudaStream_t st);
int ngd_solve_device(double *G, int nw, const double *b, int nb, double mu, double *u,
                     cudaStream_t st);
// the same step by the dual (Gram-space) route, app/optimizer_module.f90:408-446
int ngd_device_dual(const double *rows, int nrow, int nw, const double *b, int nb, double mu,
                    double *u, int prec, cudaStream_t st);

// The same step on caller device buffers with the metric in a fixed
// scratch area of the library (no device allocation); nw <= ngd_noalloc_maxw().
int ngd_device_noalloc(const double *rows, int nrow, int nw, const double *b, int nb,
                       double mu, double *u, cudaStream_t st);
int ngd_noalloc_maxw();

// Extended Kalman filter (lib/kalman_module.f90): device scalars of the
// filter and of the observation being applied.
struct KfState {
  double lam, lam0, q, gate;       // current lambda, schedule, process noise, gate
  double lamk, denom, sg, xi;      // observation k: its lambda, denominator, gate scale, innovation
  int ngated;                      // gated updates so far
  int status;                      // 0, or 1 + the observation whose denominator was not positive
};

// grid barrier of the one-launch Kalman sequence
struct KfBar {
  unsigned count, gen;
};

// covariance in packed 32 x 32 tiles of each block's upper triangle
struct KfDev {
  int nw = 0, ntile = 0, nred = 0;
  bool dense = false;        // a single block (the global filter)
  double *P = nullptr;       // [ntile][32][32]
  int4 *tiles = nullptr;     // per tile: block offset, block size, I | J << 16, slot offset
  int4 *rtl = nullptr;       // per row tile: first weight, rows, slots, slot offset
  double *part = nullptr;    // per block [row tile][slot][32]: partial products
                             // of P with the next row
  double *pj = nullptr;      // [nw] P j of the observation being applied
  double *dotp = nullptr;    // per row tile: its shares of j.Pj and of j.(w- - w)
  unsigned *ctr = nullptr;   // reduce CTAs finished
  KfState *st = nullptr;
  KfBar *bar = nullptr;
  int seq_grid = 0;          // CTAs of the one-launch sequence (0: no cooperative launch)
  double *wprior = nullptr;  // [nw] iterated EKF: the prior weights
  bool prior = false;        // set by an IEKF begin
  double *stage = nullptr;   // host-call staging (rows, innovations, scales, weights)
  size_t stage_bytes = 0;
  void release();
};

// blocks (sizes bsz at flat offsets boff; one block of nw for the dense
// filter), P = p0 I
int kf_create(KfDev &d, const std::vector<int> &bsz, const std::vector<int> &boff, double p0,
              double lam_ini, double lam0, double q, double gate);
// nobs updates of kf_update_grad in order: rows[k*ld + i] = dy/dw_i,
// xi[k] = target - prediction, scale[k] (null = 1); w[nw] updated in place.
// Stops at the first nonpositive denominator (KfState::status = kbase + k + 1).
// A sequence split into calls passes kbase = the index of its first
// observation (the status is reset when it is 0); first forms the products
// with row 0 (false when the previous call's last pass formed them); a call
// with has_next also stages row nobs (the next call's first), whose products
// its last tile pass forms.
int kf_run(KfDev &d, int nobs, const double *rows, size_t ld, const double *xi,
           const double *scale, double *w, cudaStream_t s, int kbase, bool has_next,
           bool first);
// xi[0] = sign * R of one point's output derivatives under a Jacobian-row
// rule (sign -1: the innovation of a residual, whose target is zero)
int kf_resid_xi(const DevRule &r, const double *out, int nout, double *xi, cudaStream_t s,
                double sign = -1.0);
// residual ir of a system rule at one point, xi[0] = sign * R_ir, and its
// seed dR_ir/dT into seed[nout][na]; src[nres] may be null
int kf_sys_seed(const DevRule &r, const double *out, int na, int nout, const double *src,
                int ir, double *seed, double *xi, double sign, cudaStream_t s);
// one relinearisation of the iterated EKF (kf_iekf_iter): row = dR/dw at
// the current weights w, resid[0] = R, scale[0] = 1/sqrt(rnoise); w <- w- +
// kv xi with the prior d.wprior; the covariance and lambda change only when
// final
// kbase numbers the observation in the status; reset clears the status
// first (a pass over points keeps it, so that a failure stops the rest)
int kf_iekf(KfDev &d, const double *row, const double *resid, const double *scale, double *w,
            bool final, cudaStream_t s, int kbase = 0, bool reset = true);
int kf_state(const KfDev &d, KfState *out, cudaStream_t s);
// the update path: -1 by size (default), 0 two launches per update, 1 one
// cooperative launch per call
int kf_force_path(int path);
// covariance to the host: dense [nw][nw], or the blocks [bsz][bsz] one after another
int kf_read_cov(const KfDev &d, const std::vector<int> &bsz, const std::vector<int> &boff,
                bool dense, double *out, cudaStream_t s);

// SMs a persistent launch may fill: the device's count, or a cap that the
// committee step sets on its host thread while it issues one member's
// launches, so that concurrent members share the device instead of each
// sizing its grid for all of it.
int grid_sms();
void set_grid_cap(int sms);

// count of kernel launches issued by this library (process-wide)
void note_launch();
long long launch_count();

// Per-kernel device timing: while enabled, every launch is bracketed by a
// pair of CUDA events recorded on its own stream; profile_read sums the
// elapsed times by kernel name.
void profile_enable(bool on);
int prof_begin(const char *name, cudaStream_t st);
void prof_end(int idx, cudaStream_t st);
std::string profile_read();

#define LAUNCH(name, st, ...)                                 \
  do {                                                        \
    int pi_ = ::dnnf90::prof_begin(name, st);                 \
    __VA_ARGS__;                                              \
    ::dnnf90::prof_end(pi_, st);                              \
    ::dnnf90::note_launch();                                  \
  } while (0)

// device selection and error text
int device_ready();
const char *last_error();
void set_error(const std::string &msg);

}  // namespace dnnf90
