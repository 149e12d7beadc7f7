// bell.hpp - warp-cooperative Bell kernels (see bell.cu, bell_plan.hpp).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "bell_plan.hpp"

namespace dnnf90 {

struct DevTables;

constexpr int BELL_WORKERS = 32;  // warps per block sharing one point's state
constexpr int BELL_UNROLL = 4;    // table records fetched ahead per step
constexpr int ADJ_WORKERS = 32;   // warps per block of the adjoint
constexpr int ADJ_UNROLL = 2;     // pairs fetched ahead: 2 * ADJ_UNROLL

// device copy of the register-tiled kernels' plan (tile_plan.hpp) and the
// shared-memory layouts of the two kernels (byte offsets)
struct TileDev {
  bool ok = false;
  int td = 0, k = 0, na = 0, nbuf0 = 0, nbuf1 = 0;
  int nfunit = 0, nfrec = 0, naunit = 0, narec = 0, nafin = 0, nscratch = 0;
  int *flist = nullptr, *funit = nullptr, *alist = nullptr, *aunit = nullptr;
  int *aflist = nullptr, *afin = nullptr, *perm = nullptr, *rowslot = nullptr;
  uint32_t *frec = nullptr, *arec = nullptr;
  float *fact = nullptr, *ifact = nullptr;
  int f_o_d0 = 0, f_o_d1 = 0, f_o_sig = 0, f_o_list = 0, f_o_unit = 0, f_o_rec = 0;
  int f_o_perm = 0, f_o_rowslot = 0, f_o_fact = 0, f_o_ifact = 0, f_smem = 0;
  int a_o_scr = 0, a_o_list = 0, a_o_flist = 0, a_o_unit = 0, a_o_fin = 0, a_o_rec = 0;
  int a_o_perm = 0, a_o_rowslot = 0, a_o_fact = 0, a_o_ifact = 0, a_smem = 0;
  void release();
};

struct DevBellPlan {
  bool ready = false;
  uint64_t id = 0;              // distinct per upload (autotuner key)
  int workers = 0, k = 0, na = 0, nslot = 0;
  int *fw_list = nullptr, *fw_arec = nullptr, *fw_grec = nullptr;
  double *fw_gc64 = nullptr;
  float *fw_gc32 = nullptr;
  int *aj_list = nullptr, *aj_orec = nullptr, *aj_pair = nullptr;
  double *aj_c64 = nullptr;
  float *aj_c32 = nullptr;
  // v3
  bool f3_ok = false;
  int nrows = 0, dt_off = 0;
  int *f3_list = nullptr, *f3_arec = nullptr, *f3_grec = nullptr;
  double *f3_gc64 = nullptr;
  float *f3_gc32 = nullptr;
  int *a3_orec = nullptr, *a3_pair = nullptr;
  uint32_t *f4_grec = nullptr, *a4_pair = nullptr;
  int nuv = 0;
  // v5
  bool f5_ok = false;
  int nrows5 = 0, dt_off5 = 0, zuv5 = 0;
  int *f5_list = nullptr, *f5_arec = nullptr, *f5_cpdst = nullptr;
  uint32_t *f5_rec = nullptr, *a5_pair = nullptr;
  uint32_t *f6_rec = nullptr;   // forward records as row indices
  int nrec32 = 0, norec = 0, npair5 = 0;
  // v7 adjoint (grouped correlation): [0] FP32 plan, [1] FP64 plan
  struct A7Dev {
    int *list = nullptr, *unit = nullptr, *out = nullptr, *fin = nullptr;
    uint32_t *glist = nullptr, *rec = nullptr;
    int nunit = 0, nout = 0, nglist = 0, nrec = 0, nfin = 0, nscratch = 0;
    bool ok = false;
  } a7[2];
  // v8 forward (F8Plan)
  struct F8Dev {
    int *list = nullptr, *hdr = nullptr, *cpdst = nullptr;
    uint32_t *rec = nullptr;
    int nrec = 0, sbase1 = 0, bbase = 0, uvbase = 0, dtbase = 0, recbase = 0, zuv = 0;
    int smem = 0;
    bool ok = false;
  } f8;
  // v9 tanh series forward (F9Plan)
  struct F9Dev {
    int *list = nullptr, *hdr = nullptr;
    uint32_t *rec = nullptr;
    double *sdeg64 = nullptr;
    float *sdeg32 = nullptr;
    int pbase = 0, qbase = 0, smem = 0;
    bool ok = false;
  } f9;
  TileDev tile;            // register-tiled kernels (dense sets, FP32)
  double *sc64 = nullptr;  // [3][na]: a!, 1/a!, 1/a! (Tb, h, Sb scales)
  float *sc32 = nullptr;
  void release();
};

int upload_bell_plan(const TableSet &t, DevBellPlan &d);

// the autotuner's choices: "kernel width precision variant ms..." lines
std::string tune_report();
// pin the variant of the Bell forward (which 0) or adjoint (which 1) kernels;
// variant -1 returns them to the autotuner.  which 2 switches the tanh
// series forward: 1 on wherever it applies, 0 or -1 off (the default: the
// Bell recurrence everywhere).
int tune_force(int which, int variant);

// RC_UNSUPPORTED when the set does not fit (K > 8 or the per-point state
// exceeds shared memory): the caller then uses the generic kernels.
int bell_fwd2(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *S,
              void *T, void *h, bool train, int prec, cudaStream_t st);
int bell_adj2(const DevBellPlan &bp, const DevTables &t, int n, int npts, const void *Tb,
              const void *h, void *Sb, double *gbias, int gstride, int prec,
              cudaStream_t st);
// register-tiled Bell forward and adjoint (bell_tile.cu): dense sets with
// K <= 7, FP32 planes, n a multiple of 4; RC_UNSUPPORTED otherwise
int upload_tile_plan(const TableSet &t, TileDev &d);
bool tile_fwd_applies(const TileDev &d, int n);
bool tile_adj_applies(const TileDev &d, int n);
int bell_fwd_tile(const TileDev &d, const DevTables &t, int n, int npts, const void *S, void *T,
                  void *h, bool train, cudaStream_t st);
int bell_adj_tile(const TileDev &d, int n, int npts, const void *Tb, const void *h, void *Sb,
                  double *gbias, int gstride, cudaStream_t st);
// The first hidden layer is analytic: h^g = s^(|g|+1)(S^0) W^g.  With these
// inputs the adjoint forms h itself (graded slots) from the s^(q) the
// forward kept, and reads no h plane.
struct L2Analytic {
  const double *W;         // the layer's weights [n][d0 + 1]
  const void *sig;         // [P][k + 2][n]: s^(q)(S^0), kept by the forward
  const int *par;          // [na]: slot of g - e_i | i << 16 (the monomial recurrence)
  int k;
  const int *dstart;       // host [k + 2]: first slot of each degree
};
// whether the adjoint can form h itself for these sizes (its shared memory)
bool bell_adj_l2s_analytic(int d0, int na, int n, int prec);
// the first hidden layer's adjoint fused with dW_2, staged through shared
// memory (RC_UNSUPPORTED when an item's rows do not fit); an: h formed in
// the kernel (null: read from the h plane)
int bell_adj_l2s(int d0, int n, int na, int npts, const int *up, const void *Tb, const void *h,
                 const double *X, double *g, double *rows, size_t nw, size_t woff, int prec,
                 cudaStream_t st, const L2Analytic *an = nullptr);

}  // namespace dnnf90
