// gemm_tc.hpp - split-BF16 layer GEMMs on the fifth-generation tensor cores
// (tcgen05.mma, operands staged by TMA, accumulators in tensor memory).
//
// Each FP32 operand x is carried as three bf16 terms x = x1 + x2 + x3
// (x1 = bf16(x), x2 = bf16(x - x1), x3 = bf16(x - x1 - x2)), and a product
// keeps the six cross terms of order <= 2 (a1b1, a1b2, a2b1, a1b3, a2b2,
// a3b1), accumulated in FP32: relative error near 2^-24 per product, the
// FP32 level.  The three GEMMs of a hidden layer:
//   fwd: S  = T_{l-1} W_l^T (+ bias on the alpha = 0 rows)
//   dt : Tb = Sb W_l
//   dw : dW += Sb^T T_{l-1}    (FP64 reduction of the per-block partials)
#pragma once
#include <cuda_runtime.h>

namespace dnnf90 {

struct DevNet;

bool gemm_tc_available();
void gemm_tc_release_weights(DevNet *net);
// Pre-splits and pre-swizzles the weight operands of every hidden layer
// from the host weights hw (flat layer layout).
int gemm_tc_prepare(DevNet *net, const double *hw, cudaStream_t st);
// Reads the wait time-out flag of the network's tensor-core GEMMs
// (synchronises st); RC_DEVICE if a wait ran out.
int gemm_tc_flag(const DevNet *net, cudaStream_t st);

int gemm_tc_fwd(const DevNet *net, int l, int M, int n, int m, int na,
                const void *A, void *C, cudaStream_t st);
int gemm_tc_dt(const DevNet *net, int l, int M, int n, int m, const void *Sb,
               void *Tb, cudaStream_t st);
int gemm_tc_dw(const DevNet *net, int l, int M, int n, int m, const void *Sb,
               const void *Tm, double *G, cudaStream_t st);

// G[i][j] += sum_r J[r][i] J[r][j] on the lower triangle (FP64 G), J in FP64
// rows carried as three bf16 terms on the tensor cores
// G[i][j] += sum_r J[r][i] J[r][j] from an FP32 copy J[nrow][ldj] (ldj a
// multiple of 4, columns nw..ldj-1 zero), G [nw][nw] FP64; synchronises st
int gemm_tc_syrk(const float *J, int nrow, int nw, int ldj, double *G, cudaStream_t st);

int weights_to_f32(const double *w, float *w32, size_t n, cudaStream_t st);

}  // namespace dnnf90
