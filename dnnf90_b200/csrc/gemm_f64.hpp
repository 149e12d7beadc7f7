// gemm_f64.hpp - the plain FP64 path's layer GEMMs on the tensor cores (DMMA).
#pragma once
#include <cuda_runtime.h>

namespace dnnf90 {

enum : int { MODE_F64_FWD = 0, MODE_F64_DT = 1, MODE_F64_DW = 2 };

// FWD: C[M][N] = A[M][K] B[N][1..K]^T + B[N][0] on rows m % na == 0
// DT:  C[M][N] = A[M][K] B[K][1..N]
// DW:  G[m][1 + n] += sum_k A[k][m] B[k][n]   (M = output rows, K = rows reduced)
// RC_UNSUPPORTED when a leading dimension or base address does not allow
// the kernel's 16-byte pieces (odd lda, unaligned base).
// pack (FWD, DT; may be null): room for N x K doubles into which the weight
// operand is first copied without its bias column, so that it loads in
// 16-byte pieces; it must belong to this call alone while the call runs.
int gemm_f64(int mode, int M, int N, int K, int na, const double *A, int lda, const double *B,
             int ldb, double *C, int ldc, double *G, int gld, cudaStream_t st,
             double *pack = nullptr);

}  // namespace dnnf90
