// ngd.cu - the damped Gauss-Newton step of app/optimizer_module.f90:221-469
// (primal route, ABS damping) on the device:
//   G = J^T J / nb + mu I,  u = G^{-1} (b / nb),
// with the metric formed from the residual-Jacobian rows J[nrow][nw] and
// solved by an FP64 Cholesky factorization (the reference eliminates with
// partial pivoting, gauss_solve :472-522; G is symmetric positive definite
// once damped, so the factorization is the natural device form).
//
// The metric build is a GEMM: in the split path J is carried as three bf16
// terms and the six cross products are accumulated in FP32 per 64-row slab
// (tensor cores), the slabs summed in FP64; in the plain path it is an FP64
// CUDA-core GEMM.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "engine.hpp"
#include "gemm_tc.hpp"

namespace dnnf90 {

#define CKN(call)                                                      \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess) {                                           \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));   \
      return e_ == cudaErrorMemoryAllocation ? RC_NOMEM : RC_DEVICE;   \
    }                                                                  \
  } while (0)

constexpr int NB = 64;

// G[i][j] += sum_{r in slab} J[r][i] J[r][j] for the lower tiles (j <= i),
// FP64 CUDA-core tiles of 64 x 64, split over rows with atomics.
__global__ void __launch_bounds__(256) k_syrk_f64(const double *J, int nrow, int nw,
                                                  double *G, int rchunk) {
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj > ti) return;
  __shared__ double As[16][65], Bs[16][65];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = ti * 64, j0 = tj * 64;
  double acc[4][4] = {};
  const int r0 = blockIdx.z * rchunk, r1 = min(nrow, r0 + rchunk);
  for (int k0 = r0; k0 < r1; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int kk = e / 64, c = e - kk * 64;
      int r = k0 + kk;
      As[kk][c] = (r < r1 && i0 + c < nw) ? J[(size_t)r * nw + i0 + c] : 0.0;
      Bs[kk][c] = (r < r1 && j0 + c < nw) ? J[(size_t)r * nw + j0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = As[kk][ty + 16 * u]; b[u] = Bs[kk][tx + 16 * u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
  for (int u = 0; u < 4; ++u) {
    int i = i0 + ty + 16 * u;
    if (i >= nw) continue;
    for (int v = 0; v < 4; ++v) {
      int j = j0 + tx + 16 * v;
      if (j < nw && j <= i) atomicAdd(G + (size_t)i * nw + j, acc[u][v]);
    }
  }
}

// G = G / nb + mu I on the lower triangle; rhs = b / nb
__global__ void k_scale_damp(double *G, int nw, double inv_nb, double mu,
                             const double *b, double *rhs) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)nw * nw;
       e += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(e / nw), j = (int)(e - (size_t)i * nw);
    if (j > i) continue;
    double v = G[e] * inv_nb;
    if (i == j) v += mu;
    G[e] = v;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x)
    rhs[i] = b[i] * inv_nb;
}

// unblocked Cholesky of the diagonal block [k0, k0+nb) in shared memory;
// info[0] receives the first non-positive pivot (1-based) if any
__global__ void k_potrf_diag(double *G, int nw, int k0, int nb, int *info) {
  __shared__ double A[NB][NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e / nb, j = e - i * nb;
    A[i][j] = j <= i ? G[(size_t)(k0 + i) * nw + k0 + j] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0) {
      double d = A[k][k];
      if (!(d > 0.0)) {
        if (info[0] == 0) info[0] = k0 + k + 1;
        d = 1.0;
      }
      A[k][k] = sqrt(d);
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < nb; i += blockDim.x) A[i][k] /= A[k][k];
    __syncthreads();
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
      int i = e / nb, j = e - i * nb;
      if (i > k && j > k && j <= i) A[i][j] -= A[i][k] * A[j][k];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e / nb, j = e - i * nb;
    if (j <= i) G[(size_t)(k0 + i) * nw + k0 + j] = A[i][j];
  }
}

// L21 = A21 L11^{-T}: every row below the block solved independently
__global__ void k_trsm_panel(double *G, int nw, int k0, int nb) {
  __shared__ double L[NB][NB + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    int i = e / nb, j = e - i * nb;
    L[i][j] = j <= i ? G[(size_t)(k0 + i) * nw + k0 + j] : 0.0;
  }
  __syncthreads();
  for (int r = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x; r < nw;
       r += gridDim.x * blockDim.x) {
    double *row = G + (size_t)r * nw + k0;
    double x[NB];
    for (int j = 0; j < nb; ++j) {
      double s = row[j];
      for (int t = 0; t < j; ++t) s -= x[t] * L[j][t];
      x[j] = s / L[j][j];
    }
    for (int j = 0; j < nb; ++j) row[j] = x[j];
  }
}

// trailing update A22 -= L21 L21^T on the lower tiles
__global__ void __launch_bounds__(256) k_syrk_trail(double *G, int nw, int k0, int nb) {
  const int base = k0 + nb;
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj > ti) return;
  const int i0 = base + ti * 64, j0 = base + tj * 64;
  __shared__ double As[16][65], Bs[16][65];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int k = 0; k < nb; k += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      int c = e / 16, kk = e - c * 16;
      int kx = k0 + k + kk;
      As[kk][c] = (i0 + c < nw && k + kk < nb) ? G[(size_t)(i0 + c) * nw + kx] : 0.0;
      Bs[kk][c] = (j0 + c < nw && k + kk < nb) ? G[(size_t)(j0 + c) * nw + kx] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = As[kk][ty + 16 * u]; b[u] = Bs[kk][tx + 16 * u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
  for (int u = 0; u < 4; ++u) {
    int i = i0 + ty + 16 * u;
    if (i >= nw) continue;
    for (int v = 0; v < 4; ++v) {
      int j = j0 + tx + 16 * v;
      if (j < nw && j <= i) G[(size_t)i * nw + j] -= acc[u][v];
    }
  }
}

// L y = r then L^T u = y, one block; rows are visited in order with a
// block-wide dot product per row
__global__ void __launch_bounds__(1024) k_chol_solve(const double *G, int nw, double *x) {
  __shared__ double red[32];
  __shared__ double val;
  for (int i = 0; i < nw; ++i) {  // forward
    double s = 0.0;
    for (int j = threadIdx.x; j < i; j += blockDim.x) s += G[(size_t)i * nw + j] * x[j];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) {
        val = (x[i] - v) / G[(size_t)i * nw + i];
        x[i] = val;
      }
    }
    __syncthreads();
  }
  for (int i = nw - 1; i >= 0; --i) {  // backward with L^T: column i of L
    double s = 0.0;
    for (int j = i + 1 + threadIdx.x; j < nw; j += blockDim.x) s += G[(size_t)j * nw + i] * x[j];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) x[i] = (x[i] - v) / G[(size_t)i * nw + i];
    }
    __syncthreads();
  }
}

// FP32 copy of the rows with a padded leading dimension (zero past nw), the
// operand of the tensor-core metric
__global__ void k_rows_f32(const double *rows, int nrow, int nw, float *J, int ldj) {
  const long tot = (long)nrow * ldj;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (long)gridDim.x * blockDim.x) {
    const long r = e / ldj;
    const int c = (int)(e - r * ldj);
    J[e] = c < nw ? (float)rows[(size_t)r * nw + c] : 0.f;
  }
}

// G[nc][nc] (lower triangle, zeroed here) = A^T A for A[nr][nc]: on the
// tensor cores in the split precision (split-BF16 products of an FP32 copy,
// FP32 accumulation per 512 rows, FP64 across them), else FP64 tiles
static int gram(const double *A, int nr, int nc, double *G, int prec, cudaStream_t st) {
  CKN(cudaMemsetAsync(G, 0, sizeof(double) * (size_t)nc * nc, st));
  int rc = RC_UNSUPPORTED;
  if (prec == PREC_SPLIT && gemm_tc_available()) {
    const int ldj = (nc + 3) / 4 * 4;
    float *J = nullptr;
    if (cudaMalloc(&J, sizeof(float) * (size_t)nr * ldj) == cudaSuccess) {
      LAUNCH("k_rows_f32", st, k_rows_f32<<<1024, 256, 0, st>>>(A, nr, nc, J, ldj));
      rc = gemm_tc_syrk(J, nr, nc, ldj, G, st);
      cudaFree(J);
    }
  }
  if (rc != RC_UNSUPPORTED) return rc;
  const int tiles = (nc + 63) / 64;
  int rchunk = std::max(64, (nr + 7) / 8);
  rchunk = (rchunk + 15) / 16 * 16;
  dim3 grid(tiles, tiles, (nr + rchunk - 1) / rchunk);
  LAUNCH("k_syrk_f64", st, k_syrk_f64<<<grid, 256, 0, st>>>(A, nr, nc, G, rchunk));
  CKN(cudaGetLastError());
  return RC_OK;
}

// Cholesky factorization of the damped G[n][n] (lower triangle) and the
// solve G x = x; -1 with the first non-positive pivot in the error text
static int chol_solve(double *G, int n, double *x, int *info, cudaStream_t st) {
  CKN(cudaMemsetAsync(info, 0, sizeof(int), st));
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int nbk = std::min(NB, n - k0);
    LAUNCH("k_potrf_diag", st, k_potrf_diag<<<1, 256, 0, st>>>(G, n, k0, nbk, info));
    CKN(cudaGetLastError());
    if (k0 + nbk < n) {
      const int rem = n - k0 - nbk;
      LAUNCH("k_trsm_panel", st, k_trsm_panel<<<std::max(1, std::min(256, (rem + 127) / 128)), 128, 0, st>>>(G, n, k0, nbk));
      CKN(cudaGetLastError());
      const int tt = (rem + 63) / 64;
      LAUNCH("k_syrk_trail", st, k_syrk_trail<<<dim3(tt, tt), 256, 0, st>>>(G, n, k0, nbk));
      CKN(cudaGetLastError());
    }
  }
  LAUNCH("k_chol_solve", st, k_chol_solve<<<1, 1024, 0, st>>>(G, n, x));
  CKN(cudaGetLastError());
  int hinfo = 0;
  CKN(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKN(cudaStreamSynchronize(st));
  if (hinfo) {
    set_error("the damped metric is not positive definite at column " + std::to_string(hinfo));
    return RC_BAD_ARG;
  }
  return RC_OK;
}

int ngd_device(const double *rows, int nrow, int nw, const double *b, int nb,
               double mu, double *u, int prec, cudaStream_t st) {
  double *G = nullptr;
  int *info = nullptr;
  CKN(cudaMalloc(&G, sizeof(double) * (size_t)nw * nw));
  if (cudaMalloc(&info, sizeof(int)) != cudaSuccess) {
    cudaFree(G);
    set_error("cudaMalloc failed for the metric pivot flag");
    return RC_NOMEM;
  }
  int rc = gram(rows, nrow, nw, G, prec, st);
  if (!rc) {
    LAUNCH("k_scale_damp", st, k_scale_damp<<<1024, 256, 0, st>>>(G, nw, 1.0 / (double)nb, mu, b, u));
    rc = cudaGetLastError() == cudaSuccess ? RC_OK : RC_DEVICE;
  }
  if (!rc) rc = chol_solve(G, nw, u, info, st);
  cudaFree(G);
  cudaFree(info);
  return rc;
}

// The two halves of the primal step, for a step whose rows are spread over
// ranks: each rank forms its own J^T J, the caller sums the metrics (and
// the gradients) over the ranks, and every rank solves the summed system,
// as app/optimizer_module.f90:310-321 does with sum_over_ranks.
int ngd_gram_device(const double *rows, int nrow, int nw, double *G, int prec, cudaStream_t st) {
  return gram(rows, nrow, nw, G, prec, st);
}

int ngd_solve_device(double *G, int nw, const double *b, int nb, double mu, double *u,
                     cudaStream_t st) {
  int *info = nullptr;
  CKN(cudaMalloc(&info, sizeof(int)));
  LAUNCH("k_scale_damp", st, k_scale_damp<<<1024, 256, 0, st>>>(G, nw, 1.0 / (double)nb, mu, b, u));
  int rc = cudaGetLastError() == cudaSuccess ? RC_OK : RC_DEVICE;
  if (!rc) rc = chol_solve(G, nw, u, info, st);
  cudaFree(info);
  return rc;
}

// ------------------------------------------------- dual (Gram-space) route
// The dual route of app/optimizer_module.f90:408-446: with G = J^T J / nb
// and the damping mu, the push-through identity gives
//   (G + mu I)^{-1} b' = (1 / mu) (b' - J^T K^{-1} (J b') / nb),
//   K = mu I + J J^T / nb  (nrow x nrow),  b' = b / nb,
// so the nw x nw metric is never formed: an nrow x nrow solve and two
// passes over the rows.  The step is the primal one to roundoff.

// T[nc][nr] = A^T for A[nr][nc], 32 x 32 tiles through shared memory
__global__ void k_transpose(const double *A, int nr, int nc, double *T) {
  __shared__ double tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < nr && c < nc) ? A[(size_t)r * nc + c] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < nc && r < nr) T[(size_t)c * nr + r] = tile[threadIdx.x][i];
  }
}

// K = K / nb + mu I on the lower triangle
__global__ void k_damp(double *K, int n, double inv_nb, double mu) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e - (size_t)i * n);
    if (j > i) continue;
    K[e] = K[e] * inv_nb + (i == j ? mu : 0.0);
  }
}

// y[r] = alpha sum_i J[r][i] x[i], one warp per row
__global__ void k_rows_dot(const double *J, int nrow, int nw, const double *x, double alpha,
                           double *y) {
  const int lane = threadIdx.x & 31;
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrow;
       r += gridDim.x * (blockDim.x >> 5)) {
    double s = 0.0;
    for (int i = lane; i < nw; i += 32) s += J[(size_t)r * nw + i] * x[i];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[r] = alpha * s;
  }
}

// u[i] = (b[i] / nb - (1 / nb) sum_r J[r][i] y[r]) / mu
__global__ void k_dual_step(const double *J, int nrow, int nw, const double *b, const double *y,
                            double inv_nb, double inv_mu, double *u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < nrow; ++r) s += J[(size_t)r * nw + i] * y[r];
    u[i] = (b[i] * inv_nb - s * inv_nb) * inv_mu;
  }
}

int ngd_device_dual(const double *rows, int nrow, int nw, const double *b, int nb, double mu,
                    double *u, int prec, cudaStream_t st) {
  if (!(mu > 0.0)) {
    set_error("the dual natural-gradient step needs a positive damping mu");
    return RC_BAD_ARG;
  }
  double *K = nullptr, *JT = nullptr, *y = nullptr;
  int *info = nullptr;
  auto cleanup = [&]() {
    if (K) cudaFree(K);
    if (JT) cudaFree(JT);
    if (y) cudaFree(y);
    if (info) cudaFree(info);
  };
  if (cudaMalloc(&K, sizeof(double) * (size_t)nrow * nrow) != cudaSuccess ||
      cudaMalloc(&JT, sizeof(double) * (size_t)nrow * nw) != cudaSuccess ||
      cudaMalloc(&y, sizeof(double) * (size_t)nrow) != cudaSuccess ||
      cudaMalloc(&info, sizeof(int)) != cudaSuccess) {
    cleanup();
    set_error("cudaMalloc failed for the dual natural-gradient step");
    return RC_NOMEM;
  }
  // K = J J^T: the Gram product of the transposed rows, always in FP64.
  // The step ends with (b' - J^T y / nb) / mu, a cancellation divided by a
  // small damping, which magnifies the rounding of split-BF16 products in K
  // far past what the primal solve sees (measured backward error 6e-3
  // against 1e-7); K is only nrow x nrow, so FP64 costs little here.
  (void)prec;
  LAUNCH("k_transpose", st, k_transpose<<<dim3((nw + 31) / 32, (nrow + 31) / 32), dim3(32, 8), 0, st>>>(rows, nrow, nw, JT));
  int rc = cudaGetLastError() == cudaSuccess ? RC_OK : RC_DEVICE;
  if (!rc) rc = gram(JT, nw, nrow, K, PREC_F64, st);
  if (!rc) {
    const double inv_nb = 1.0 / (double)nb;
    LAUNCH("k_damp", st, k_damp<<<1024, 256, 0, st>>>(K, nrow, inv_nb, mu));
    LAUNCH("k_rows_dot", st, k_rows_dot<<<std::max(1, std::min(4096, (nrow + 7) / 8)), 256, 0, st>>>(rows, nrow, nw, b, inv_nb, y));
    rc = cudaGetLastError() == cudaSuccess ? RC_OK : RC_DEVICE;
    if (!rc) rc = chol_solve(K, nrow, y, info, st);
    if (!rc) {
      LAUNCH("k_dual_step", st, k_dual_step<<<std::max(1, (nw + 255) / 256), 256, 0, st>>>(rows, nrow, nw, b, y, inv_nb, 1.0 / mu, u));
      rc = cudaGetLastError() == cudaSuccess ? RC_OK : RC_DEVICE;
      if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = RC_DEVICE;
    }
  }
  if (rc == RC_DEVICE) set_error("the dual natural-gradient step failed on the device");
  cleanup();
  return rc;
}

// ------------------------------------------------- no-allocation variant
// dnnf90_ngd_step_noalloc runs the plain FP64 route above on caller
// buffers without allocating device memory: the damped metric and the
// pivot flag live in this fixed area instead.  The array belongs to every
// GPU that loads the library, for the life of the process (8 MiB).
constexpr int NGD_NOALLOC_MAXW = 1024;
static __device__ __align__(256) double
    g_ngd_scratch[(size_t)NGD_NOALLOC_MAXW * NGD_NOALLOC_MAXW + 32];

int ngd_noalloc_maxw() { return NGD_NOALLOC_MAXW; }

// Device address of the scratch on the current device, looked up once per
// device (host code cannot use the array's name as a device address) and
// kept for the life of the process: it does not survive cudaDeviceReset.
// With lazy module loading (the CUDA 12 default) the array is backed when
// this file's module first loads on a device, which the lookup itself
// triggers, so that first call may take the 8 MiB from the device.
static double *ngd_scratch_ptr() {
  static std::mutex mu;
  static double *ptr[256] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!ptr[dev]) {
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_ngd_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetSymbolAddress(ngd scratch): ") + cudaGetErrorString(e));
      return nullptr;
    }
    ptr[dev] = p;
  }
  return ptr[dev];
}

int ngd_device_noalloc(const double *rows, int nrow, int nw, const double *b, int nb,
                       double mu, double *u, cudaStream_t st) {
  if (nw > NGD_NOALLOC_MAXW) {
    set_error("dnnf90_ngd_step_noalloc: nweights " + std::to_string(nw) +
              " is above the fixed scratch limit of " + std::to_string(NGD_NOALLOC_MAXW));
    return RC_BAD_ARG;
  }
  if (!(mu > 0.0)) {
    set_error("dnnf90_ngd_step_noalloc: the damping mu must be positive");
    return RC_BAD_ARG;
  }
  // the call reads the pivot flag back into host memory and waits for its
  // stream, neither of which a stream being captured allows
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    set_error("dnnf90_ngd_step_noalloc cannot be captured into a CUDA graph (it waits for "
              "its stream and reads a status back)");
    return RC_UNSUPPORTED;
  }
  double *G = ngd_scratch_ptr();
  if (!G) return RC_DEVICE;
  int *info = (int *)(G + (size_t)NGD_NOALLOC_MAXW * NGD_NOALLOC_MAXW);
  // the scratch keeps the previous call's contents: clear what accumulates
  CKN(cudaMemsetAsync(G, 0, sizeof(double) * (size_t)nw * nw, st));
  CKN(cudaMemsetAsync(info, 0, sizeof(int), st));
  const int tiles = (nw + 63) / 64;
  {
    int rchunk = std::max(64, (nrow + 7) / 8);
    rchunk = (rchunk + 15) / 16 * 16;
    dim3 grid(tiles, tiles, (nrow + rchunk - 1) / rchunk);
    LAUNCH("k_syrk_f64", st, k_syrk_f64<<<grid, 256, 0, st>>>(rows, nrow, nw, G, rchunk));
    CKN(cudaGetLastError());
  }
  LAUNCH("k_scale_damp", st, k_scale_damp<<<1024, 256, 0, st>>>(G, nw, 1.0 / (double)nb, mu, b, u));
  CKN(cudaGetLastError());
  for (int k0 = 0; k0 < nw; k0 += NB) {
    const int nbk = std::min(NB, nw - k0);
    LAUNCH("k_potrf_diag", st, k_potrf_diag<<<1, 256, 0, st>>>(G, nw, k0, nbk, info));
    CKN(cudaGetLastError());
    if (k0 + nbk < nw) {
      const int rem = nw - k0 - nbk;
      LAUNCH("k_trsm_panel", st, k_trsm_panel<<<std::max(1, std::min(256, (rem + 127) / 128)), 128, 0, st>>>(G, nw, k0, nbk));
      CKN(cudaGetLastError());
      const int tt = (rem + 63) / 64;
      LAUNCH("k_syrk_trail", st, k_syrk_trail<<<dim3(tt, tt), 256, 0, st>>>(G, nw, k0, nbk));
      CKN(cudaGetLastError());
    }
  }
  LAUNCH("k_chol_solve", st, k_chol_solve<<<1, 1024, 0, st>>>(G, nw, u));
  CKN(cudaGetLastError());
  int hinfo = 0;
  CKN(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKN(cudaStreamSynchronize(st));
  if (hinfo) {
    set_error("the damped metric is not positive definite at column " + std::to_string(hinfo));
    return RC_BAD_ARG;
  }
  return RC_OK;
}

}  // namespace dnnf90
