// kernels.cuh - device functions shared by the kernels of the engine.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace dnnf90 {

constexpr int KMAX = 15;     // largest derivative order (table_args_ok)
constexpr int D0MAX = 16;    // largest input width on the device path

// sigma^(q)(a), q = 0..k+1, in FP64.  tanh: Horner on the integer
// polynomials P_q(t), t = tanh(a) (tanh_derivs_ts,
// lib/multi_index_bell_module.f90:852-867); sin: sin(a + q pi/2)
// (sin_derivs, :745-755); erf: Hermite functions (erf_derivs, :831-850).
// The CUDA tanh/sin/exp/erf are called, never re-derived.
__device__ __forceinline__ void sigma_derivs(int iact, const double *__restrict__ tpc,
                                             int k, double a, double *d) {
  const int nq = k + 1;
  if (iact == 1) {
    double s, c;
    sincos(a, &s, &c);
    for (int q = 0; q <= nq; ++q) {
      int r = q & 3;
      d[q] = r == 0 ? s : r == 1 ? c : r == 2 ? -s : -c;
    }
    return;
  }
  if (iact == 2) {
    d[0] = erf(a);
    if (nq < 1) return;
    double psi_m1 = 0.0, psi = exp(-a * a);
    const double c2spi = 1.12837916709551257390;  // 2/sqrt(pi)
    for (int q = 1; q <= nq; ++q) {
      d[q] = c2spi * ((q - 1) & 1 ? -1.0 : 1.0) * psi;
      double nx = 2.0 * a * psi - 2.0 * (double)(q - 1) * psi_m1;
      psi_m1 = psi;
      psi = nx;
    }
    return;
  }
  const int ld = k + 3;
  const double t = tanh(a);
  for (int q = 0; q <= nq; ++q) {
    double v = __ldg(tpc + q * ld + q + 1);
    for (int i = q; i >= 0; --i) v = v * t + __ldg(tpc + q * ld + i);
    d[q] = v;
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace dnnf90
