// kernels.cuh - device functions shared by the kernels of the engine.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace dnnf90 {

constexpr int KMAX = 15;     // largest derivative order (table_args_ok)
constexpr int D0MAX = 16;    // largest input width on the device path

// J_0(x) .. J_n(x) (n <= KMAX + 2): for |x| < 1e-5 two terms of the power
// series, otherwise Miller's backward recurrence
//   J_{k-1}(x) = (2k / x) J_k(x) - J_{k+1}(x)
// from an even start index well above max(n, |x|), normalised by
// J_0 + 2 sum_{k >= 1} J_{2k} = 1 (Abramowitz & Stegun 9.1.27, 9.1.46, 9.12),
// rescaled whenever the unnormalised values pass 1e200; J_n(-x) =
// (-1)^n J_n(x).  Agrees with scipy's jv to 1e-15 on [-40, 40].
static __device__ __noinline__ void besj_all(int n, double x, double *bj) {
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
    j = jm1;  // J_{k-1}
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

// J0 (shift 0) or J1 (shift 1) and its derivatives to order nq: the
// binomial combinations of besj0_derivs / besj1_derivs
// (lib/multi_index_bell_module.f90:757-826),
//   J_s^(q) = ((-1)^q / 2^q) sum_k (-1)^k C(q,k) J_{s+q-2k},  J_{-n} = (-1)^n J_n.
// Not inlined, so that its locals stay out of the kernels that never use it.
static __device__ __noinline__ void besj_derivs(int shift, double a, int nq, double *d) {
  double bj[KMAX + 4];
  besj_all(nq + shift, a, bj);
  for (int q = 0; q <= nq; ++q) {
    double term = 0.0, c = 1.0;
    for (int kk = 0; kk <= q; ++kk) {
      const int m = shift + q - 2 * kk;
      const double sk = (kk & 1) ? -1.0 : 1.0;
      if (m >= 0) term = term + sk * c * bj[m];
      else term = term + sk * c * ((-m) & 1 ? -1.0 : 1.0) * bj[-m];
      c = c * (double)(q - kk) / (double)(kk + 1);
    }
    d[q] = (q & 1 ? -1.0 : 1.0) * term / ldexp(1.0, q);
  }
}

// sigma^(q)(a), q = 0..k+1, in FP64.  tanh: Horner on the integer
// polynomials P_q(t), t = tanh(a) (tanh_derivs_ts,
// lib/multi_index_bell_module.f90:852-867); sin: sin(a + q pi/2)
// (sin_derivs, :745-755); erf: Hermite functions (erf_derivs, :831-850);
// J0 / J1: the binomial combinations of J_n (besj0_derivs, besj1_derivs,
// :757-826).  The CUDA tanh/sin/exp/erf are called, never re-derived.
__device__ __forceinline__ void sigma_derivs(int iact, const double *__restrict__ tpc,
                                             int k, double a, double *d) {
  const int nq = k + 1;
  if (iact == 3 || iact == 4) {
    // the callee fills its own array, so d itself is never passed by
    // address and stays in registers wherever k is a compile-time constant
    double tmp[KMAX + 2];
    besj_derivs(iact - 3, a, nq, tmp);
    for (int q = 0; q <= nq; ++q) d[q] = tmp[q];
    return;
  }
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
