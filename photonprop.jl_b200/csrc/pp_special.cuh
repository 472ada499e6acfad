// FP64 digamma and trigamma for the device: upward recurrence to x >= 6,
// then the asymptotic series
//   psi(x)  = ln x - 1/(2x) - sum_k B_2k / (2k x^2k)
//   psi'(x) = 1/x + 1/(2x^2) + sum_k B_2k / x^(2k+1)
// (Bernoulli numbers B_2..B_10); relative error below 1e-14 for x > 0.
#pragma once

namespace ppsf {

__device__ __forceinline__ double digamma_d(double x) {
  double r = 0.0;
  while (x < 6.0) {
    r -= 1.0 / x;
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  return r + log(x) - 0.5 / x - f * (1.0 / 12 - f * (1.0 / 120 - f * (1.0 / 252 - f * (1.0 / 240 - f / 132))));
}

__device__ __forceinline__ double trigamma_d(double x) {
  double r = 0.0;
  while (x < 6.0) {
    r += 1.0 / (x * x);
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  return r + 1.0 / x + 0.5 * f + (1.0 / x) * f * (1.0 / 6 - f * (1.0 / 30 - f * (1.0 / 42 - f / 30)));
}

}  // namespace ppsf
