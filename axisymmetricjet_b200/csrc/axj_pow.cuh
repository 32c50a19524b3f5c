// axj_pow.cuh -- mu = T**0.666 in FP64 (ModAssign.f90:20, Tvec**0.666D0) from tables,
// shared by the kernels and the host (the same operations in the same order, so the
// host evaluation reproduces the device's bits).
//
// Method (a table-driven reduction with a binomial series, after Tang's table-driven
// logarithm): T = 2^e m with m in [1, 2); j = the top 7 bits of m's fraction; c_j a 10-bit
// approximation of 1/F_j (F_j = 1 + (j + 1/2) / 128, the centre of m's interval);
// r = m c_j - 1 with one rounding (|r| < 0.006). Then
//     T^a = 2^(a e) * c_j^(-a) * (1 + r)^a,
// the first two factors from tables held as double-double (hi + lo), the third from the
// binomial series 1 + sum_{k=1..6} binom(a, k) r^k (the first term left out is below
// 3e-18). The product is formed in double-double and rounded once: within 1 ulp of
// the correctly rounded power. Exponents e outside [-16, 15] (T outside [2^-16, 2^16)),
// zero, negative, subnormal and non-finite T take exp2(a log2 T).
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#include "axj_common.cuh"

namespace axj {

constexpr int POW_NJ = 128;                        // mantissa intervals
constexpr int POW_E0 = -16, POW_NE = 32;           // exponents e = POW_E0 .. POW_E0 + POW_NE - 1
constexpr int POW_TAB = 3 * POW_NJ + 2 * POW_NE;   // {c_j, G_hi, G_lo} per j, then {E_hi, E_lo} per e
constexpr double POW_A = 0.666;                    // the exponent 0.666D0
// binom(a, k), k = 1..6
constexpr double POW_B1 = POW_A;
constexpr double POW_B2 = POW_B1 * (POW_A - 1.0) / 2.0;
constexpr double POW_B3 = POW_B2 * (POW_A - 2.0) / 3.0;
constexpr double POW_B4 = POW_B3 * (POW_A - 3.0) / 4.0;
constexpr double POW_B5 = POW_B4 * (POW_A - 4.0) / 5.0;
constexpr double POW_B6 = POW_B5 * (POW_A - 5.0) / 6.0;

#ifdef __CUDA_ARCH__
#define AXJ_POW_LD(p) __ldg(p)
AXJ_HD long long pow_bits(double x) { return __double_as_longlong(x); }
AXJ_HD double pow_from_bits(long long b) { return __longlong_as_double(b); }
AXJ_HD double pow_fallback(double T) { return exp2(POW_A * log2(T)); }
#else
#define AXJ_POW_LD(p) (*(p))
inline long long pow_bits(double x) {
  long long b;
  std::memcpy(&b, &x, sizeof b);
  return b;
}
inline double pow_from_bits(long long b) {
  double x;
  std::memcpy(&x, &b, sizeof x);
  return x;
}
inline double pow_fallback(double T) { return std::exp2(POW_A * std::log2(T)); }
#endif

// T**0.666 from the tables tab[POW_TAB] (pow0666_fill).
AXJ_HD double pow0666(double T, const double* __restrict__ tab) {
  const long long bits = pow_bits(T);
  const int hi = (int)(bits >> 32);
  const int e = (hi >> 20) - 1023;
  if (!(T > 0.0) || e < POW_E0 || e >= POW_E0 + POW_NE) return pow_fallback(T);
  const int j = (hi >> 13) & (POW_NJ - 1);
  const double m = pow_from_bits((bits & 0x000FFFFFFFFFFFFFLL) | 0x3FF0000000000000LL);
  const double c = AXJ_POW_LD(tab + 3 * j);
  const double gh = AXJ_POW_LD(tab + 3 * j + 1), gl = AXJ_POW_LD(tab + 3 * j + 2);
  const double* te = tab + 3 * POW_NJ + 2 * (e - POW_E0);
  const double eh = AXJ_POW_LD(te), el = AXJ_POW_LD(te + 1);
  const double r = fma(m, c, -1.0);
  double t = fma(r, POW_B6, POW_B5);
  t = fma(r, t, POW_B4);
  t = fma(r, t, POW_B3);
  t = fma(r, t, POW_B2);
  t = fma(r, t, POW_B1);
  const double q = r * t;  // (1 + r)^a - 1
  // P = 2^(a e) c_j^(-a) as ph + pl, then P (1 + q) rounded once
  const double ph = eh * gh;
  const double pl = fma(eh, gh, -ph) + fma(eh, gl, el * gh);
  return ph + fma(ph, q, pl);
}

// The tables of pow0666, evaluated on the host in long double (64-bit significand) and
// split into double hi + lo parts.
inline void pow0666_fill(double* tab) {
  const long double a = (long double)POW_A;
  for (int j = 0; j < POW_NJ; ++j) {
    const long double F = 1.0L + ((long double)j + 0.5L) / (long double)POW_NJ;
    const double c = std::ldexp(std::nearbyint(std::ldexp((double)(1.0L / F), 9)), -9);  // 10 bits
    const long double g = powl((long double)c, -a);
    tab[3 * j] = c;
    tab[3 * j + 1] = (double)g;
    tab[3 * j + 2] = (double)(g - (long double)tab[3 * j + 1]);
  }
  for (int k = 0; k < POW_NE; ++k) {
    const long double v = exp2l(a * (long double)(POW_E0 + k));
    double* te = tab + 3 * POW_NJ + 2 * k;
    te[0] = (double)v;
    te[1] = (double)(v - (long double)te[0]);
  }
}

}  // namespace axj
