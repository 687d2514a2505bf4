// mhy_pow_third.h -- V^(1./3.) for the characteristic length, identical on host and device.
//
// MaHyCo evaluates the characteristic length as math::pow(volume, 1./3.)
// (mahyco/src/MahycoModule.cc:1226,1259, option "racine-cubique-volume").
// std::pow (glibc) and CUDA's pow may differ by an ulp, which would make a
// bitwise comparison between the CPU oracle and the GPU impossible.  This
// header gives one function, written from the mathematics, that both sides can
// call so that they produce the same bits:
//
//   t = fl(1/3) = 1/3 - delta,  delta = 2^-54 / 3  (exact: fl(1/3) = 6004799503160661 * 2^-54)
//   V^t = cbrt(V) * exp(-delta * ln V) = cbrt(V) * (1 - delta ln V) + O(delta^2 ln^2 V)
//
// cbrt(V) is obtained from Newton's iteration for the reciprocal cube root of
// m (the mantissa scaled into [1,8)), which needs no division, then refined to
// a double-double y + ylo with an exact residual m - y^3 built from error-free products (fma(a,b,-ab) is the exact rounding
// error of a*b; Dekker 1971 / Ogita-Rump-Oishi 2005).  ln V is needed only to
// ~1e-10 relative (the correction term is at most 1.4e-14 of the result) and is
// taken from the atanh series ln m = 2 atanh((m-1)/(m+1)) on m in [sqrt(1/2), sqrt(2)).
// The result is the double-double value rounded once, i.e. correctly rounded
// except when the exact value lies within ~1e-25 relative of a rounding
// boundary.  Only +, -, *, /, fma and bit manipulation are used; every one of
// them is correctly rounded on both x86-64 and sm_100a, so host and device agree
// bit for bit provided the compiler does not contract a*b+c on its own
// (build with -ffp-contract=off / --fmad=false).
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define MHY_POW_HD __host__ __device__ __forceinline__
#else
#define MHY_POW_HD inline
#endif

namespace mhy {

MHY_POW_HD uint64_t pow3_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u; memcpy(&u, &x, sizeof u); return u;
#endif
}

MHY_POW_HD double pow3_from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x; memcpy(&x, &u, sizeof x); return x;
#endif
}

MHY_POW_HD double pow3_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

// V^(1./3.) for V > 0; NaN for V < 0 or NaN, 0 for +-0, +inf for +inf (the
// values std::pow returns for these arguments with a positive non-integer exponent).
MHY_POW_HD double pow_third(double v) {
  if (!(v > 0.0)) {
    if (v == 0.0) return 0.0;
    return pow3_from_bits(0x7ff8000000000000ull);      // NaN
  }
  uint64_t b = pow3_bits(v);
  int be = (int)((b >> 52) & 0x7ff);
  if (be == 0x7ff) return v;                            // +inf
  int ex_adj = 0;
  if (be == 0) {                                        // subnormal: scale by 2^120 (exact)
    v = v * pow3_from_bits((uint64_t)(1023 + 120) << 52);
    b = pow3_bits(v);
    be = (int)((b >> 52) & 0x7ff);
    ex_adj = -120;
  }
  const int ex = be - 1023 + ex_adj;                    // V = m * 2^ex, m in [1,2)
  const double m = pow3_from_bits((b & 0x000fffffffffffffull) | (0x3ffull << 52));

  // ex = 3q + r with r in {0,1,2}
  int q = (ex >= 0) ? ex / 3 : -((-ex + 2) / 3);
  const int r = ex - 3 * q;
  const double mr = m * (double)(1 << r);               // [1,8), exact

  // Reciprocal cube root w ~ m^(-1/3) 2^(-r/3) by Newton's iteration
  // w <- w + w (1 - mr w^3) / 3, which needs no division, from a quadratic
  // start on [1,2) (max rel. error 3e-3) -> 3 iterations reach full precision.
  double w = (0.09202394 * m - 0.47733264) * m + 1.38237822;
  w = w * (r == 0 ? 1.0 : (r == 1 ? 0.7937005259840998 : 0.6299605249474366));
  const double third = 1.0 / 3.0;
  for (int it = 0; it < 3; ++it) {
    const double w3 = (w * w) * w;
    w = w + w * ((1.0 - mr * w3) * third);
  }
  const double w2 = w * w;
  double y = mr * w2;                                   // cbrt(mr), within a few ulps
  // one Newton step on y itself, using 1/(3 y^2) ~ w^2 / 3
  {
    const double yy = y * y;
    y = y - (yy * y - mr) * (w2 * third);
  }
  // Exact-ish residual res = mr - y^3 with error-free transformations.
  const double y2 = y * y;
  const double e2 = pow3_fma(y, y, -y2);                // y*y = y2 + e2 exactly
  const double y3 = y2 * y;
  const double e3 = pow3_fma(y2, y, -y3);               // y2*y = y3 + e3 exactly
  // y^3 = y3 + e3 + e2*y (+ e2*... terms below 2^-150 relative)
  const double res = ((mr - y3) - e3) - e2 * y;         // mr - y3 exact (Sterbenz)
  const double ylo = res * (w2 * third);                // res / (3 y^2) to ~1e-15 relative

  // ln V = ex*ln2 + ln m with m folded into [sqrt(1/2), sqrt(2)).
  double mm = m;
  int exl = ex;
  if (mm > 1.4142135623730951) { mm = mm * 0.5; exl += 1; }
  const double s = (mm - 1.0) / (mm + 1.0);
  const double s2 = s * s;
  // 2*(s + s^3/3 + ... + s^15/15): truncation < 1e-13 for |s| <= 0.1716
  double poly = 1.0 / 15.0;
  poly = poly * s2 + 1.0 / 13.0;
  poly = poly * s2 + 1.0 / 11.0;
  poly = poly * s2 + 1.0 / 9.0;
  poly = poly * s2 + 1.0 / 7.0;
  poly = poly * s2 + 1.0 / 5.0;
  poly = poly * s2 + 1.0 / 3.0;
  poly = poly * s2 + 1.0;
  const double lnv = (double)exl * 0.6931471805599453 + 2.0 * s * poly;
  const double delta = 1.850371707708594e-17;          // 2^-54 / 3
  const double eps = delta * lnv;

  // V^t = (y + ylo) * (1 - eps) * 2^q, rounded once.
  const double corr = ylo - y * eps;
  const double out = y + corr;
  // scale by 2^q (q in [-358, 341]); two steps keep every factor normal.
  const int q1 = q / 2, q2 = q - q1;
  return out * pow3_from_bits((uint64_t)(1023 + q1) << 52)
             * pow3_from_bits((uint64_t)(1023 + q2) << 52);
}

}  // namespace mhy
