// gvh_format.hpp -- printf's "%g" (6 significant digits) for one double, fast.
//
// The reference writes surface.dat through an ofstream in its default format, which is
// printf's %g with precision 6 (HydroPlugin.cpp:315-372). std::to_chars(general, 6) gives the
// same characters but costs ~80 ns a number; a surface.dat row has 20 numbers, the
// benchmark event's surface 50 M rows. This does the common case with one scaling by an
// exact power of ten and integer digit emission, and hands every case it cannot decide
// exactly to std::to_chars:
//  * the six digits are D = round(|x| 10^(5-E)). The scaling is one correctly rounded
//    multiplication or division by 10^k, k <= 22 (exact powers), so the computed quotient is
//    within 2^-53 relative (under 1.2e-10 absolute below 1e6) of the exact one. When its
//    fractional part is within 1e-7 of 1/2 the rounding direction (and printf's tie rule)
//    cannot be read off it, and the exact path formats the number instead;
//  * E is the decimal exponent after rounding, as printf chooses it: D must land in
//    [1e5, 1e6), otherwise E moves by one and the scaling is redone;
//  * zero is written directly ("0", "-0"); non-finite values and exponents outside
//    [-17, 27] go to the exact path.
// g6_fast is the fast path alone, for host and device: it returns nullptr where the exact
// path must decide (the device leaves those numbers to the host).
// Fixed notation for -4 <= E < 6, else d.ddddde+XX, trailing zeros and a bare decimal point
// removed: printf's %g rules.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#ifndef __CUDA_ARCH__
#include <charconv>
#endif

#ifdef __CUDACC__
#define GVH_FMT_HD __host__ __device__
#else
#define GVH_FMT_HD
#endif

namespace gvh {
namespace fmt {

// 1e0 .. 1e22, each exactly representable
GVH_FMT_HD inline double pow10_exact(int k) {
#ifdef __CUDA_ARCH__
  double r = 1.0;
  for (int i = 0; i < k; ++i) r *= 10.0;  // exact: 10^i = 2^i 5^i and 5^22 < 2^53
  return r;
#else
  static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                    1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
  return kPow10[k];
#endif
}

// The fast path of %g (6 significant digits) for x at p (at most 16 characters); returns the
// end, or nullptr when the exact path must format x (nothing is written then).
GVH_FMT_HD inline char *g6_fast(char *p, double x) {
  if (!isfinite(x)) return nullptr;
  int64_t bits;
  memcpy(&bits, &x, sizeof bits);
  if (x == 0.0) {  // printf writes "0" and "-0"
    if (bits < 0) *p++ = '-';
    *p++ = '0';
    return p;
  }
  const double a = fabs(x);
  // decimal exponent estimate from the binary one (a = m 2^b, m in [1, 2)): floor(b log10 2)
  // is E or E - 1; the loop below corrects it
  const int b = (int)(((bits & 0x7fffffffffffffffll) >> 52) & 0x7ff) - 1023;
  int E = (b * 78913) >> 18;  // floor(b * log10(2)) for |b| < 2^11 (78913 / 2^18 = 0.30103)
  uint32_t D = 0;
  for (int attempt = 0;; ++attempt) {
    const int k = 5 - E;
    if (k > 22 || k < -22 || attempt > 2) return nullptr;
    const double q = k >= 0 ? a * pow10_exact(k) : a / pow10_exact(-k);
    const double fl = floor(q);
    const double frac = q - fl;
    if (fabs(frac - 0.5) < 1e-7) return nullptr;
    const double r = frac > 0.5 ? fl + 1.0 : fl;
    if (r >= 1e6) { ++E; continue; }
    if (r < 1e5) { --E; continue; }
    D = (uint32_t)r;
    break;
  }
  char dig[6];
  for (int i = 5; i >= 0; --i) {
    dig[i] = (char)('0' + D % 10);
    D /= 10;
  }
  int nd = 6;  // significant digits left after removing trailing zeros
  while (nd > 1 && dig[nd - 1] == '0') --nd;
  if (x < 0) *p++ = '-';
  if (E >= -4 && E < 6) {
    if (E >= 0) {
      for (int i = 0; i <= E; ++i) *p++ = dig[i];
      if (nd > E + 1) {
        *p++ = '.';
        for (int i = E + 1; i < nd; ++i) *p++ = dig[i];
      }
    } else {
      *p++ = '0';
      *p++ = '.';
      for (int i = 0; i < -E - 1; ++i) *p++ = '0';
      for (int i = 0; i < nd; ++i) *p++ = dig[i];
    }
  } else {
    *p++ = dig[0];
    if (nd > 1) {
      *p++ = '.';
      for (int i = 1; i < nd; ++i) *p++ = dig[i];
    }
    *p++ = 'e';
    int ex = E;
    if (ex < 0) {
      *p++ = '-';
      ex = -ex;
    } else {
      *p++ = '+';
    }
    if (ex >= 100) {
      *p++ = (char)('0' + ex / 100);
      ex %= 100;
      *p++ = (char)('0' + ex / 10);
      *p++ = (char)('0' + ex % 10);
    } else {
      *p++ = (char)('0' + ex / 10);
      *p++ = (char)('0' + ex % 10);
    }
  }
  return p;
}

#ifndef __CUDA_ARCH__
inline char *g6_exact(char *p, char *end, double x) {
  return std::to_chars(p, end, x, std::chars_format::general, 6).ptr;
}

// Writes %g of x at p (at most 16 characters); returns the end.
inline char *g6(char *p, char *end, double x) {
  char *q = g6_fast(p, x);
  return q ? q : g6_exact(p, end, x);
}
#endif

}  // namespace fmt
}  // namespace gvh
