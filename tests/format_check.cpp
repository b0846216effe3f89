// Checks gvh::fmt::g6 (the surface.dat number formatter) against printf's "%g" and
// std::to_chars(general, 6) on random values, exact ties at the seventh digit, powers of ten
// and the boundaries where %g switches notation. Built and run by test_format_host.py.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <random>

#include "gvh_format.hpp"

int main() {
  std::mt19937_64 rng(12345);
  long long bad = 0, n = 0;
  auto check = [&](double x) {
    char a[64], b[64], c[64];
    *gvh::fmt::g6(a, a + sizeof a, x) = 0;
    *std::to_chars(b, b + sizeof b, x, std::chars_format::general, 6).ptr = 0;
    snprintf(c, sizeof c, "%g", x);
    ++n;
    if (strcmp(a, b) || strcmp(a, c)) {
      if (bad < 10) printf("mismatch %.17g: '%s' to_chars '%s' printf '%s'\n", x, a, b, c);
      ++bad;
    }
  };
  std::uniform_int_distribution<int> ed(-30, 30);
  std::uniform_real_distribution<double> ud(1.0, 10.0);
  for (int i = 0; i < 1000000; ++i) {
    double x = ud(rng) * pow(10.0, ed(rng));
    check((rng() & 1) ? -x : x);
  }
  for (int e = -20; e <= 25; ++e)
    for (int m = 0; m < 2000; ++m) {
      const double tie = (100000 + (double)(rng() % 900000)) + 0.5;  // a tie at the 7th digit
      check(tie * pow(10.0, e - 5));
      check(nextafter(tie, 0.0) * pow(10.0, e - 5));
      check((double)(rng() % 1000000) * pow(10.0, e));
      check(pow(10.0, e));
      check(nextafter(pow(10.0, e), 0.0));
      check(999999.5 * pow(10.0, e));
      check(99999.5 * pow(10.0, e));
    }
  const double special[] = {0.0, -0.0, 1.0, -1.0, 1e-4, 1e-5, 9.99995e-5, 123456, 1234567, 999999.5, 999999.49999,
                            0.5, 1e22, 1e23, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
                            INFINITY, -INFINITY, NAN};
  for (double x : special) check(x);
  printf("%lld values, %lld mismatches\n", n, bad);
  return bad != 0;
}
