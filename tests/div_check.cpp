// Host check of chq::div6 and chq::divz (chasqui_b200/csrc/chq_divide.cuh) against IEEE
// division: special values, every power-of-two scale, random significands across the whole
// exponent range, and exhaustive significands near the fast-path limits. Built and run by
// tests/test_divide.py; prints "ok <cases>" or the first mismatch.
#include <cstdint>
#include <cstdlib>
#include <initializer_list>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <limits>
#include "chq_divide.cuh"

template <class T, class U> static U bits(T x) { U u; std::memcpy(&u, &x, sizeof(u)); return u; }

template <class T, class U> static bool same(T a, T b) {
  if (std::isnan(a) && std::isnan(b)) return true;
  return bits<T, U>(a) == bits<T, U>(b);
}

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint64_t next() {   // splitmix64
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class T, class U> static long check(T x, T y, long &n) {
  ++n;
  if (!same<T, U>(chq::div6(x), x / T(6))) {
    std::printf("div6 mismatch x=%a got %a want %a\n", (double)x, (double)chq::div6(x), (double)(x / T(6)));
    return 1;
  }
  if (!same<T, U>(chq::divz(x, y), x / y)) {
    std::printf("divz mismatch a=%a b=%a got %a want %a\n", (double)x, (double)y, (double)chq::divz(x, y), (double)(x / y));
    return 1;
  }
  return 0;
}

int main(int argc, char **argv) {
  const long nrand = (argc > 1) ? std::atol(argv[1]) : 20000000;
  long n = 0, bad = 0;
  const double sp[] = {0.0, -0.0, 1.0, -1.0, 6.0, 3.0, 0x1p-1022, 0x1p-1074, -0x1p-1074, 0x1p-1000, 0x1p+1000,
                       1.7976931348623157e308, -1.7976931348623157e308, INFINITY, -INFINITY, NAN, 1e-300, 1e300};
  for (double a : sp)
    for (double b : sp) bad += check<double, uint64_t>(a, b, n);
  for (float a : {0.0f, -0.0f, 1.0f, 6.0f, 0x1p-126f, 0x1p-149f, 0x1p-120f, 0x1p+120f, 3.4e38f, INFINITY, NAN})
    for (float b : {0.0f, -0.0f, 1.0f, -2.5f, INFINITY, NAN, 0x1p-149f}) bad += check<float, uint32_t>(a, b, n);
  // random significands at random exponents over the whole range
  for (long q = 0; q < nrand && !bad; ++q) {
    const uint64_t r = next();
    const double x = bits<uint64_t, double>(r);
    const double y = bits<uint64_t, double>(next());
    bad += check<double, uint64_t>(x, y, n);
    bad += check<double, uint64_t>(std::ldexp(1.0 + (double)(r >> 12) * 0x1p-52, (int)(r % 2001) - 1000), 1.5, n);
    const float xf = bits<uint32_t, float>((uint32_t)r), yf = bits<uint32_t, float>((uint32_t)(r >> 32));
    bad += check<float, uint32_t>(xf, yf, n);
  }
  // every float significand at three exponents (fast path, both limits)
  for (uint32_t m = 0; m < (1u << 23) && !bad; ++m)
    for (int e : {-120, 0, 119}) bad += check<float, uint32_t>(std::ldexp(1.0f + (float)m * 0x1p-23f, e), 3.0f, n);
  if (bad) return 1;
  std::printf("ok %ld\n", n);
  return 0;
}
