// chasqui_b200 — correctly rounded divisions for the two shapes that dominate the flux kernel.
//
// On sm_100a an IEEE division whose numerator is zero (or subnormal) leaves the fast path of
// the division sequence and runs about 3x slower than an ordinary one (measured with CUDA
// events on a B200). Cells of a quiet region produce many exact zeros: vanishing slopes, zero
// velocities, a zero face-normal field. Both helpers return exactly the IEEE quotient, so
// the bitwise parity of the FP64 form is unchanged.
//
//   div6(x)     RN(x / 6): the constant divisor of the PPM / PPMX / WENO-Z interface
//               formulas, without a division. q = RN(x c) with c = RN(1/6); the remainder
//               r = x - 6 q is exact when q is within one ulp of x/6 (it is), and one
//               correction q + r c (Markstein, IBM J. Res. Dev. 34 (1990) 111) differs from
//               x/6 by less than 2^-p ulp. The significand of x/6 is an integer divided by 3
//               times a power of two, so x/6 is never closer than 1/6 ulp to a rounding
//               midpoint; the corrected value therefore rounds to RN(x/6). Zero, tiny,
//               infinite and NaN arguments take the plain path (exact product or division).
//   divz(a, b)  a / b with a fast exit for a == 0: for finite nonzero b the product a * b is
//               the same signed zero as the quotient.
// Compiles for the host as well (tests/div_check.cpp checks both against the division).
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define CHQ_DIV_HD __host__ __device__ __forceinline__
#else
#define CHQ_DIV_HD inline
#endif

namespace chq {

template <class T> struct DivConst;
template <> struct DivConst<double> {
  static constexpr double sixth = 1.0 / 6.0;     // RN(1/6), folded by the compiler
  static constexpr double tiny = 0x1p-1000;      // below this the quotient may lose bits
  static constexpr double huge = 0x1p+1000;
  static constexpr double maxv = 1.7976931348623157e308;   // largest finite double
};
template <> struct DivConst<float> {
  static constexpr float sixth = 1.0f / 6.0f;
  static constexpr float tiny = 0x1p-120f;
  static constexpr float huge = 0x1p+120f;
  static constexpr float maxv = 3.40282347e38f;            // largest finite float
};

CHQ_DIV_HD double fma_(double a, double b, double c) { return fma(a, b, c); }
CHQ_DIV_HD float fma_(float a, float b, float c) { return fmaf(a, b, c); }
CHQ_DIV_HD double mul_rn(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
CHQ_DIV_HD float mul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}

template <class T> CHQ_DIV_HD T div6(T x) {
  const T c = DivConst<T>::sixth;
  const T ax = (x < T(0)) ? -x : x;
  if (ax >= DivConst<T>::tiny && ax <= DivConst<T>::huge) {
    const T q = mul_rn(x, c);
    const T r = fma_(T(-6), q, x);
    return fma_(r, c, q);
  }
  if (x == T(0)) return mul_rn(x, c);   // the signed zero of x / 6
  return x / T(6);
}

template <class T> CHQ_DIV_HD T divz(T a, T b) {
  const T ab = (b < T(0)) ? -b : b;
  if (a == T(0) && ab != T(0) && ab <= DivConst<T>::maxv) return mul_rn(a, b);
  return a / b;
}

}  // namespace chq
