// Elementary functions with a fixed operation sequence, compiled identically for the host (g++) and the
// device (nvcc).  Every step is a correctly rounded IEEE-754 binary32 operation (add, mul, fma, rint), so the
// CPU oracle and the parity build of the GPU kernels produce the same bits for the same argument.
//
// Methods (from the mathematics, not from any vendor library):
//  * ps_expf: Cody–Waite argument reduction x = k·ln2 + r (ln2 split into a 16-bit head and a tail, both
//    products folded with fma), then the degree-7 Taylor polynomial of e^r on |r| <= ln2/2 evaluated by Horner's
//    rule, then scaling by 2^k through the exponent field.  Truncation error of the polynomial is below
//    (ln2/2)^8/8! ~ 5e-9 relative; measured error is about 1 ulp.  Results below 2^-126·(e^-0.35) are flushed
//    to +0 (arguments below -87.33); arguments above 88.0 return +inf.  All call sites in this project pass
//    arguments <= 0.
//  * ps_exp64: binary64 e^x by the same scheme: x = k·ln2 + r with ln2 split into a head of 32 significant bits
//    (k·ln2_hi exact for |k| < 2^21) and a tail, both products folded with fma; the degree-13 Taylor polynomial of
//    e^r on |r| <= ln2/2 (truncation below 2^-57 relative) by Horner's rule with fma; scaling by 2^k through the
//    exponent field (in two steps below 2^-1022).  Arguments above 709 give +inf, below -745.2 give +0.
//  * ps_acos64: binary64 arc cosine on [-1, 1]: acos x = pi/2 - asin x for |x| <= 1/2, 2·asin(sqrt((1 - x)/2)) above
//    and pi - 2·asin(sqrt((1 + x)/2)) below (1 ∓ x and the halving are exact there); asin y on |y| <= 1/2 by its Taylor
//    series y·Σ c_n y^(2n), c_n = (2n)!/(4^n (n!)^2 (2n+1)), 28 terms by Horner's rule with fma (truncation below
//    2^-60 relative).
//  * ps_sincosf: Cody–Waite reduction by pi/2 (three-part split of pi/2 folded with fma, valid for |x| < 1e5),
//    then Taylor polynomials of degree 9 (sin) and 10 (cos) on |r| <= pi/4 (truncation error < 2e-9), with the
//    quadrant selecting sign and swap.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define PS_HD __host__ __device__ __forceinline__
#else
#define PS_HD static inline
#endif

PS_HD float ps_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, sizeof f);
  return f;
#endif
}

PS_HD uint32_t ps_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, sizeof u);
  return u;
#endif
}

PS_HD float ps_expf(float x) {
  if (!(x == x)) return x;                        // NaN in, NaN out
  if (x > 88.0f) return ps_u2f(0x7f800000u);      // +inf
  if (x < -87.33f) return 0.0f;                   // below the smallest normal: flushed to zero
  const float log2e = (float)1.4426950408889634;  // 1/ln 2
  const float ln2_hi = (float)0.693145751953125;  // ln 2 rounded to 16 significant bits (k·ln2_hi exact)
  const float ln2_lo = (float)1.4286068203094173e-06;  // ln 2 - ln2_hi
  float k = rintf(x * log2e);
  float r = fmaf(-k, ln2_hi, x);
  r = fmaf(-k, ln2_lo, r);
  float p = (float)(1.0 / 5040.0);
  p = fmaf(p, r, (float)(1.0 / 720.0));
  p = fmaf(p, r, (float)(1.0 / 120.0));
  p = fmaf(p, r, (float)(1.0 / 24.0));
  p = fmaf(p, r, (float)(1.0 / 6.0));
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  int ki = (int)k;                                // k in [-126, 127]
  return p * ps_u2f((uint32_t)(ki + 127) << 23);
}

PS_HD double ps_u2d(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double f;
  memcpy(&f, &u, sizeof f);
  return f;
#endif
}

PS_HD double ps_exp64(double x) {
  if (!(x == x)) return x;
  if (x > 709.0) return ps_u2d(0x7ff0000000000000ull);
  if (x < -745.2) return 0.0;
  const double ln2_hi = 0.6931471803691238;     // ln 2 to 32 significant bits
  const double ln2_lo = 1.9082149292705877e-10;  // ln 2 - ln2_hi
  const double k = rint(x * 1.4426950408889634);
  double r = fma(-k, ln2_hi, x);
  r = fma(-k, ln2_lo, r);
  double p = 1.6059043836821613e-10;  // 1/13!
  p = fma(p, r, 2.08767569878681e-09);
  p = fma(p, r, 2.505210838544172e-08);
  p = fma(p, r, 2.755731922398589e-07);
  p = fma(p, r, 2.7557319223985893e-06);
  p = fma(p, r, 2.48015873015873e-05);
  p = fma(p, r, 0.0001984126984126984);
  p = fma(p, r, 0.001388888888888889);
  p = fma(p, r, 0.008333333333333333);
  p = fma(p, r, 0.041666666666666664);
  p = fma(p, r, 0.16666666666666666);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const int ki = (int)k;  // -1075 .. 1023
  if (ki >= -1022) return p * ps_u2d((uint64_t)(ki + 1023) << 52);
  return (p * ps_u2d((uint64_t)(ki + 1023 + 600) << 52)) * ps_u2d((uint64_t)(1023 - 600) << 52);
}

PS_HD double ps_asin_half64(double y) {  // |y| <= 1/2
  const double y2 = y * y;
  double p = 0.0019650336162772837;
  p = fma(p, y2, 0.0020776610325181676);
  p = fma(p, y2, 0.0022014739737101384);
  p = fma(p, y2, 0.002338091892111975);
  p = fma(p, y2, 0.0024894486782468836);
  p = fma(p, y2, 0.00265787063820729);
  p = fma(p, y2, 0.002846178401108942);
  p = fma(p, y2, 0.0030578216492580306);
  p = fma(p, y2, 0.003297059503473485);
  p = fma(p, y2, 0.0035692053938259347);
  p = fma(p, y2, 0.003880964558837669);
  p = fma(p, y2, 0.004240907093679363);
  p = fma(p, y2, 0.004660143486915096);
  p = fma(p, y2, 0.005153309682319905);
  p = fma(p, y2, 0.005740037670841924);
  p = fma(p, y2, 0.006447210311889649);
  p = fma(p, y2, 0.0073125258735988454);
  p = fma(p, y2, 0.008390335809616815);
  p = fma(p, y2, 0.009761609529194078);
  p = fma(p, y2, 0.011551800896139705);
  p = fma(p, y2, 0.01396484375);
  p = fma(p, y2, 0.017352764423076924);
  p = fma(p, y2, 0.022372159090909092);
  p = fma(p, y2, 0.030381944444444444);
  p = fma(p, y2, 0.044642857142857144);
  p = fma(p, y2, 0.075);
  p = fma(p, y2, 0.16666666666666666);
  return fma(y * y2, p, y);
}

PS_HD double ps_acos64(double x) {
  if (!(x == x)) return x;
  if (x > 0.5) return 2.0 * ps_asin_half64(sqrt((1.0 - x) * 0.5));
  if (x < -0.5) return 3.141592653589793 - 2.0 * ps_asin_half64(sqrt((1.0 + x) * 0.5));
  return 1.5707963267948966 - ps_asin_half64(x);
}

PS_HD void ps_sincosf(float x, float* s, float* c) {
  const float two_over_pi = (float)0.63661977236758134;
  const float pio2_1 = (float)1.5707963267948966;             // pi/2 rounded to binary32
  const float pio2_2 = (float)(1.5707963267948966 - (double)(float)1.5707963267948966);
  const float pio2_3 = (float)((1.5707963267948966 - (double)(float)1.5707963267948966) -
                               (double)(float)(1.5707963267948966 - (double)(float)1.5707963267948966));
  float q = rintf(x * two_over_pi);
  float r = fmaf(-q, pio2_1, x);
  r = fmaf(-q, pio2_2, r);
  r = fmaf(-q, pio2_3, r);
  float r2 = r * r;
  float ps = (float)(1.0 / 362880.0);
  ps = fmaf(ps, r2, (float)(-1.0 / 5040.0));
  ps = fmaf(ps, r2, (float)(1.0 / 120.0));
  ps = fmaf(ps, r2, (float)(-1.0 / 6.0));
  float sn = fmaf(ps * r2, r, r);
  float pc = (float)(-1.0 / 3628800.0);
  pc = fmaf(pc, r2, (float)(1.0 / 40320.0));
  pc = fmaf(pc, r2, (float)(-1.0 / 720.0));
  pc = fmaf(pc, r2, (float)(1.0 / 24.0));
  pc = fmaf(pc, r2, -0.5f);
  float cs = fmaf(pc, r2, 1.0f);
  int qi = ((int)q) & 3;
  float so = sn, co = cs;
  if (qi == 1) { so = cs; co = -sn; }
  else if (qi == 2) { so = -sn; co = -cs; }
  else if (qi == 3) { so = -cs; co = sn; }
  *s = so;
  *c = co;
}
