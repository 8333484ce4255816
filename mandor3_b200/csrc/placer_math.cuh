// Box-Muller transform of the ranmar placer with its own logarithm and
// sine/cosine, built only from IEEE additions, multiplications, divisions
// and square roots (each correctly rounded on the host and on the GPU, no
// fused multiply-add under --fmad=false), so that a marker's momenta are
// the same bits on the device as in a C restatement on the host.
//
//   u in [0, 1) (a multiple of 2^-24, a ranmar draw):
//   r = sqrt(-2 log(1 - u3)),  (cos, sin)(2 pi u4)  and likewise u5, u6.
//
// log v, v in (0, 1]: v = m 2^e with m in [sqrt(1/2), sqrt(2)) (frexp, then
// one exact doubling), log v = e ln2 + 2 atanh(s), s = (m - 1)/(m + 1),
// |s| < 0.1716, and 2 atanh(s) = 2 s (1 + s^2/3 + s^4/5 + ...) summed by
// Horner's rule over 12 terms (the 13th is below 2^-60 of the sum); ln2 is
// split in a part whose product with e is exact and a correction.
//
// (cos, sin)(2 pi u): 4u = q + f with integer quadrant q and f in [0, 1)
// (both exact); the angle (pi/2) min(f, 1 - f) lies in [0, pi/4], where
// the Taylor series of sin (terms to t^17) and cos (to t^18) are summed by
// Horner's rule in t^2; the complementary angle swaps sin and cos, and the
// quadrant rotates the pair.
//
// Coefficients are the doubles nearest 1/(2n+1), (-1)^n/(2n+1)! and
// (-1)^n/(2n)!, written as hexadecimal literals.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define PM_FN __host__ __device__ __forceinline__
#else
#define PM_FN static inline
#endif

PM_FN double pm_log (double v)
{
   int e = 0;
   double m = frexp (v, &e);                     // v = m 2^e, m in [1/2, 1)
   if (m < 0x1.6a09e667f3bcdp-1) {               // sqrt(1/2)
      m = m*2.0;
      e = e - 1;
   }
   const double s = (m - 1.0)/(m + 1.0);
   const double z = s*s;
   double p = 0x1.47ae147ae147bp-5;              // 1/25
   p = p*z + 0x1.642c8590b2164p-5;               // 1/23
   p = p*z + 0x1.8618618618618p-5;               // 1/21
   p = p*z + 0x1.af286bca1af28p-5;               // 1/19
   p = p*z + 0x1.e1e1e1e1e1e1ep-5;               // 1/17
   p = p*z + 0x1.1111111111111p-4;               // 1/15
   p = p*z + 0x1.3b13b13b13b14p-4;               // 1/13
   p = p*z + 0x1.745d1745d1746p-4;               // 1/11
   p = p*z + 0x1.c71c71c71c71cp-4;               // 1/9
   p = p*z + 0x1.2492492492492p-3;               // 1/7
   p = p*z + 0x1.999999999999ap-3;               // 1/5
   p = p*z + 0x1.5555555555555p-2;               // 1/3
   p = p*z + 1.0;
   const double ln2_hi = 0x1.62e42fee00000p-1;   // ln 2 to 32 bits: e ln2_hi is exact
   const double ln2_lo = 0x1.a39ef35793c76p-33;  // ln 2 - ln2_hi
   const double de = (double) e;
   return de*ln2_hi + (de*ln2_lo + 2.0*s*p);
}

PM_FN void pm_sincos_2pi (double u, double *sn, double *cs)
{
   const double x = 4.0*u;
   const double q = floor (x);
   double f = x - q;
   const int swap = f > 0.5;
   if (swap)
      f = 1.0 - f;
   const double t = f*0x1.921fb54442d18p+0;      // pi/2
   const double z = t*t;
   double ps = 0x1.952c77030ad4ap-49;            // 1/17!
   ps = ps*z - 0x1.ae7f3e733b81fp-41;            // 1/15!
   ps = ps*z + 0x1.6124613a86d09p-33;            // 1/13!
   ps = ps*z - 0x1.ae64567f544e4p-26;            // 1/11!
   ps = ps*z + 0x1.71de3a556c734p-19;            // 1/9!
   ps = ps*z - 0x1.a01a01a01a01ap-13;            // 1/7!
   ps = ps*z + 0x1.1111111111111p-7;             // 1/5!
   ps = ps*z - 0x1.5555555555555p-3;             // 1/3!
   ps = ps*z + 1.0;
   double pc = -0x1.6827863b97d97p-53;           // 1/18!
   pc = pc*z + 0x1.ae7f3e733b81fp-45;            // 1/16!
   pc = pc*z - 0x1.93974a8c07c9dp-37;            // 1/14!
   pc = pc*z + 0x1.1eed8eff8d898p-29;            // 1/12!
   pc = pc*z - 0x1.27e4fb7789f5cp-22;            // 1/10!
   pc = pc*z + 0x1.a01a01a01a01ap-16;            // 1/8!
   pc = pc*z - 0x1.6c16c16c16c17p-10;            // 1/6!
   pc = pc*z + 0x1.5555555555555p-5;             // 1/4!
   pc = pc*z - 0.5;                              // 1/2!
   pc = pc*z + 1.0;
   const double st = t*ps;
   const double s0 = swap ? pc : st, c0 = swap ? st : pc;
   switch ((int) q) {
   case 0:  *sn = s0;  *cs = c0;  break;
   case 1:  *sn = c0;  *cs = -s0; break;
   case 2:  *sn = -s0; *cs = -c0; break;
   default: *sn = -c0; *cs = s0;  break;
   }
}

// Normal pair of one marker's draws: (r cos, r sin) of (u_r, u_t).
PM_FN void pm_box_muller (double u_r, double u_t, double *a, double *b)
{
   const double r = sqrt (-2.0*pm_log (1.0 - u_r));
   double sn, cs;
   pm_sincos_2pi (u_t, &sn, &cs);
   *a = r*cs;
   *b = r*sn;
}

#undef PM_FN
