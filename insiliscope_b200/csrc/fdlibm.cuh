// Float64 log, exp and cos that round exactly as the world core's (core/src/jsmath.h: V8's port of fdlibm 5.3, the
// Sun Microsystems freely distributable math library), so blink schedules drawn on the device are the core's bit for
// bit. Restated here from fdlibm's published algorithms and coefficients:
//   log  (e_log.c): x = 2^k (1 + f), f in [sqrt(2)/2 - 1, sqrt(2) - 1]; s = f / (2 + f); log(1 + f) = f - s (f - R)
//        with R a degree-14 minimax polynomial in s (Lg1..Lg7), or the hfsq form where f is not small;
//   exp  (e_exp.c): x = k ln2 + r with ln2 in two parts; exp(r) = 1 + r + r c / (2 - c), c = r - r^2 P(r^2) (P1..P5);
//        scaled by 2^k in the exponent field;
//   cos  (s_cos.c, k_cos.c, k_sin.c, e_rem_pio2.c): |x| <= pi/4 directly, else x = n pi/2 + (y0 + y1) with pi/2 in
//        three parts (the medium-size reduction, valid for |x| < 2^19 pi/2; the large-argument Payne-Hanek path is
//        not restated: the schedules' arguments are in [0, 2 pi)), then the degree-14 cosine (C1..C6) or sine
//        (S1..S6) kernel of the quadrant.
// Every operation is a float64 add, multiply or divide in the published order (no contraction: units that include this
// are compiled with --fmad=false, the core with -ffp-contract=off) and IEEE division is exact in CUDA, so the results
// are the core's for every input in the domains above.
#pragma once

#include <cstdint>

namespace iscu {
namespace fd {

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ int32_t Hi(double x) { return __double2hiint(x); }
__device__ __forceinline__ uint32_t Lo(double x) { return static_cast<uint32_t>(__double2loint(x)); }
__device__ __forceinline__ double Words(int32_t hi, uint32_t lo) { return __hiloint2double(hi, static_cast<int>(lo)); }
#else
inline int32_t Hi(double x)
{
   uint64_t b;
   __builtin_memcpy(&b, &x, 8);
   return static_cast<int32_t>(b >> 32);
}
inline uint32_t Lo(double x)
{
   uint64_t b;
   __builtin_memcpy(&b, &x, 8);
   return static_cast<uint32_t>(b);
}
inline double Words(int32_t hi, uint32_t lo)
{
   const uint64_t b = (static_cast<uint64_t>(static_cast<uint32_t>(hi)) << 32) | lo;
   double x;
   __builtin_memcpy(&x, &b, 8);
   return x;
}
#endif

__host__ __device__ inline double Log(double x)
{
   const double ln2Hi = 6.93147180369123816490e-01, ln2Lo = 1.90821492927058770002e-10;
   const double two54 = 1.80143985094819840000e+16;
   const double lg1 = 6.666666666666735130e-01, lg2 = 3.999999999940941908e-01, lg3 = 2.857142874366239149e-01,
                lg4 = 2.222219843214978396e-01, lg5 = 1.818357216161805012e-01, lg6 = 1.531383769920937332e-01,
                lg7 = 1.479819860511658591e-01;
   int32_t hx = Hi(x);
   const uint32_t lx = Lo(x);
   int32_t k = 0;
   if (hx < 0x00100000)   // subnormal, zero or negative
   {
      if (((hx & 0x7fffffff) | static_cast<int32_t>(lx)) == 0)
         return -two54 / 0.0;
      if (hx < 0)
         return (x - x) / 0.0;
      k -= 54;
      x *= two54;
      hx = Hi(x);
   }
   if (hx >= 0x7ff00000)
      return x + x;
   k += (hx >> 20) - 1023;
   hx &= 0x000fffff;
   int32_t i = (hx + 0x95f64) & 0x100000;
   x = Words(hx | (i ^ 0x3ff00000), Lo(x));   // x or x / 2, in [sqrt(2)/2, sqrt(2))
   k += i >> 20;
   const double f = x - 1.0;
   if ((0x000fffff & (2 + hx)) < 3)   // |f| < 2^-20
   {
      if (f == 0.0)
      {
         if (k == 0)
            return 0.0;
         const double dk = static_cast<double>(k);
         return dk * ln2Hi + dk * ln2Lo;
      }
      const double R = f * f * (0.5 - 0.33333333333333333 * f);
      if (k == 0)
         return f - R;
      const double dk = static_cast<double>(k);
      return dk * ln2Hi - ((R - dk * ln2Lo) - f);
   }
   const double s = f / (2.0 + f);
   const double dk = static_cast<double>(k);
   const double z = s * s;
   i = hx - 0x6147a;
   const double w = z * z;
   const int32_t j = 0x6b851 - hx;
   const double t1 = w * (lg2 + w * (lg4 + w * lg6));
   const double t2 = z * (lg1 + w * (lg3 + w * (lg5 + w * lg7)));
   i |= j;
   const double R = t2 + t1;
   if (i > 0)
   {
      const double hfsq = 0.5 * f * f;
      if (k == 0)
         return f - (hfsq - s * (hfsq + R));
      return dk * ln2Hi - ((hfsq - (s * (hfsq + R) + dk * ln2Lo)) - f);
   }
   if (k == 0)
      return f - s * (f - R);
   return dk * ln2Hi - ((s * (f - R) - dk * ln2Lo) - f);
}

__host__ __device__ inline double Exp(double x)
{
   const double oThreshold = 7.09782712893383973096e+02, uThreshold = -7.45133219101941108420e+02;
   const double ln2Hi = 6.93147180369123816490e-01, ln2Lo = 1.90821492927058770002e-10;
   const double invLn2 = 1.44269504088896338700e+00;
   const double p1 = 1.66666666666666019037e-01, p2 = -2.77777777770155933842e-03, p3 = 6.61375632143793436117e-05,
                p4 = -1.65339022054652515390e-06, p5 = 4.13813679705723846039e-08;
   const double huge = 1.0e+300, twom1000 = 9.33263618503218878990e-302;
   double hi = 0.0, lo = 0.0;
   int32_t k = 0;
   uint32_t hx = static_cast<uint32_t>(Hi(x));
   const int32_t xsb = static_cast<int32_t>((hx >> 31) & 1u);
   hx &= 0x7fffffffu;
   if (hx >= 0x40862E42u)   // |x| >= 709.78
   {
      if (hx >= 0x7ff00000u)
      {
         if (((hx & 0xfffffu) | Lo(x)) != 0)
            return x + x;
         return xsb == 0 ? x : 0.0;
      }
      if (x > oThreshold)
         return huge * huge;
      if (x < uThreshold)
         return twom1000 * twom1000;
   }
   if (hx > 0x3fd62e42u)   // |x| > ln2 / 2
   {
      if (hx < 0x3FF0A2B2u)   // |x| < 1.5 ln2
      {
         hi = xsb ? x + ln2Hi : x - ln2Hi;
         lo = xsb ? -ln2Lo : ln2Lo;
         k = 1 - xsb - xsb;
      }
      else
      {
         k = static_cast<int32_t>(invLn2 * x + (xsb ? -0.5 : 0.5));
         const double t = static_cast<double>(k);
         hi = x - t * ln2Hi;
         lo = t * ln2Lo;
      }
      x = hi - lo;
   }
   else if (hx < 0x3e300000u)   // |x| < 2^-28
   {
      if (huge + x > 1.0)
         return 1.0 + x;
   }
   else
   {
      k = 0;
   }
   const double t = x * x;
   const double c = x - t * (p1 + t * (p2 + t * (p3 + t * (p4 + t * p5))));
   if (k == 0)
      return 1.0 - ((x * c) / (c - 2.0) - x);
   const double y = 1.0 - ((lo - (x * c) / (2.0 - c)) - hi);
   if (k >= -1021)
      return Words(Hi(y) + (k << 20), Lo(y));
   return Words(Hi(y) + ((k + 1000) << 20), Lo(y)) * twom1000;
}

// cos(x + y) for |x + y| <= pi/4 (y the tail of a reduced argument)
__host__ __device__ inline double KernelCos(double x, double y)
{
   const double c1 = 4.16666666666666019037e-02, c2 = -1.38888888888741095749e-03, c3 = 2.48015872894767294178e-05,
                c4 = -2.75573143513906633035e-07, c5 = 2.08757232129817482790e-09, c6 = -1.13596475577881948265e-11;
   const int32_t ix = Hi(x) & 0x7fffffff;
   if (ix < 0x3e400000)   // |x| < 2^-27
      if (static_cast<int32_t>(x) == 0)
         return 1.0;
   const double z = x * x;
   const double r = z * (c1 + z * (c2 + z * (c3 + z * (c4 + z * (c5 + z * c6)))));
   if (ix < 0x3FD33333)   // |x| < 0.3
      return 1.0 - (0.5 * z - (z * r - x * y));
   const double qx = ix > 0x3fe90000 ? 0.28125 : Words(ix - 0x00200000, 0u);   // |x| / 4, low word cleared
   const double hz = 0.5 * z - qx;
   const double a = 1.0 - qx;
   return a - (hz - (z * r - x * y));
}

// sin(x + y) for |x + y| <= pi/4; iy = 0: y is zero
__host__ __device__ inline double KernelSin(double x, double y, int iy)
{
   const double s1 = -1.66666666666666324348e-01, s2 = 8.33333333332248946124e-03, s3 = -1.98412698298579493134e-04,
                s4 = 2.75573137070700676789e-06, s5 = -2.50507602534068634195e-08, s6 = 1.58969099521155010221e-10;
   const int32_t ix = Hi(x) & 0x7fffffff;
   if (ix < 0x3e400000)
      if (static_cast<int32_t>(x) == 0)
         return x;
   const double z = x * x;
   const double v = z * x;
   const double r = s2 + z * (s3 + z * (s4 + z * (s5 + z * s6)));
   if (iy == 0)
      return x + v * (s1 + z * r);
   return x - ((z * (0.5 * y - v * r) - y) - v * s1);
}

// x = n pi/2 + y0 + y1 for |x| < 2^19 pi/2 (fdlibm's small and medium cases); returns n.
__host__ __device__ inline int32_t RemPio2(double x, double& y0, double& y1)
{
   const double invPio2 = 6.36619772367581382433e-01;
   const double pio2a = 1.57079632673412561417e+00, pio2at = 6.07710050650619224932e-11;
   const double pio2b = 6.07710050630396597660e-11, pio2bt = 2.02226624879595063154e-21;
   const double pio2c = 2.02226624871116645580e-21, pio2ct = 8.47842766036889956997e-32;
   const int32_t hx = Hi(x), ix = hx & 0x7fffffff;
   if (ix <= 0x3fe921fb)
   {
      y0 = x;
      y1 = 0.0;
      return 0;
   }
   if (ix < 0x4002d97c)   // |x| < 3 pi/4: n = +-1
   {
      if (hx > 0)
      {
         double z = x - pio2a;
         if (ix != 0x3ff921fb)
         {
            y0 = z - pio2at;
            y1 = (z - y0) - pio2at;
         }
         else
         {
            z -= pio2b;
            y0 = z - pio2bt;
            y1 = (z - y0) - pio2bt;
         }
         return 1;
      }
      double z = x + pio2a;
      if (ix != 0x3ff921fb)
      {
         y0 = z + pio2at;
         y1 = (z - y0) + pio2at;
      }
      else
      {
         z += pio2b;
         y0 = z + pio2bt;
         y1 = (z - y0) + pio2bt;
      }
      return -1;
   }
   // medium size: n = rint(|x| 2/pi), the remainder in up to three steps of pi/2's parts
   const double t0 = x < 0.0 ? -x : x;
   const int32_t n = static_cast<int32_t>(t0 * invPio2 + 0.5);
   const double fn = static_cast<double>(n);
   double r = t0 - fn * pio2a;
   double w = fn * pio2at;
   // (the high word of n pi/2: where r may have cancelled to few bits)
   const int32_t nHw = Hi(fn * 1.5707963267948966192);
   if (n < 32 && ix != nHw)
   {
      y0 = r - w;
   }
   else
   {
      const int32_t j = ix >> 20;
      y0 = r - w;
      int32_t i = j - ((Hi(y0) >> 20) & 0x7ff);
      if (i > 16)
      {
         double t = r;
         w = fn * pio2b;
         r = t - w;
         w = fn * pio2bt - ((t - r) - w);
         y0 = r - w;
         i = j - ((Hi(y0) >> 20) & 0x7ff);
         if (i > 49)
         {
            t = r;
            w = fn * pio2c;
            r = t - w;
            w = fn * pio2ct - ((t - r) - w);
            y0 = r - w;
         }
      }
   }
   y1 = (r - y0) - w;
   if (hx < 0)
   {
      y0 = -y0;
      y1 = -y1;
      return -n;
   }
   return n;
}

__host__ __device__ inline double Cos(double x)
{
   const int32_t ix = Hi(x) & 0x7fffffff;
   if (ix <= 0x3fe921fb)
      return KernelCos(x, 0.0);
   if (ix >= 0x7ff00000)
      return x - x;
   double y0, y1;
   const int32_t n = RemPio2(x, y0, y1);
   switch (n & 3)
   {
   case 0:
      return KernelCos(y0, y1);
   case 1:
      return -KernelSin(y0, y1, 1);
   case 2:
      return -KernelCos(y0, y1);
   default:
      return KernelSin(y0, y1, 1);
   }
}

} // namespace fd
} // namespace iscu
