// Device restatement of the engine's counter-based noise stream and its draws.
//
//  - Pcg4d: adapter/inSiliScope/Simulation/SMLMCounterRng.h:37-56 (= core/src/rng.h:18-33), pure uint32 arithmetic.
//  - CounterRng: SMLMCounterRng.h:60-91. A pixel's stream is (seed, frame, pixel, counter): one pcg4d per 4
//    uniforms, consumed a, b, c, d; uniform = ((x >> 9) + 0.5) * 2^-23, exact in float64.
//  - Gauss / Poisson / Gamma: SMLMCounterRng.h:95-138, in float64 with the same operations in the same order.
//
// Bit-exactness with the CPU path rests on (1) no floating-point contraction: every translation unit that includes
// this header is compiled with --fmad=false, as the reference is with -ffp-contract=off (core/CMakeLists.txt:41);
// (2) IEEE float64 sqrt and division (always correctly rounded in CUDA); (3) CUDA's float64 log/exp/cos, which, like
// glibc's, are within an ulp: an integer draw can differ only when its argument sits within ~1e-16 of a count
// boundary. A normal draw that only feeds a rounding (DrawGauss) is first tried in float32: the count it gives is
// taken only when no rounding boundary lies within the float32 form's error bound of it, so every count is the one
// the float64 form gives.
#pragma once

#include <cstdint>

namespace iscu {

__device__ __forceinline__ void Pcg4d(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d)
{
   a = a * 1664525u + 1013904223u;
   b = b * 1664525u + 1013904223u;
   c = c * 1664525u + 1013904223u;
   d = d * 1664525u + 1013904223u;
   a += b * d;
   b += c * a;
   c += a * b;
   d += b * c;
   a ^= a >> 16;
   b ^= b >> 16;
   c ^= c >> 16;
   d ^= d >> 16;
   a += b * d;
   b += c * a;
   c += a * b;
   d += b * c;
}

// The stream's uniform of word x: ((x >> 9) + 0.5) * 2^-23 = v * 2^-24 with v = (x >> 8) | 1, odd and below 2^24.
// Formed exactly without an integer conversion: the double with exponent 2^28 and low word v is 2^28 + v * 2^-24,
// and taking 2^28 away leaves v * 2^-24 (exact: the result is representable).
__device__ __forceinline__ double UniformOf(uint32_t x)
{
   return __hiloint2double(0x41B00000, static_cast<int>((x >> 8) | 1u)) - 268435456.0;
}

// One frame's uniform source; Pixel(p) rewinds it to pixel p's stream. The four words of the current hash are
// consumed in order by shifting, which keeps them in registers.
struct CounterRng
{
   uint32_t seed, frame, pix, ctr;
   uint32_t q0, q1, q2, q3;
   int k;

   __device__ __forceinline__ CounterRng(uint32_t s, uint32_t f) : seed(s), frame(f), pix(0), ctr(0), k(4)
   {
      q0 = q1 = q2 = q3 = 0u;
   }
   __device__ __forceinline__ void Pixel(uint32_t p)
   {
      pix = p;
      ctr = 0;
      k = 4;
   }
   __device__ __forceinline__ double Uniform()
   {
      if (k == 4)
      {
         uint32_t a = seed, b = frame, c = pix, d = ctr;
         Pcg4d(a, b, c, d);
         q0 = a;
         q1 = b;
         q2 = c;
         q3 = d;
         ++ctr;
         k = 0;
      }
      const uint32_t x = q0;
      q0 = q1;
      q1 = q2;
      q2 = q3;
      ++k;
      return UniformOf(x);
   }
   // After a hash drawn outside Uniform() of which `used` words (1..3) were consumed: the rest stays queued.
   __device__ __forceinline__ void Rest(uint32_t r0, uint32_t r1, uint32_t r2, int used)
   {
      q0 = r0;
      q1 = r1;
      q2 = r2;
      k = used;
   }
};

// Box-Muller, radius first, angle second (SMLMCounterRng.h:95-100).
__device__ __forceinline__ double CounterGauss(CounterRng& u)
{
   const double r = sqrt(-2.0 * log(u.Uniform()));
   return r * cos(6.283185307179586 * u.Uniform());
}

// A Box-Muller normal whose value matters only through a rounding to an integer (the read noise of an ADU, the
// rounded normal of a large-mean Poisson draw): the stream's next two uniforms, drawn as CounterGauss draws them
// (radius first, angle second), and gf, the same formula in float32. The uniforms are 24-bit values, exact in float;
// logf and cospif are within 1 ulp and sqrtf is correctly rounded (CUDA's documented bounds), so with |g| <= 5.8
// (u1 >= 2^-24) |gf - g| stays below 2e-6 -- kGaussFastErr is 5x that, covering bounds up to 4 ulp.
constexpr double kGaussFastErr = 1e-5;

struct GaussDraw
{
   double u1, u2;
   float gf;
};

__device__ __forceinline__ GaussDraw DrawGauss(CounterRng& u)
{
   GaussDraw d;
   d.u1 = u.Uniform();
   d.u2 = u.Uniform();
   d.gf = sqrtf(-2.0f * logf(static_cast<float>(d.u1))) * cospif(2.0f * static_cast<float>(d.u2));
   return d;
}

// CounterGauss's value of a draw, with its operations in its order.
__device__ __forceinline__ double GaussExact(const GaussDraw& d)
{
   const double r = sqrt(-2.0 * log(d.u1));
   return r * cos(6.283185307179586 * d.u2);
}

// floor(v + 0.5) for a v known only to within m of vf: true (and the value) when no rounding boundary n + 0.5 lies
// within m of vf, so that every v in [vf - m, vf + m] rounds alike.
__device__ __forceinline__ bool RoundsSurely(double vf, double m, double& out)
{
   const double t = vf + 0.5, f = floor(t);
   if (t - f > m && f + 1.0 - t > m)
   {
      out = f;
      return true;
   }
   return false;
}

// Knuth inversion up to mean 60, the rounded normal beyond; 1000-iteration cap (SMLMCounterRng.h:102-118). The
// rounded normal floor(l + sqrt(l) g + 0.5) is decided from the float32 normal when no rounding boundary is within
// sqrt(l) kGaussFastErr of it, else from CounterGauss's float64 value of the same uniforms: the same count either way.
__device__ __forceinline__ double CounterPoisson(double l, CounterRng& u)
{
   if (l > 60.0)
   {
      const double s = sqrt(l);
      const GaussDraw d = DrawGauss(u);
      double r;
      // (l > 60: l + s g >= sqrt(l) (sqrt(l) - 5.8) > 0, so the fmax never acts on a count decided here)
      if (RoundsSurely(l + s * static_cast<double>(d.gf), s * kGaussFastErr + 1e-9 * l, r) && r >= 1.0)
         return r;
      const double g = GaussExact(d);
      return fmax(0.0, floor(l + s * g + 0.5));
   }
   if (!(l > 0.0))
      return 0.0;
   const double L = exp(-l);
   int k = 0;
   double p = 1.0;
   if (u.k < 4)
   {
      // mid-hash (not the case for a pixel's first draw): one uniform at a time
      do
      {
         ++k;
         p *= u.Uniform();
      } while (p > L && k < 1000);
      return static_cast<double>(k - 1);
   }
   // At a hash boundary: do { ++k; p *= uniform; } while (p > L && k < 1000), a hash (four uniforms) per block;
   // block b's fourth factor is the 4b + 4-th, so only block 249 ends at k = 1000. Every factor lies in (0, 1), so
   // the rounded products never increase: when the block's last product is still above L so are the three before
   // it, and one test per block decides whether the loop goes on. The products are the same roundings in the same
   // order as one factor at a time.
   for (int blk = 0;; ++blk)
   {
      uint32_t a = u.seed, b = u.frame, c = u.pix, d = u.ctr;
      Pcg4d(a, b, c, d);
      ++u.ctr;
      const double p1 = p * UniformOf(a), p2 = p1 * UniformOf(b), p3 = p2 * UniformOf(c), p4 = p3 * UniformOf(d);
      if (p4 > L && blk != 249)
      {
         p = p4;
         continue;
      }
      if (!(p1 > L))
      {
         u.Rest(b, c, d, 1);
         return static_cast<double>(4 * blk);
      }
      if (!(p2 > L))
      {
         u.Rest(c, d, 0u, 2);
         return static_cast<double>(4 * blk + 1);
      }
      if (!(p3 > L))
      {
         u.Rest(d, 0u, 0u, 3);
         return static_cast<double>(4 * blk + 2);
      }
      u.k = 4;
      return static_cast<double>(4 * blk + 3);
   }
}

// Marsaglia-Tsang Gamma(k, 1), 1000-iteration cap (SMLMCounterRng.h:120-136).
__device__ __forceinline__ double CounterGamma(double k, CounterRng& u)
{
   const double d = k - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
   for (int it = 0; it < 1000; ++it)
   {
      const double x = CounterGauss(u), t = 1.0 + c * x;
      if (t <= 0.0)
         continue;
      const double v = t * t * t, w = u.Uniform();
      if (w < 1.0 - 0.0331 * x * x * x * x)
         return d * v;
      if (log(w) < 0.5 * x * x + d * (1.0 - v + log(v)))
         return d * v;
   }
   return d;
}

// CounterGamma's draw with its decisions taken in float32 where each is sure: every iteration's normal from
// DrawGauss (within kGaussFastErr of CounterGauss's value of the same uniforms), then the sign of t = 1 + c x, the
// squeeze w < 1 - 0.0331 x^4 and the logarithmic test log w < x^2 / 2 + d (1 - v + log v), each taken only when no
// normal within that error could decide it the other way. The draws are CounterGamma's, in its order, so the stream
// ends where CounterGamma leaves it. true: out = d v within outErr of CounterGamma's value. false: a decision was in
// doubt (about one iteration in 10^4); the caller draws again from its saved stream with CounterGamma. Taking the
// logarithmic test here too matters: the squeeze alone fails for ~10 % of draws (E[0.0331 x^4] = 0.1), which would
// send nearly every warp down the float64 path as well.
__device__ __forceinline__ bool GammaSure(double k, CounterRng& u, double& out, double& outErr)
{
   const double d = k - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
   const double e = kGaussFastErr, dt = c * e;
   for (int it = 0; it < 1000; ++it)
   {
      const GaussDraw g = DrawGauss(u);
      const double x = static_cast<double>(g.gf), t = 1.0 + c * x;
      if (t + dt <= 0.0)   // t <= 0 for every normal within e of x: CounterGamma draws again
         continue;
      if (!(t - dt > 0.0))
         return false;
      const double tt = t + dt, v = t * t * t, dv = 3.0 * tt * tt * dt + 1e-15 * v;
      const double w = u.Uniform();
      const double ax = fabs(x) + e;
      const double s = 1.0 - 0.0331 * x * x * x * x, ds = 4.0 * 0.0331 * ax * ax * ax * e + 1e-12;
      if (w < s - ds)
      {
         out = d * v;
         outErr = d * dv + 1e-12 * out;
         return true;
      }
      if (!(w >= s + ds))
         return false;
      // log w: w is a 24-bit value, exact in float, and logf is within 1 ulp (bounded here at 4). log v from logf of
      // v's float value (relative rounding 2^-24, so 6e-8 in the logarithm). The normal's error reaches the right side
      // through x^2 / 2 (at most (|x| + e) e) and through v (d (1 - v + log v) / dv = 1 / v - 1, bounded with slack).
      const double lw = static_cast<double>(logf(static_cast<float>(w)));
      const double lv = static_cast<double>(logf(static_cast<float>(v)));
      const double rhs = 0.5 * x * x + d * (1.0 - v + lv);
      const double m = 4.8e-7 * fabs(lw) + ax * e + d * ((fabs(1.0 / v - 1.0) + dv / v) * dv + 6e-8 + 4.8e-7 * fabs(lv)) +
                       1e-12 * (1.0 + d);
      if (lw < rhs - m)
      {
         out = d * v;
         outErr = d * dv + 1e-12 * out;
         return true;
      }
      if (!(lw > rhs + m))
         return false;
   }
   out = d;
   outErr = 0.0;
   return true;
}

} // namespace iscu
