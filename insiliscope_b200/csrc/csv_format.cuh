// The ground-truth tables' numbers (sim::AppendCsvNumber, adapter/inSiliScope/Simulation/CsvNumber.cpp:13-32):
// printf's "%.<p>f" / "%.<p>g" of a double in the "C" locale, at most 47 characters, nothing for NaN and infinities.
//
// printf converts the double's exact binary value and rounds the exact decimal expansion half to even. Restated
// here from that definition, for host and device alike: |x| = m 2^e exactly (m < 2^53); its integer part's decimal
// digits come from a big integer divided by 10^9 repeatedly, its fraction's digits one at a time by multiplying the
// fraction (a k-bit big integer, k = -e) by 10 and taking the bits above k; the digit string is rounded at the
// precision half to even, "sticky" meaning any nonzero digit past the next one; then the layout:
//   %.pf  [-]integer digits, and "." with p fraction digits when p > 0;
//   %.Pg  (P = 0 read as 1) with X the decimal exponent after rounding to P significant digits: exponential
//         d[.ddd]e+XX (at least two exponent digits) when X < -4 or X >= P, else fixed with P - 1 - X decimals;
//         trailing fraction zeros removed, and the "." when none remain; zero is "0" (or "-0").
// The sign is the sign bit's ("-0.000000", and "-0.0000" for a negative value that rounds to zero).
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#endif
#endif

namespace iscu {
namespace csv {

constexpr int kFieldMax = 47;   // characters kept (a printf into 48 bytes)
constexpr int kLimbs = 36;      // 1152 bits: 2^1024 for the integer part, 1074 + 4 bits for the fraction

// A little-endian big integer of 32-bit limbs; n limbs in use.
struct Big
{
   uint32_t w[kLimbs];
   int n;
};

__host__ __device__ inline uint32_t DivSmall(Big& b, uint32_t d)   // b /= d, returns the remainder
{
   uint64_t r = 0;
   for (int i = b.n - 1; i >= 0; --i)
   {
      const uint64_t t = (r << 32) | b.w[i];
      b.w[i] = static_cast<uint32_t>(t / d);
      r = t % d;
   }
   while (b.n > 0 && b.w[b.n - 1] == 0)
      --b.n;
   return static_cast<uint32_t>(r);
}

// The fraction f / 2^k (k bits; limbs 0 .. (k >> 5) + 1 in use): one decimal digit out.
__host__ __device__ inline int NextFractionDigit(Big& f, int k)
{
   const int top = (k >> 5) + 1;
   uint64_t carry = 0;
   for (int i = 0; i <= top; ++i)
   {
      const uint64_t t = static_cast<uint64_t>(f.w[i]) * 10u + carry;
      f.w[i] = static_cast<uint32_t>(t);
      carry = t >> 32;
   }
   const int li = k >> 5, bi = k & 31;
   uint32_t d;
   if (bi == 0)
   {
      d = f.w[li];
      f.w[li] = 0;
   }
   else
   {
      d = (f.w[li] >> bi) | (f.w[li + 1] << (32 - bi));
      f.w[li] &= (1u << bi) - 1u;
      f.w[li + 1] = 0;
   }
   return static_cast<int>(d & 15u);
}

__host__ __device__ inline bool Nonzero(const Big& f, int k)
{
   for (int i = 0; i <= (k >> 5) + 1; ++i)
      if (f.w[i])
         return true;
   return false;
}

// The exact decimal expansion of |x| = m 2^e: integer digits (most significant first) and a fraction digit source.
struct Expansion
{
   char ip[320];   // the integer part's digits ("0" when it is zero)
   int nip;
   bool ipZero;
   Big frac;
   int k;          // fraction bits (0: no fraction)

   __host__ __device__ int Next() { return k > 0 ? NextFractionDigit(frac, k) : 0; }
   __host__ __device__ bool FracNonzero() const { return k > 0 && Nonzero(frac, k); }
};

__host__ __device__ inline void Expand(uint64_t m, int e, Expansion& x)
{
   Big ib;
   ib.n = 0;
   for (int i = 0; i < kLimbs; ++i)
   {
      ib.w[i] = 0;
      x.frac.w[i] = 0;
   }
   x.k = 0;
   if (e >= 0)
   {
      // integer m 2^e: limbs of m shifted left by e bits
      const int ls = e >> 5, bs = e & 31;
      const uint32_t lo = static_cast<uint32_t>(m), hi = static_cast<uint32_t>(m >> 32);
      if (bs == 0)
      {
         ib.w[ls] = lo;
         ib.w[ls + 1] = hi;
      }
      else
      {
         ib.w[ls] = lo << bs;
         ib.w[ls + 1] = (lo >> (32 - bs)) | (hi << bs);
         ib.w[ls + 2] = hi >> (32 - bs);
      }
      ib.n = ls + 3;
   }
   else
   {
      const int k = -e;
      const uint64_t ipart = k >= 64 ? 0 : (m >> k);
      const uint64_t f = k >= 64 ? m : (m & ((uint64_t(1) << k) - 1));
      ib.w[0] = static_cast<uint32_t>(ipart);
      ib.w[1] = static_cast<uint32_t>(ipart >> 32);
      ib.n = 2;
      x.k = k;
      x.frac.w[0] = static_cast<uint32_t>(f);
      x.frac.w[1] = static_cast<uint32_t>(f >> 32);
      x.frac.n = (k >> 5) + 2;
   }
   while (ib.n > 0 && ib.w[ib.n - 1] == 0)
      --ib.n;
   // integer digits, nine at a time from the least significant end
   char rev[320];
   int nr = 0;
   while (ib.n > 0)
   {
      uint32_t r = DivSmall(ib, 1000000000u);
      const bool last = ib.n == 0;
      for (int j = 0; j < 9 && (!last || r); ++j)
      {
         rev[nr++] = static_cast<char>('0' + r % 10);
         r /= 10;
      }
   }
   x.ipZero = nr == 0;
   if (x.ipZero)
      rev[nr++] = '0';
   x.nip = nr;
   for (int i = 0; i < nr; ++i)
      x.ip[i] = rev[nr - 1 - i];
}

// The same expansion when the integer part and the fraction both fit 64 bits (|x| < 2^64 with at most 60 fraction
// bits: every value the tables hold but the tiny ones); the fraction's digits as f * 10, shifted, in one word.
struct SmallExpansion
{
   char ip[20];
   int nip;
   bool ipZero;
   uint64_t f;
   int k;

   __host__ __device__ int Next()
   {
      if (k == 0)
         return 0;
      f *= 10u;   // f < 2^60: no overflow
      const int d = static_cast<int>(f >> k);
      f &= (uint64_t(1) << k) - 1u;
      return d;
   }
   __host__ __device__ bool FracNonzero() const { return k > 0 && f != 0; }
};

// m 2^e fits SmallExpansion: e >= 0 with m 2^e < 2^64, or -60 <= e < 0.
__host__ __device__ inline bool FitsSmall(uint64_t m, int e)
{
   if (e < 0)
      return e >= -60;
   return e < 64 && (e == 0 || (m >> (64 - e)) == 0);
}

__host__ __device__ inline void ExpandSmall(uint64_t m, int e, SmallExpansion& x)
{
   uint64_t ipart;
   if (e >= 0)
   {
      ipart = m << e;
      x.k = 0;
      x.f = 0;
   }
   else
   {
      x.k = -e;
      ipart = m >> x.k;
      x.f = m & ((uint64_t(1) << x.k) - 1u);
   }
   char rev[20];
   int nr = 0;
   while (ipart)
   {
      rev[nr++] = static_cast<char>('0' + ipart % 10u);
      ipart /= 10u;
   }
   x.ipZero = nr == 0;
   if (x.ipZero)
      rev[nr++] = '0';
   x.nip = nr;
   for (int i = 0; i < nr; ++i)
      x.ip[i] = rev[nr - 1 - i];
}

// Adds one unit in the last place of the n digits d (ASCII); true when they all carried (999 -> 000).
__host__ __device__ inline bool Increment(char* d, int n)
{
   for (int i = n - 1; i >= 0; --i)
   {
      if (d[i] == '9')
         d[i] = '0';
      else
      {
         ++d[i];
         return false;
      }
   }
   return true;
}

// The layout of printf's conversion from the value's digits: the sign, then %.pf or %.Pg (kMaxOut characters of
// conversion, kMaxDigits digits of %.pf at most for this expansion).
template <int kMaxOut, int kMaxDigits, class Exp>
__host__ __device__ inline int Layout(bool neg, uint64_t m, Exp& x, char kind, int prec, char* out)
{
   char s[kMaxOut];   // the whole conversion, then its first 47 characters
   int n = 0;
   if (neg)
      s[n++] = '-';
   if (kind == 'f')
   {
      char d[kMaxDigits];   // integer digits, then prec fraction digits
      int nd = 0;
      for (int i = 0; i < x.nip; ++i)
         d[nd++] = x.ip[i];
      for (int i = 0; i < prec; ++i)
         d[nd++] = static_cast<char>('0' + x.Next());
      const int r = x.Next();
      const bool sticky = x.FracNonzero();
      const bool odd = (d[nd - 1] - '0') & 1;
      bool lead = false;
      if (r > 5 || (r == 5 && (sticky || odd)))
         lead = Increment(d, nd);
      if (lead)
         s[n++] = '1';
      for (int i = 0; i < nd - prec; ++i)
         s[n++] = d[i];
      if (prec > 0)
      {
         s[n++] = '.';
         for (int i = nd - prec; i < nd; ++i)
            s[n++] = d[i];
      }
   }
   else
   {
      const int P = prec == 0 ? 1 : prec;
      char d[12];
      int X;
      if (m == 0)
      {
         for (int i = 0; i < P; ++i)
            d[i] = '0';
         X = 0;
      }
      else
      {
         // the significant digits: from the integer part, or after the fraction's leading zeros
         int nd = 0, r;
         bool sticky = false;
         if (!x.ipZero)
         {
            X = x.nip - 1;
            int i = 0;
            for (; i < x.nip && nd < P; ++i)
               d[nd++] = x.ip[i];
            while (nd < P)
               d[nd++] = static_cast<char>('0' + x.Next());
            if (i < x.nip)
            {
               r = x.ip[i++] - '0';
               for (; i < x.nip; ++i)
                  sticky = sticky || x.ip[i] != '0';
               sticky = sticky || x.FracNonzero();
            }
            else
            {
               r = x.Next();
               sticky = x.FracNonzero();
            }
         }
         else
         {
            int z = 0, dig;
            while ((dig = x.Next()) == 0)
               ++z;
            X = -(z + 1);
            d[nd++] = static_cast<char>('0' + dig);
            while (nd < P)
               d[nd++] = static_cast<char>('0' + x.Next());
            r = x.Next();
            sticky = x.FracNonzero();
         }
         const bool odd = (d[P - 1] - '0') & 1;
         if (r > 5 || (r == 5 && (sticky || odd)))
            if (Increment(d, P))
            {
               d[0] = '1';   // 999 -> 1000: one more decade
               ++X;
            }
      }
      int last = P - 1;   // trailing zeros go
      if (X < -4 || X >= P)
      {
         while (last > 0 && d[last] == '0')
            --last;
         s[n++] = d[0];
         if (last > 0)
         {
            s[n++] = '.';
            for (int i = 1; i <= last; ++i)
               s[n++] = d[i];
         }
         s[n++] = 'e';
         s[n++] = X < 0 ? '-' : '+';
         int a = X < 0 ? -X : X;
         char ed[4];
         int ne = 0;
         do
         {
            ed[ne++] = static_cast<char>('0' + a % 10);
            a /= 10;
         } while (a);
         if (ne < 2)
            ed[ne++] = '0';
         while (ne)
            s[n++] = ed[--ne];
      }
      else
      {
         // fixed, P - 1 - X decimals; digits d[0..P-1] with the point after d[X] (X >= 0) or leading zeros
         const int minLast = X >= 0 ? X : -1;   // the last integer digit's index
         while (last > minLast && last >= 0 && d[last] == '0')
            --last;
         if (X >= 0)
         {
            for (int i = 0; i <= X; ++i)
               s[n++] = d[i];
            if (last > X)
            {
               s[n++] = '.';
               for (int i = X + 1; i <= last; ++i)
                  s[n++] = d[i];
            }
         }
         else
         {
            s[n++] = '0';
            s[n++] = '.';
            for (int i = 0; i < -X - 1; ++i)
               s[n++] = '0';
            for (int i = 0; i <= last; ++i)
               s[n++] = d[i];
         }
      }
   }
   const int len = n < kFieldMax ? n : kFieldMax;
   for (int i = 0; i < len; ++i)
      out[i] = s[i];
   return len;
}

// printf(fmt, v) as AppendCsvNumber keeps it: into out (>= 48 bytes), returns the length (0 for NaN / infinity).
// kind 'f' or 'g', prec 0..9.
__host__ __device__ inline int Format(double v, char kind, int prec, char* out)
{
   uint64_t bits;
   {
      union
      {
         double d;
         uint64_t u;
      } c;
      c.d = v;
      bits = c.u;
   }
   const bool neg = (bits >> 63) != 0;
   const int be = static_cast<int>((bits >> 52) & 0x7FF);
   const uint64_t frac = bits & ((uint64_t(1) << 52) - 1);
   if (be == 0x7FF)
      return 0;   // NaN, infinity: nothing
   uint64_t m;
   int e;
   if (be == 0)
   {
      m = frac;
      e = -1074;
   }
   else
   {
      m = frac | (uint64_t(1) << 52);
      e = be - 1075;
   }
   while (m && !(m & 1) && e < 0)   // fewer fraction bits, the same value
   {
      m >>= 1;
      ++e;
   }
   if (m == 0)
      e = 0;
   if (FitsSmall(m, e))
   {
      SmallExpansion x;
      ExpandSmall(m, e, x);
      return Layout<40, 32>(neg, m, x, kind, prec, out);
   }
   Expansion x;
   Expand(m, e, x);
   return Layout<360, 340>(neg, m, x, kind, prec, out);
}

} // namespace csv
} // namespace iscu
