// Blink schedules on the device (iscu_dye_blinks_dev): the world core's per-dye blink lists (core/src/dyes.cpp), one
// thread per dye, bit for bit the core's -- the same address-keyed pcg4d draws (DYE_CH channels) and the same float64
// arithmetic, with fdlibm's log / exp / cos (fdlibm.cuh) as the core's jsmath port has them.
//
//   dSTORM, PALM  LabelSchedule (dyes.cpp:440-478) -> DyeSchedule / DyeScheduleFrom (dyes.cpp:293-321): first
//                 activation after Exp(1) / activation rate (ACT), then per blink j on channels SCHED0 + 8 j + {ON,
//                 BRIGHT1, BRIGHT2, BLEACH, OFF}: ON for Exp(1) onSec, brightness log-normal with mean 1 and CV
//                 photonCV (Box-Muller), bleach with probability clamp(bleachProb, 0.01, 1), else dark for
//                 Exp(1) offSec; at most 1000 blinks. dSTORM starts its blinks after an initial ON of Exp(1)
//                 initialOnSec (INIT_ON). Under a kinetics history of two or more segments each state's
//                 unit-exponential draw is spent over the segments' rates (DyeScheduleHistory, dyes.cpp:333-425).
//   DNA-PAINT     PersistentBlinks (dyes.cpp:533-646): per 1 s bin a Poisson count (inverse CDF up to mean 30, the
//                 rounded normal beyond) of blinks at uniform starts, ON Exp(1) onSec capped at 20 onSec; the draws
//                 keyed by (site key, bin, j, purpose); a history splits a bin at segment starts into pieces with
//                 their own draws.
//   WideField     no blinks.
//
// A dye's rows are its blinks overlapping [t0, t1) in the order the core appends them; the bleaching schedules run to
// t1 + 1 s (the schedule up to a time does not depend on where it stops), then tOn < t1 and tOff > t0 select.
// Three launches: counts per dye, an exclusive scan, the rows.
#include "iscu_internal.h"
#include "counter_rng.cuh"
#include "fdlibm.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace iscu {
namespace {

constexpr int kMaxSegments = 64;
constexpr int kMaxBlinks = 1000;            // DYE_MAX_BLINKS
constexpr double kBinSec = 1.0;             // PERSIST_BIN_SEC
constexpr double kOnCap = 20.0;             // PERSIST_ON_CAP
constexpr double kPi = 3.141592653589793;   // jsm::PI
constexpr double kMaxWindowSec = 36000.0, kMaxTimeSec = 1e6, kMaxRate = 1e5, kMaxOnSec = 1000.0;

// DYE_CH channels (dyes.h:48-63)
constexpr uint32_t kChAct = 4, kChPersist = 5, kChInitOn = 7, kChSched0 = 16, kChSchedStride = 8;
constexpr uint32_t kChOn = 0, kChBright1 = 1, kChBright2 = 2, kChBleach = 3, kChOff = 4;

struct Kin
{
   double act, on, off, bleach, cv, initOn;
};

struct Params
{
   const iscu_dye* dyes;
   uint32_t nDyes;
   int32_t mode;
   Kin kin;                 // the label's kinetics, or the one segment's
   int32_t nSeg;            // >= 2: a history in tStart / segKin
   double t0, t1;
   const double* tStart;
   const Kin* segKin;
   uint32_t* counts;        // count pass: per dye
   const uint32_t* first;   // row pass: per dye's first row
   double* rows;
   uint32_t maxRows;
};

__device__ __forceinline__ double UnitOf(uint32_t a) { return (static_cast<double>(a >> 9) + 0.5) * 1.1920928955078125e-7; }

__device__ __forceinline__ uint32_t HashA(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
   Pcg4d(a, b, c, d);
   return a;
}

struct LogNormal
{
   double sigma, mu;
};

__device__ __forceinline__ LogNormal LogNormalFor(double cv)
{
   const double s2 = fd::Log(1.0 + cv * cv);
   return {sqrt(s2), -s2 / 2.0};
}

__device__ __forceinline__ double LogNormalMean1(const LogNormal& ln, double u1, double u2)
{
   const double z = sqrt(-2.0 * fd::Log(u1)) * fd::Cos(2.0 * kPi * u2);
   return fd::Exp(ln.mu + ln.sigma * z);
}

__device__ long PoissonInverse(double m, double expM, double u)
{
   double p = expM, F = p;
   long c = 0;
   while (u > F && c < 1000)
   {
      c++;
      p *= m / static_cast<double>(c);
      F += p;
   }
   return c;
}

__device__ long PoissonFromUniform(double m, double u, double u2)
{
   if (!(m > 0.0))
      return 0;
   if (m > 30.0)
   {
      const double z = sqrt(-2.0 * fd::Log(u)) * fd::Cos(2.0 * kPi * u2);
      const long v = static_cast<long>(floor(m + sqrt(m) * z + 0.5));
      return v > 0 ? v : 0;
   }
   return PoissonInverse(m, fd::Exp(-m), u);
}

// The rows of one dye: counted (rows == nullptr) or written from row `at`.
struct Sink
{
   const iscu_dye* d;
   double t0, t1;
   double* rows;
   uint32_t at, maxRows;
   uint32_t n = 0;
   __device__ void Blink(double tOn, double tOff, double brightness)
   {
      if (!(tOn < t1) || !(tOff > t0))
         return;
      const uint32_t r = at + n++;
      if (rows && r < maxRows)
      {
         double* o = rows + static_cast<size_t>(r) * ISCU_EVENT_STRIDE;
         o[0] = d->x;
         o[1] = d->y;
         o[2] = d->z;
         o[3] = tOn;
         o[4] = tOff;
         o[5] = brightness;
         o[6] = static_cast<double>(d->id);
         o[7] = static_cast<double>(d->structure);
         o[8] = 0.0;   // ISC_STATE_BLINK
         o[9] = 0.0;
      }
   }
};

// ---------------------------------------------------------------- history walks (dyes.cpp:333-380)
struct HazardWalk
{
   const Params& p;
   double t0;
   int i = 0;
   __device__ HazardWalk(const Params& pp, double t) : p(pp), t0(t) {}
   __device__ double End(int s) const { return s + 1 < p.nSeg ? p.tStart[s + 1] - t0 : INFINITY; }
   __device__ int Sync(double tau)
   {
      while (i + 1 < p.nSeg && p.tStart[i + 1] - t0 <= tau)
         i++;
      return i;
   }
   // rate: 0 activation
   __device__ double AfterRateAct(double tau, double E)
   {
      for (int s = Sync(tau);; s++)
      {
         const double a = p.segKin[s].act, end = End(s);
         if (a > 0.0)
         {
            const double t = tau + E / a;
            if (!(t >= end))
               return t;
            E = fmax(0.0, E - a * (end - tau));
         }
         else if (end == INFINITY)
         {
            return INFINITY;
         }
         tau = end;
      }
   }
   // scale: 0 onSec, 1 offSec, 2 initialOnSec
   __device__ double AfterScale(double tau, double E, int which)
   {
      for (int s = Sync(tau);; s++)
      {
         const Kin& q = p.segKin[s];
         const double sc = which == 0 ? q.on : which == 1 ? q.off : q.initOn, end = End(s);
         if (!(sc > 0.0))
            return tau;
         const double t = tau + E * sc;
         if (!(t >= end))
            return t;
         E = fmax(0.0, E - (end - tau) / sc);
         tau = end;
      }
   }
};

__device__ __forceinline__ int SegmentAt(const Params& p, double t)
{
   int lo = 0, hi = p.nSeg;
   while (hi - lo > 1)
   {
      const int mid = (lo + hi) / 2;
      if (p.tStart[mid] <= t)
         lo = mid;
      else
         hi = mid;
   }
   return lo;
}

// ---------------------------------------------------------------- bleaching schedules (dyes.cpp:293-425)
// DyeScheduleFrom with one set of kinetics; blinks shifted by `shift` (the dSTORM initial ON) before they are kept.
__device__ void ScheduleFrom(uint32_t h1, uint32_t k, uint32_t n, const Kin& kin, double t, double tMax, double shift,
                             Sink& out)
{
   const double pBleach = fmin(1.0, fmax(0.01, kin.bleach));
   const double cv = fmax(0.0, kin.cv);
   const LogNormal ln = LogNormalFor(cv);
   for (int j = 0; j < kMaxBlinks; j++)
   {
      if (t >= tMax)
         break;
      const uint32_t base = kChSched0 + static_cast<uint32_t>(j) * kChSchedStride;
      const double on = -fd::Log(UnitOf(HashA(h1, k, n, base + kChOn))) * kin.on;
      double b = 1.0;
      if (cv > 0.0)
      {
         const double u1 = UnitOf(HashA(h1, k, n, base + kChBright1));
         const double u2 = UnitOf(HashA(h1, k, n, base + kChBright2));
         b = LogNormalMean1(ln, u1, u2);
      }
      if (shift != 0.0)
         out.Blink(t + shift, (t + on) + shift, b);
      else
         out.Blink(t, t + on, b);
      if (UnitOf(HashA(h1, k, n, base + kChBleach)) < pBleach)
         break;
      t += on - fd::Log(UnitOf(HashA(h1, k, n, base + kChOff))) * kin.off;
   }
}

// DyeScheduleHistoryFrom in the dye's local time (absolute - t0 = shift).
__device__ void ScheduleHistoryFrom(const Params& p, uint32_t h1, uint32_t k, uint32_t n, double t0, double t,
                                    double tMax, Sink& out)
{
   HazardWalk w(p, t0);
   double lnCv = -1.0;
   LogNormal ln = {0.0, 0.0};
   for (int j = 0; j < kMaxBlinks; j++)
   {
      if (t >= tMax)
         break;
      const uint32_t base = kChSched0 + static_cast<uint32_t>(j) * kChSchedStride;
      const int seg = w.Sync(t);
      const Kin& q = p.segKin[seg];
      const double end = w.End(seg);
      const double eOn = -fd::Log(UnitOf(HashA(h1, k, n, base + kChOn)));
      const double on = eOn * q.on;
      double b = 1.0;
      const double cv = fmax(0.0, q.cv);
      if (cv > 0.0)
      {
         if (cv != lnCv)
         {
            ln = LogNormalFor(cv);
            lnCv = cv;
         }
         const double u1 = UnitOf(HashA(h1, k, n, base + kChBright1));
         const double u2 = UnitOf(HashA(h1, k, n, base + kChBright2));
         b = LogNormalMean1(ln, u1, u2);
      }
      const bool onInSeg = !(t + on >= end);
      const double tOff = onInSeg ? t + on : w.AfterScale(t, eOn, 0);
      if (t0 != 0.0)
         out.Blink(t + t0, tOff + t0, b);
      else
         out.Blink(t, tOff, b);
      const double pBleach = fmin(1.0, fmax(0.01, p.segKin[w.Sync(tOff)].bleach));
      if (UnitOf(HashA(h1, k, n, base + kChBleach)) < pBleach)
         break;
      const double eOff = -fd::Log(UnitOf(HashA(h1, k, n, base + kChOff)));
      const double off = eOff * q.off;
      if (onInSeg && !(t + (on + off) >= end))
         t += on + off;
      else
         t = w.AfterScale(tOff, eOff, 1);
   }
}

// LabelSchedule's blinks (dyes.cpp:440-478) for dSTORM and PALM, run to tMax (absolute).
__device__ void LabelBlinks(const Params& p, uint32_t h1, uint32_t k, uint32_t n, double tMax, Sink& out)
{
   const bool multi = p.nSeg >= 2;
   const Kin& kin = p.kin;
   double shift = 0.0;
   if (p.mode == ISCU_LABEL_DSTORM)
   {
      if (!multi && kin.initOn > 0.0)
         shift = -fd::Log(UnitOf(HashA(h1, k, n, kChInitOn))) * kin.initOn;
      else if (multi && p.segKin[0].initOn > 0.0)
         shift = HazardWalk(p, 0.0).AfterScale(0.0, -fd::Log(UnitOf(HashA(h1, k, n, kChInitOn))), 2);
   }
   if (multi)
   {
      const double t = HazardWalk(p, shift).AfterRateAct(0.0, -fd::Log(UnitOf(HashA(h1, k, n, kChAct))));
      ScheduleHistoryFrom(p, h1, k, n, shift, t, tMax - shift, out);
   }
   else if (kin.act > 0.0)
   {
      const double t = -fd::Log(UnitOf(HashA(h1, k, n, kChAct))) / kin.act;
      ScheduleFrom(h1, k, n, kin, t, tMax - shift, shift, out);
   }
}

// ---------------------------------------------------------------- persistent sites (dyes.cpp:533-646)
struct BinKin
{
   double rate, onSec, cv, maxOn, m, expM;
   bool small;
   LogNormal ln;
};

__device__ BinKin BinKinOf(const Kin& q)
{
   BinKin b;
   b.rate = q.act;
   b.onSec = q.on;
   b.cv = fmax(0.0, q.cv);
   b.ln = LogNormalFor(b.cv);
   b.maxOn = kOnCap * q.on;
   b.m = b.rate * kBinSec;
   b.small = b.m <= 30.0;
   b.expM = b.small ? fd::Exp(-b.m) : 0.0;
   return b;
}

// the blinks of one piece of a bin: c starts in [lo, hi) (piece 0: (bin + u) x 1 s), channels o + purpose
__device__ void Piece(uint32_t key, uint32_t bin, long c, const BinKin& q, uint32_t o, double lo, double hi, Sink& out)
{
   for (long j = 0; j < c; j++)
   {
      const uint32_t jj = static_cast<uint32_t>(j);
      const double u = UnitOf(HashA(key, bin, jj, o + 2));
      const double tOn = o == 0 ? (static_cast<double>(bin) + u) * kBinSec : lo + u * (hi - lo);
      if (!(tOn < hi))
         continue;
      const double on = fmin(q.maxOn, -fd::Log(UnitOf(HashA(key, bin, jj, o + 3))) * q.onSec);
      if (!(tOn < out.t1 && tOn + on > out.t0))   // PersistentBlinks' keep, before the brightness draws
         continue;
      double br = 1.0;
      if (q.cv > 0.0)
      {
         const double u1 = UnitOf(HashA(key, bin, jj, o + 4));
         const double u2 = UnitOf(HashA(key, bin, jj, o + 5));
         br = LogNormalMean1(q.ln, u1, u2);
      }
      out.Blink(tOn, tOn + on, br);
   }
}

__device__ void PersistentBlinks(const Params& p, uint32_t h1, uint32_t k, uint32_t n, Sink& out)
{
   const double t0 = p.t0, t1 = p.t1;
   if (!(t1 > t0))
      return;
   const bool multi = p.nSeg >= 2;
   double maxOn = 0.0;
   if (p.nSeg == 0)
      maxOn = kOnCap * p.kin.on;
   else
      for (int s = 0; s < p.nSeg; ++s)
         maxOn = fmax(maxOn, kOnCap * p.segKin[s].on);
   const long b0 = max(0L, static_cast<long>(floor((t0 - maxOn) / kBinSec)));
   const long b1 = static_cast<long>(floor(t1 / kBinSec));
   if (!multi && !(p.kin.act > 0.0))
      return;
   const uint32_t key = HashA(h1, k, n, kChPersist);
   int seg = multi ? SegmentAt(p, static_cast<double>(b0) * kBinSec) : 0;
   BinKin q0 = BinKinOf(multi ? p.segKin[seg] : p.kin);
   for (long b = b0; b <= b1; b++)
   {
      const uint32_t bin = static_cast<uint32_t>(b);
      const double binEnd = static_cast<double>(b + 1) * kBinSec;
      double pEnd = INFINITY;
      if (multi)
      {
         const int s = SegmentAt(p, static_cast<double>(b) * kBinSec);
         if (s != seg)
         {
            seg = s;
            q0 = BinKinOf(p.segKin[s]);
         }
         if (s + 1 < p.nSeg && p.tStart[s + 1] < binEnd)
            pEnd = p.tStart[s + 1];
      }
      if (q0.rate > 0.0)
      {
         const long c = q0.small ? PoissonInverse(q0.m, q0.expM, UnitOf(HashA(key, bin, 0u, 0u)))
                                 : PoissonFromUniform(q0.m, UnitOf(HashA(key, bin, 0u, 0u)),
                                                      UnitOf(HashA(key, bin, 0u, 1u)));
         Piece(key, bin, c, q0, 0u, static_cast<double>(b) * kBinSec, pEnd, out);
      }
      if (!(pEnd < binEnd))
         continue;
      uint32_t i = 1;
      for (int s = seg + 1; s < p.nSeg && p.tStart[s] < binEnd; s++, i++)
      {
         const double a = p.tStart[s];
         const double e = s + 1 < p.nSeg && p.tStart[s + 1] < binEnd ? p.tStart[s + 1] : binEnd;
         const BinKin q = BinKinOf(p.segKin[s]);
         if (!(e > a) || !(q.rate > 0.0))
            continue;
         const double m = q.rate * (e - a);
         const uint32_t o = 8u * i;
         const long c = m <= 30.0 ? PoissonInverse(m, fd::Exp(-m), UnitOf(HashA(key, bin, 0u, o)))
                                  : PoissonFromUniform(m, UnitOf(HashA(key, bin, 0u, o)),
                                                       UnitOf(HashA(key, bin, 0u, o + 1u)));
         Piece(key, bin, c, q, o, a, e, out);
      }
   }
}

__device__ void DyeRows(const Params& p, uint32_t dye, Sink& out)
{
   const iscu_dye& d = p.dyes[dye];
   const uint32_t k = static_cast<uint32_t>(d.k), n = static_cast<uint32_t>(d.n);
   if (p.mode == ISCU_LABEL_DNA_PAINT)
      PersistentBlinks(p, d.h1, k, n, out);
   else if (p.mode == ISCU_LABEL_DSTORM || p.mode == ISCU_LABEL_PALM)
      LabelBlinks(p, d.h1, k, n, p.t1 + 1.0, out);
}

__global__ void __launch_bounds__(128) CountKernel(Params p)
{
   const uint32_t dye = blockIdx.x * blockDim.x + threadIdx.x;
   if (dye >= p.nDyes)
      return;
   Sink s{&p.dyes[dye], p.t0, p.t1, nullptr, 0u, 0u};
   DyeRows(p, dye, s);
   p.counts[dye] = s.n;
}

__global__ void __launch_bounds__(128) RowsKernel(Params p)
{
   const uint32_t dye = blockIdx.x * blockDim.x + threadIdx.x;
   if (dye >= p.nDyes)
      return;
   Sink s{&p.dyes[dye], p.t0, p.t1, p.rows, p.first[dye], p.maxRows};
   DyeRows(p, dye, s);
}

// Exclusive scan of n counts into first[0..n] (first[n] = the total, and *total) in three launches: the sums of
// blocks of kScanItems counts, their exclusive scan by one CTA, and each block's scan from its offset.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanItems = kScanThreads * kScanPer;

// Inclusive scan of x across the CTA (warp scans, then the warps' totals); the CTA's total in *blockTotal.
__device__ __forceinline__ uint32_t CtaInclusiveScan(uint32_t x, uint32_t* warpSums, uint32_t* blockTotal)
{
   const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   for (int o = 1; o < 32; o <<= 1)
   {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= static_cast<uint32_t>(o))
         x += y;
   }
   if (lane == 31)
      warpSums[warp] = x;
   __syncthreads();
   if (warp == 0)
   {
      uint32_t w = lane < (blockDim.x >> 5) ? warpSums[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1)
      {
         const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
         if (lane >= static_cast<uint32_t>(o))
            w += y;
      }
      warpSums[lane] = w;   // inclusive over warps
      if (lane == 31)
         *blockTotal = w;
   }
   __syncthreads();
   return x + (warp ? warpSums[warp - 1] : 0u);
}

__global__ void __launch_bounds__(kScanThreads) ScanSumsKernel(const uint32_t* __restrict__ counts, uint32_t n,
                                                               uint32_t* __restrict__ sums)
{
   __shared__ uint32_t warpSums[32];
   const size_t i0 = static_cast<size_t>(blockIdx.x) * kScanItems + static_cast<size_t>(threadIdx.x) * kScanPer;
   uint32_t x = 0;
#pragma unroll
   for (int k = 0; k < kScanPer; ++k)
      if (i0 + k < n)
         x += counts[i0 + k];
   for (int o = 16; o; o >>= 1)
      x += __shfl_down_sync(0xffffffffu, x, o);
   if ((threadIdx.x & 31) == 0)
      warpSums[threadIdx.x >> 5] = x;
   __syncthreads();
   if (threadIdx.x == 0)
   {
      uint32_t t = 0;
      for (int w = 0; w < kScanThreads / 32; ++w)
         t += warpSums[w];
      sums[blockIdx.x] = t;
   }
}

// The block sums' exclusive scan in place (nb of them), the total into first[n] and *total.
__global__ void __launch_bounds__(kScanThreads) ScanOffsetsKernel(uint32_t* __restrict__ sums, uint32_t nb,
                                                                  uint32_t* __restrict__ first, uint32_t n,
                                                                  uint32_t* __restrict__ total)
{
   __shared__ uint32_t warpSums[32];
   __shared__ uint32_t chunkTotal;
   uint32_t carry = 0;
   for (uint32_t base = 0; base < nb; base += kScanThreads)
   {
      const uint32_t i = base + threadIdx.x;
      const uint32_t v = i < nb ? sums[i] : 0u;
      const uint32_t inc = CtaInclusiveScan(v, warpSums, &chunkTotal);
      if (i < nb)
         sums[i] = carry + inc - v;
      carry += chunkTotal;
      __syncthreads();   // warpSums and chunkTotal are rewritten by the next chunk
   }
   if (threadIdx.x == 0)
   {
      first[n] = carry;
      *total = carry;
   }
}

__global__ void __launch_bounds__(kScanThreads) ScanWriteKernel(const uint32_t* __restrict__ counts, uint32_t n,
                                                                const uint32_t* __restrict__ offsets,
                                                                uint32_t* __restrict__ first)
{
   __shared__ uint32_t warpSums[32];
   __shared__ uint32_t blockTotal;
   const size_t i0 = static_cast<size_t>(blockIdx.x) * kScanItems + static_cast<size_t>(threadIdx.x) * kScanPer;
   uint32_t v[kScanPer], x = 0;
#pragma unroll
   for (int k = 0; k < kScanPer; ++k)
   {
      v[k] = i0 + k < n ? counts[i0 + k] : 0u;
      x += v[k];
   }
   uint32_t at = offsets[blockIdx.x] + CtaInclusiveScan(x, warpSums, &blockTotal) - x;
#pragma unroll
   for (int k = 0; k < kScanPer; ++k)
      if (i0 + k < n)
      {
         first[i0 + k] = at;
         at += v[k];
      }
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" int iscu_dye_blinks_dev(iscu_ctx* ctx, const iscu_label* label, const double* hist_t_start,
                                   const iscu_kinetics* hist_kin, uint32_t n_seg, const iscu_dye* dyes_dev,
                                   uint32_t n_dyes, double t0, double t1, double* rows_dev, uint32_t max_rows,
                                   uint32_t* dye_first_dev, uint32_t* n_rows_dev)
{
   if (!ctx || !label || !n_rows_dev || (n_dyes && !dyes_dev) || (max_rows && !rows_dev) ||
       (n_seg && (!hist_t_start || !hist_kin)))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (label->mode < ISCU_LABEL_DSTORM || label->mode > ISCU_LABEL_WIDEFIELD)
      return Fail(ISCU_ERR_ARG, "label mode is not one of dSTORM, PALM, DNA-PAINT, WideField");
   if (n_seg > static_cast<uint32_t>(kMaxSegments))
      return Fail(ISCU_ERR_LIMIT, "at most 64 history segments");
   // bounds on the per-dye loops: bins of the window (DNA-PAINT), blinks per bin, the ON lookback
   if (!(std::isfinite(t0) && std::isfinite(t1)) || t1 - t0 > kMaxWindowSec || t1 > kMaxTimeSec)
      return Fail(ISCU_ERR_LIMIT, "the window must be finite, at most 36000 s long and end by 1e6 s");
   auto kinOk = [](const iscu_kinetics& q) {
      return !(q.activation_rate_per_sec > kMaxRate) && !(q.on_sec > kMaxOnSec) && !std::isnan(q.activation_rate_per_sec) &&
             !std::isnan(q.on_sec);
   };
   if (!kinOk(label->kin))
      return Fail(ISCU_ERR_LIMIT, "rates at most 1e5 per s, ON times at most 1000 s");
   for (uint32_t q = 0; q < n_seg; ++q)
      if (!kinOk(hist_kin[q]))
         return Fail(ISCU_ERR_LIMIT, "rates at most 1e5 per s, ON times at most 1000 s");
   if (n_seg && hist_t_start[0] != 0.0)
      return Fail(ISCU_ERR_ARG, "a history's first segment starts at 0");
   for (uint32_t s = 1; s < n_seg; ++s)
      if (!(hist_t_start[s] > hist_t_start[s - 1]))
         return Fail(ISCU_ERR_ARG, "history segment starts must increase");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   cudaStream_t s = ctx->stream;
   Params p{};
   p.dyes = dyes_dev;
   p.nDyes = n_dyes;
   p.mode = label->mode;
   const iscu_kinetics& lk = n_seg == 1 ? hist_kin[0] : label->kin;
   p.kin = {lk.activation_rate_per_sec, lk.on_sec, lk.off_sec, lk.bleach_prob, lk.photon_cv, lk.initial_on_sec};
   p.nSeg = n_seg >= 2 ? static_cast<int32_t>(n_seg) : (n_seg == 1 ? 1 : 0);
   p.t0 = t0;
   p.t1 = t1;
   // staging: history (start times, kinetics), per-dye counts, first rows
   const size_t histB = static_cast<size_t>(n_seg) * (sizeof(double) + sizeof(Kin));
   const size_t cntB = static_cast<size_t>(n_dyes) * sizeof(uint32_t);
   const size_t firstB = (static_cast<size_t>(n_dyes) + 1) * sizeof(uint32_t);
   const size_t sumsB = ((static_cast<size_t>(n_dyes) + kScanItems - 1) / kScanItems) * sizeof(uint32_t);
   ISCU_CK(ctx->dSchedule.Reserve(histB + cntB + (dye_first_dev ? 0 : firstB) + sumsB + 64));
   char* b = ctx->dSchedule.as<char>();
   double* dStart = reinterpret_cast<double*>(b);
   Kin* dKin = reinterpret_cast<Kin*>(b + static_cast<size_t>(n_seg) * sizeof(double));
   uint32_t* dCounts = reinterpret_cast<uint32_t*>(b + ((histB + 15) & ~size_t(15)));
   uint32_t* dFirst = dye_first_dev ? dye_first_dev : dCounts + n_dyes;
   uint32_t* dSums = dCounts + n_dyes + (dye_first_dev ? 0 : static_cast<size_t>(n_dyes) + 1);
   if (n_seg)
   {
      std::vector<Kin> kin(n_seg);
      for (uint32_t k = 0; k < n_seg; ++k)
         kin[k] = {hist_kin[k].activation_rate_per_sec, hist_kin[k].on_sec, hist_kin[k].off_sec,
                   hist_kin[k].bleach_prob, hist_kin[k].photon_cv, hist_kin[k].initial_on_sec};
      ISCU_CK(cudaMemcpyAsync(dStart, hist_t_start, n_seg * sizeof(double), cudaMemcpyHostToDevice, s));
      ISCU_CK(cudaMemcpyAsync(dKin, kin.data(), n_seg * sizeof(Kin), cudaMemcpyHostToDevice, s));
      ISCU_CK(cudaStreamSynchronize(s));   // (the host vector goes out of scope)
   }
   p.tStart = dStart;
   p.segKin = dKin;
   p.counts = dCounts;
   p.first = dFirst;
   p.rows = rows_dev;
   p.maxRows = max_rows;
   if (n_dyes == 0)
   {
      ISCU_CK(cudaMemsetAsync(n_rows_dev, 0, sizeof(uint32_t), s));
      if (dye_first_dev)
         ISCU_CK(cudaMemsetAsync(dye_first_dev, 0, sizeof(uint32_t), s));
      return ISCU_OK;
   }
   const unsigned blocks = (n_dyes + 127) / 128;
   CountKernel<<<blocks, 128, 0, s>>>(p);
   ISCU_CK_LAUNCH(ctx, "CountKernel");
   const uint32_t scanBlocks = static_cast<uint32_t>((static_cast<size_t>(n_dyes) + kScanItems - 1) / kScanItems);
   ScanSumsKernel<<<scanBlocks, kScanThreads, 0, s>>>(dCounts, n_dyes, dSums);
   ISCU_CK_LAUNCH(ctx, "ScanSumsKernel");
   ScanOffsetsKernel<<<1, kScanThreads, 0, s>>>(dSums, scanBlocks, dFirst, n_dyes, n_rows_dev);
   ISCU_CK_LAUNCH(ctx, "ScanOffsetsKernel");
   ScanWriteKernel<<<scanBlocks, kScanThreads, 0, s>>>(dCounts, n_dyes, dSums, dFirst);
   ISCU_CK_LAUNCH(ctx, "ScanWriteKernel");
   if (max_rows)
   {
      RowsKernel<<<blocks, 128, 0, s>>>(p);
      ISCU_CK_LAUNCH(ctx, "RowsKernel");
   }
   return ISCU_OK;
}
