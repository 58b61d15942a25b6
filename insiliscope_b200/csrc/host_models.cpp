// Host-side per-movie models around the path, restated from the reference (they run once per movie, on the host,
// as the reference runs them; built with -ffp-contract=off so they round as the reference's build does):
//  - the sample drift walker (adapter/inSiliScope/Simulation/Drift.cpp:24-124): a directed part whose xy direction
//    and xy / z strengths wander as unit Ornstein-Uhlenbeck processes, plus a per-frame random walk, every draw from
//    the counter stream of (DriftSeed(seed), frame);
//  - the illumination field (SMLMBackground.cpp:8-38) and the background fade (SMLMBackground.cpp:52-55).
//
// The counter stream (pcg4d, four uniforms per hash, Box-Muller) is restated here for the host
// (SMLMCounterRng.h:37-99); the device form is counter_rng.cuh.

#include "iscu_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace iscu {

namespace {

constexpr double kPi = 3.14159265358979323846;

void HostPcg4d(uint32_t v[4])
{
   for (int i = 0; i < 4; ++i)
      v[i] = v[i] * 1664525u + 1013904223u;
   v[0] += v[1] * v[3];
   v[1] += v[2] * v[0];
   v[2] += v[0] * v[1];
   v[3] += v[1] * v[2];
   for (int i = 0; i < 4; ++i)
      v[i] ^= v[i] >> 16;
   v[0] += v[1] * v[3];
   v[1] += v[2] * v[0];
   v[2] += v[0] * v[1];
   v[3] += v[1] * v[2];
}

struct HostCounterRng
{
   uint32_t seed, frame, pix = 0, ctr = 0, buf[4] = {0, 0, 0, 0};
   int k = 4;
   HostCounterRng(uint32_t s, uint32_t f) : seed(s), frame(f) {}
   void Pixel(uint32_t p)
   {
      pix = p;
      ctr = 0;
      k = 4;
   }
   double Uniform()
   {
      if (k == 4)
      {
         buf[0] = seed;
         buf[1] = frame;
         buf[2] = pix;
         buf[3] = ctr++;
         HostPcg4d(buf);
         k = 0;
      }
      return (static_cast<double>(buf[k++] >> 9) + 0.5) * (1.0 / 8388608.0);
   }
};

double HostGauss(HostCounterRng& u)
{
   const double r = std::sqrt(-2.0 * std::log(u.Uniform()));
   return r * std::cos(6.283185307179586 * u.Uniform());
}

uint32_t DriftSeedOf(int64_t randomSeed)
{
   return static_cast<uint32_t>(static_cast<uint64_t>(randomSeed) ^ 0x44524654ULL);   // "DRFT"
}

// erf(x / sqrt 2), Abramowitz & Stegun 7.1.26.
double DriftSwing(double x)
{
   const double z = std::fabs(x) / std::sqrt(2.0);
   const double t = 1.0 / (1.0 + 0.3275911 * z);
   const double poly = ((((1.061405429 * t - 1.453152027) * t + 1.421413741) * t - 0.284496736) * t + 0.254829592) * t;
   const double e = 1.0 - poly * std::exp(-z * z);
   return x < 0.0 ? -e : e;
}

} // namespace

} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_drift_trajectory(int64_t random_seed, int64_t frames, double frame_sec, const iscu_drift_settings* s,
                          double* xyz_nm)
{
   if (!s || (frames > 0 && !xyz_nm) || frames < 0)
      return Fail(ISCU_ERR_ARG, "null argument or negative frame count");
   ClearError();
   for (int64_t f = 0; f < frames; ++f)
      xyz_nm[3 * f] = xyz_nm[3 * f + 1] = xyz_nm[3 * f + 2] = 0.0;
   const bool on = s->xy_nm_per_sqrt_sec > 0.0 || s->z_nm_per_sqrt_sec > 0.0 || s->xy_speed_nm_per_sec != 0.0 ||
                   s->z_speed_nm_per_sec != 0.0;
   if (!on || frames <= 1)
      return ISCU_OK;
   // DriftWalker(randomSeed, s, 0)
   const uint32_t seed = DriftSeedOf(random_seed);
   HostCounterRng a(seed, 0xFFFFFFFFu);
   a.Pixel(2);
   const double theta0 = 2.0 * kPi * a.Uniform();
   const bool zUp = a.Uniform() < 0.5;
   HostCounterRng u0(seed, 0u);
   u0.Pixel(1);
   double phi = HostGauss(u0);
   double sxy = HostGauss(u0);
   double sz = HostGauss(u0);
   HostCounterRng v0(seed, 0u);
   v0.Pixel(3);
   double psi = HostGauss(v0);
   double dx = 0.0, dy = 0.0, dz = 0.0;
   for (int64_t f = 1; f < frames; ++f)
   {
      // Step(frameSec)
      const double dt = std::max(0.0, frame_sec);
      const double theta = (s->xy_angle_deg >= 0.0 ? s->xy_angle_deg * kPi / 180.0 : theta0) +
                           s->angle_wander_deg * kPi / 180.0 * DriftSwing(phi);
      const double w = s->speed_wander_pct / 100.0;
      const double vxy = s->xy_speed_nm_per_sec * std::max(0.0, 1.0 + w * sxy);
      const double up = s->z_direction > 0 ? 1.0 : s->z_direction < 0 ? -1.0 : (zUp ? 1.0 : -1.0);
      const double vz = up * s->z_speed_nm_per_sec * std::max(0.0, 1.0 + w * sz) *
                        std::cos(s->z_angle_wander_deg * kPi / 180.0 * DriftSwing(psi));
      const double vx = vxy * std::cos(theta), vy = vxy * std::sin(theta);
      // DriftStep(seed, f, frameSec): x, y, z in that order
      HostCounterRng st(seed, static_cast<uint32_t>(f));
      st.Pixel(0);
      const double gx = HostGauss(st);
      const double gy = HostGauss(st);
      const double gzs = HostGauss(st);
      const double r = std::sqrt(std::max(0.0, frame_sec));
      dx = dx + vx * dt + s->xy_nm_per_sqrt_sec * r * gx;
      dy = dy + vy * dt + s->xy_nm_per_sqrt_sec * r * gy;
      dz = dz + vz * dt + s->z_nm_per_sqrt_sec * r * gzs;
      // the wanders
      HostCounterRng u(seed, static_cast<uint32_t>(f));
      u.Pixel(1);
      const double gp = HostGauss(u);
      const double gs = HostGauss(u);
      const double gz = HostGauss(u);
      const double aa = s->wander_time_sec > 0.0 ? std::exp(-dt / s->wander_time_sec) : 0.0;
      const double bb = std::sqrt(std::max(0.0, 1.0 - aa * aa));
      phi = aa * phi + bb * gp;
      sxy = aa * sxy + bb * gs;
      sz = aa * sz + bb * gz;
      HostCounterRng v(seed, static_cast<uint32_t>(f));
      v.Pixel(3);
      psi = aa * psi + bb * HostGauss(v);
      xyz_nm[3 * f] = dx;
      xyz_nm[3 * f + 1] = dy;
      xyz_nm[3 * f + 2] = dz;
   }
   return ISCU_OK;
}

int iscu_illumination_field(uint32_t width, uint32_t height, int32_t profile, double fwhm_pct, float* out,
                            double* mean_factor)
{
   ClearError();
   if (mean_factor)
      *mean_factor = 1.0;
   if (profile < 0 || profile > 2)
      return Fail(ISCU_ERR_ARG, "profile: 0 flat, 1 Gaussian, 2 flat-top");
   if (profile == 0 || width == 0 || height == 0)
      return ISCU_OK;
   if (!out)
      return Fail(ISCU_ERR_ARG, "null output");
   const double cx = (width - 1) / 2.0, cy = (height - 1) / 2.0;
   const double fwhm = std::max(1e-6, (fwhm_pct / 100.0) * width);
   const double sig = fwhm / 2.3548, r0 = fwhm / 2.0, edge = std::max(1e-6, 0.15 * r0);
   double sum = 0.0, peak = 0.0;
   for (uint32_t y = 0; y < height; ++y)
      for (uint32_t x = 0; x < width; ++x)
      {
         const double r = std::hypot(x - cx, y - cy);
         const double v = profile == 1 ? std::exp(-(r * r) / (2.0 * sig * sig)) : 1.0 / (1.0 + std::exp((r - r0) / edge));
         out[static_cast<size_t>(y) * width + x] = static_cast<float>(v);
         sum += v;
         peak = std::max(peak, v);
      }
   if (!(peak > 0.0))
      return Fail(ISCU_ERR_ARG, "the field has no positive value");
   const size_t n = static_cast<size_t>(width) * height;
   for (size_t i = 0; i < n; ++i)
      out[i] = static_cast<float>(out[i] / peak);
   if (mean_factor)
      *mean_factor = sum / (static_cast<double>(width) * height) / peak;
   return ISCU_OK;
}

double iscu_background_fade_scale(double t, double decay)
{
   return decay > 0.0 ? 0.3 + 0.7 * std::exp(-t / decay) : 1.0;
}

} // extern "C"
