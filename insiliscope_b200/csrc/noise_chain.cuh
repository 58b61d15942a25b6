// The per-pixel camera noise chain (ApplyNoiseChain, adapter/inSiliScope/Simulation/SMLMNoise.cpp:142-216) as a
// device function, shared by the kernels that end in camera frames (splat_noise.cu, widefield.cu). Every translation
// unit that includes it is compiled with --fmad=false, so its float64 arithmetic rounds as the reference's
// -ffp-contract=off build does.
#pragma once

#include "counter_rng.cuh"
#include "iscu_internal.h"

namespace iscu {

// Pixel i (of the frame; the sensor pixel is i + pixel_base) of a frame whose stream u is keyed by (seed, frame):
// sCMOS or EMCCD, per-pixel maps where set, else the camera scalars (offset 0).
__device__ __forceinline__ uint16_t NoisePixel(float photonValue, uint32_t i, const CameraView& cam,
                                               const StaticView& st, CounterRng& u)
{
   u.Pixel(i + st.pixelBase);
   const double pv = static_cast<double>(photonValue);
   const double photons = pv > 0.0 ? pv : 0.0;   // std::max(0.0, v)
   if (cam.emccd)
   {
      const double ne = CounterPoisson(photons * cam.qe + cam.dark + cam.cic, u);
      const double readE = (st.readNoise ? static_cast<double>(st.readNoise[i]) : cam.readNoise) / cam.emGain;
      const double gain = st.gain ? static_cast<double>(st.gain[i]) : cam.gain;
      const double offset = st.offset ? static_cast<double>(st.offset[i]) : 0.0;
      // The register's Gamma with float32 decisions (GammaSure), else CounterGamma from the saved stream; then the
      // rounding (before the clamp) from the float32 read-noise normal when no boundary is within the bound of both
      // float32 errors, else the Gamma (if it was not exact) and the normal again in float64 from the saved stream.
      const CounterRng saved = u;
      double out = 0.0, outErr = 0.0;
      bool exact = true;
      if (ne > 0.0)
      {
         exact = !GammaSure(ne, u, out, outErr);
         if (exact)
         {
            u = saved;
            out = CounterGamma(ne, u);
            outErr = 0.0;
         }
      }
      GaussDraw d = DrawGauss(u);
      const double af = offset + (out + readE * static_cast<double>(d.gf)) / gain;
      const double m = (outErr + fabs(readE) * kGaussFastErr) / fabs(gain) + 1e-9 * (1.0 + fabs(af));
      double adu;
      if (!RoundsSurely(af, m, adu))
      {
         if (!exact)
         {
            u = saved;
            out = CounterGamma(ne, u);
            d = DrawGauss(u);
         }
         adu = floor(offset + (out + readE * GaussExact(d)) / gain + 0.5);
      }
      return static_cast<uint16_t>(adu < 0.0 ? 0.0 : (adu > cam.maxAdu ? cam.maxAdu : adu));
   }
   const double ne = CounterPoisson(photons * cam.qe + cam.dark, u);
   const double readNoise = st.readNoise ? static_cast<double>(st.readNoise[i]) : cam.readNoise;
   const double gain = st.gain ? static_cast<double>(st.gain[i]) : cam.gain;
   const double offset = st.offset ? static_cast<double>(st.offset[i]) : 0.0;
   const GaussDraw d = DrawGauss(u);
   // The ADU from the float32 normal when it is sure: inside (0, 65535) and no rounding boundary within
   // |readNoise / gain| kGaussFastErr of it (the float64 operations' own rounding, ~1e-13, inside the 1e-9 term).
   const double af = offset + (ne + readNoise * static_cast<double>(d.gf)) / gain;
   const double m = fabs(readNoise / gain) * kGaussFastErr + 1e-9 * (1.0 + fabs(af));
   double r;
   if (af > m && af < 65535.0 - m && RoundsSurely(af, m, r))
      return static_cast<uint16_t>(r);
   const double g = GaussExact(d);
   double adu = offset + (ne + readNoise * g) / gain;
   adu = adu < 0.0 ? 0.0 : (adu > 65535.0 ? 65535.0 : adu);
   return static_cast<uint16_t>(floor(adu + 0.5));
}

} // namespace iscu
