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
      const double out = ne > 0.0 ? CounterGamma(ne, u) : 0.0;
      const double readE = (st.readNoise ? static_cast<double>(st.readNoise[i]) : cam.readNoise) / cam.emGain;
      const double gain = st.gain ? static_cast<double>(st.gain[i]) : cam.gain;
      const double offset = st.offset ? static_cast<double>(st.offset[i]) : 0.0;
      const double g = CounterGauss(u);
      const double adu = floor(offset + (out + readE * g) / gain + 0.5);
      return static_cast<uint16_t>(adu < 0.0 ? 0.0 : (adu > cam.maxAdu ? cam.maxAdu : adu));
   }
   const double ne = CounterPoisson(photons * cam.qe + cam.dark, u);
   const double readNoise = st.readNoise ? static_cast<double>(st.readNoise[i]) : cam.readNoise;
   const double gain = st.gain ? static_cast<double>(st.gain[i]) : cam.gain;
   const double offset = st.offset ? static_cast<double>(st.offset[i]) : 0.0;
   const double g = CounterGauss(u);
   double adu = offset + (ne + readNoise * g) / gain;
   adu = adu < 0.0 ? 0.0 : (adu > 65535.0 ? 65535.0 : adu);
   return static_cast<uint16_t>(floor(adu + 0.5));
}

} // namespace iscu
