// TEST INFRASTRUCTURE -- the reference itself, as a checker and as the timed CPU baseline. Never part of the product.
//
// A C-ABI harness over inSiliScope's own C++ render engine, compiled together with the reference's source files
// where they lie (oracle/Makefile; output oracle/_ref/libiscref.so). It drives the hot-path functions directly with
// plain arrays, the way the reference's GPU self-check does (adapter/inSiliScope/Simulation/SplatGpu.cpp:464-540):
//   ComputeZernikePsfPlanes / BuildZernikePsfKernelCache (ZernikePsf.cpp:160, :382), block sums
//   (PsfGeneratorBridge.cpp:1069), WithHaloCut (:1186), RenderPhotonImage (SMLMSimulation.cpp:103),
//   CollectGpuEmitters (:219), ApplyNoiseChain (SMLMNoise.cpp:142), the camera maps (SMLMNoise.cpp:89-140), the
//   counter RNG (SMLMCounterRng.h, core/src/rng.h), and a movie loop shaped like FluorescenceMovie::Render's
//   (ScopeMovie.cpp:7267, :7649: frames in parallel on the reference's own thread pool, ParallelFor).
#include "BinnedBlinks.h"
#include "CsvNumber.h"
#include "Drift.h"
#include "WidefieldRender.h"
#include "PsfGeneratorBridge.h"
#include "SMLMBackground.h"
#include "Parallel.h"
#include "SMLMCounterRng.h"
#include "SMLMNoise.h"
#include "SMLMSimulation.h"
#include "SMLMZernike.h"
#include "ZernikePsf.h"
#include "dyes.h"
#include "rng.h"
#include "tiff_writer.h"

#include "../include/iscu.h"

#include <algorithm>
#include <charconv>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

std::string FullPrecisionZernike(const double* z)
{
   std::string s;
   char buf[64];
   for (int j = 0; j < 28; ++j)
   {
      std::snprintf(buf, sizeof(buf), "%s%.17g", j ? "," : "", z[j]);
      s += buf;
   }
   return s;
}

sim::PsfGeneratorRequest ToRequest(const iscu_psf_request& r)
{
   sim::PsfGeneratorRequest q;
   q.model = sim::PsfModelKind::GibsonLanniZernike;
   q.wavelengthNm = r.wavelength_nm;
   q.na = r.na;
   q.immersionIndex = r.immersion_index;
   q.sampleIndex = r.sample_index;
   q.workingDistanceUm = r.working_distance_um;
   q.sampleDepthNm = r.sample_depth_nm;
   q.pixelSizeNm = r.pixel_size_nm;
   q.zernikeCoefficients = FullPrecisionZernike(r.zernike);
   q.maskType = r.mask_double_helix ? sim::PsfMaskType::DoubleHelix : sim::PsfMaskType::None;
   q.maskModes = r.mask_modes;
   q.maskWaist = r.mask_waist;
   q.oversampling = r.oversampling;
   q.kernelHalfWidthPx = r.kernel_half_width_px;
   q.nz = r.nz;
   q.zStepNm = r.z_step_nm;
   q.pupilSamples = r.pupil_samples;
   q.interpMode = static_cast<sim::PsfInterpMode>(r.interp);
   return q;
}

sim::CameraNoiseParams ToCamera(const iscu_camera& c)
{
   sim::CameraNoiseParams p;
   p.quantumEfficiency = c.quantum_efficiency;
   p.darkCurrentElectrons = c.dark_electrons;
   p.gainPhotonsPerAdu = c.gain;
   p.readNoiseElectrons = c.read_noise_e;
   p.emccd = c.emccd != 0;
   p.bitDepth = c.bit_depth;
   p.emGain = c.em_gain;
   p.cicElectrons = c.cic_electrons;
   return p;
}

std::vector<sim::BlinkEvent> ToEvents(const iscu_blink_event* ev, uint32_t n)
{
   std::vector<sim::BlinkEvent> out(n);
   for (uint32_t i = 0; i < n; ++i)
   {
      out[i].xUm = ev[i].x_um;
      out[i].yUm = ev[i].y_um;
      out[i].zNm = ev[i].z_nm;
      out[i].tStart = ev[i].t_start;
      out[i].tEnd = ev[i].t_end;
      out[i].brightness = ev[i].brightness;
      out[i].excite = ev[i].excite;
   }
   return out;
}

struct Maps
{
   sim::PixelOffsetMap off;
   sim::PixelGainMap gain;
   sim::PixelReadNoiseMap rn;
};

void FillMaps(Maps& m, unsigned w, unsigned h, const float* off, const float* gain, const float* rn)
{
   const size_t n = static_cast<size_t>(w) * h;
   if (off)
   {
      m.off.width = w;
      m.off.height = h;
      m.off.offset.assign(off, off + n);
   }
   if (gain)
   {
      m.gain.width = w;
      m.gain.height = h;
      m.gain.gainPhotonsPerAdu.assign(gain, gain + n);
   }
   if (rn)
   {
      m.rn.width = w;
      m.rn.height = h;
      m.rn.readNoiseElectrons.assign(rn, rn + n);
   }
}

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void ref_set_threads(unsigned n) { sim::ParallelThreadCap().store(n); }
unsigned ref_threads(void) { return sim::HardwareThreads(); }

// ------------------------------------------------------------------------------------------- RNG
void ref_pcg4d(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t* out)
{
   sim::Pcg4d(a, b, c, d);
   out[0] = a;
   out[1] = b;
   out[2] = c;
   out[3] = d;
}

double ref_hash_unit(uint32_t seed, int32_t cx, int32_t cy, uint32_t k) { return isc::HashUnit(seed, cx, cy, k); }

void ref_hash_stream(uint32_t seed, int32_t cx, int32_t cy, uint32_t base, uint32_t n, double* out)
{
   isc::HashStream hs(seed, cx, cy, base);
   for (uint32_t i = 0; i < n; ++i)
      out[i] = hs.Next();
}

void ref_counter_uniforms(uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix, uint32_t per, double* out)
{
   sim::CounterRng u(seed, frame);
   for (uint32_t i = 0; i < npix; ++i)
   {
      u.Pixel(pixel0 + i);
      for (uint32_t j = 0; j < per; ++j)
         out[static_cast<size_t>(i) * per + j] = u.Uniform();
   }
}

double ref_counter_poisson(uint32_t seed, uint32_t frame, uint32_t pixel, double l)
{
   sim::CounterRng u(seed, frame);
   u.Pixel(pixel);
   return sim::CounterPoisson(l, u);
}

double ref_counter_gamma(uint32_t seed, uint32_t frame, uint32_t pixel, double k)
{
   sim::CounterRng u(seed, frame);
   u.Pixel(pixel);
   return sim::CounterGamma(k, u);
}

// ------------------------------------------------------------------------------------------- camera
void ref_camera_maps(uint32_t w, uint32_t h, uint64_t seed, double offMean, double offStd, double gainNom,
                     double gainFrac, double rnNom, double rnFrac, uint32_t keepY0, uint32_t keepRows, float* off,
                     float* gain, float* rn)
{
   std::mt19937_64 rng(seed);
   sim::PixelOffsetMap o;
   sim::PixelGainMap g;
   sim::PixelReadNoiseMap r;
   o.Generate(w, h, offMean, offStd, rng, keepY0, keepRows);
   g.Generate(w, h, gainNom, gainFrac, rng, keepY0, keepRows);
   r.Generate(w, h, rnNom, rnFrac, rng, keepY0, keepRows);
   std::memcpy(off, o.offset.data(), o.offset.size() * sizeof(float));
   std::memcpy(gain, g.gainPhotonsPerAdu.data(), g.gainPhotonsPerAdu.size() * sizeof(float));
   std::memcpy(rn, r.readNoiseElectrons.data(), r.readNoiseElectrons.size() * sizeof(float));
}

// ApplyNoiseChain on one frame. off/gain/rn: w*h or NULL.
void ref_noise_chain(const float* photons, uint32_t w, uint32_t h, const iscu_camera* cam, const float* off,
                     const float* gain, const float* rn, uint32_t seed, uint32_t frame, uint32_t pixelBase,
                     int parallel, uint16_t* out)
{
   Maps m;
   FillMaps(m, w, h, off, gain, rn);
   const std::vector<float> img(photons, photons + static_cast<size_t>(w) * h);
   std::vector<uint16_t> adu;
   sim::ApplyNoiseChain(img, adu, w, h, ToCamera(*cam), m.off, m.gain, m.rn, seed, frame, parallel != 0, pixelBase);
   std::memcpy(out, adu.data(), adu.size() * sizeof(uint16_t));
}

// ------------------------------------------------------------------------------------------- PSF
int ref_psf_geometry(const iscu_psf_request* r, int* M)
{
   *M = sim::ZernikePupilSamples(ToRequest(*r));
   return 0;
}

// ComputeZernikePsfPlanes: raw |E|^2 planes (nz * size * size floats).
int ref_zernike_planes(const iscu_psf_request* r, float* out)
{
   std::vector<std::vector<float>> planes;
   if (!sim::ComputeZernikePsfPlanes(ToRequest(*r), planes, g_err))
      return 1;
   size_t o = 0;
   for (const auto& p : planes)
   {
      std::memcpy(out + o, p.data(), p.size() * sizeof(float));
      o += p.size();
   }
   return 0;
}

void* ref_kernel_build(const iscu_psf_request* r)
{
   auto* c = new sim::PsfKernelCache();
   if (!sim::BuildZernikePsfKernelCache(ToRequest(*r), *c, g_err))
   {
      delete c;
      return nullptr;
   }
   c->PrepareSplat();
   return c;
}

// A kernel cache from planes made elsewhere (sum-1 expected), as ComputePsfKernelCache fills one.
void* ref_kernel_from_planes(const float* planes, int size, int nz, int os, double zStepNm, int interp)
{
   auto* c = new sim::PsfKernelCache();
   c->oversampling = os;
   c->halfWidthOversampled = (size - 1) / 2;
   c->sizeOversampled = size;
   c->nz = nz;
   c->zStepNm = zStepNm;
   c->interpMode = static_cast<sim::PsfInterpMode>(interp);
   c->blockSumWidth = size + os - 1;
   sim::PsfKernelPlanes d;
   d.planes.resize(static_cast<size_t>(nz));
   for (int z = 0; z < nz; ++z)
      d.planes[static_cast<size_t>(z)].assign(planes + static_cast<size_t>(z) * size * size,
                                              planes + static_cast<size_t>(z + 1) * size * size);
   c->SetData(std::move(d));
   c->valid = true;
   c->PrepareSplat();
   return c;
}

void* ref_kernel_halo(void* h, double threshold)
{
   auto* c = new sim::PsfKernelCache(sim::WithHaloCut(*static_cast<sim::PsfKernelCache*>(h), threshold));
   return c;
}

void ref_kernel_free(void* h) { delete static_cast<sim::PsfKernelCache*>(h); }

void ref_kernel_info(void* h, int* size, int* nz, int* os, int* bw)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   *size = c->sizeOversampled;
   *nz = c->nz;
   *os = c->oversampling;
   *bw = c->blockSumWidth;
}

void ref_kernel_planes(void* h, float* out)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   size_t o = 0;
   for (const auto& p : c->Planes())
   {
      std::memcpy(out + o, p.data(), p.size() * sizeof(float));
      o += p.size();
   }
}

void ref_kernel_block_sums(void* h, float* out)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   size_t o = 0;
   for (int z = 0; z < c->nz; ++z)
   {
      const std::vector<float> b = c->BlockSums(z).RowMajor();
      std::memcpy(out + o, b.data(), b.size() * sizeof(float));
      o += b.size();
   }
}

// PsfHaloSpans of a halo-cut cache: lo/hi (nz * (2 camRad + 1)), radius2 (nz). Returns camRad, or -1 without a cut.
int ref_kernel_spans(void* h, int16_t* lo, int16_t* hi, int32_t* radius2)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   if (!c->halo)
      return -1;
   std::memcpy(lo, c->halo->lo.data(), c->halo->lo.size() * sizeof(int16_t));
   std::memcpy(hi, c->halo->hi.data(), c->halo->hi.size() * sizeof(int16_t));
   std::memcpy(radius2, c->halo->radius2.data(), c->halo->radius2.size() * sizeof(int32_t));
   return c->halo->camRad;
}

int ref_nearest_z(void* h, double zUm)
{
   return static_cast<sim::PsfKernelCache*>(h)->NearestZIndex(zUm);
}

// ------------------------------------------------------------------------------------------- render
// RenderPhotonImage for one frame (background + splats), the camera-independent part.
void ref_render_photon_image(void* h, const iscu_blink_event* ev, uint32_t nEv, int64_t frame, uint32_t w, uint32_t hgt,
                             double pixelNm, double photonsPerBlink, double bg, double driftX, double driftY,
                             double globalZ, const float* illum, const float* bgMap, double bgScale,
                             double minPhotons, int parallel, int accumulate, float* out)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   const std::vector<sim::BlinkEvent> events = ToEvents(ev, nEv);
   std::vector<float> il, bm;
   sim::RenderExtras ex;
   const size_t n = static_cast<size_t>(w) * hgt;
   if (illum)
   {
      il.assign(illum, illum + n);
      ex.illumField = &il;
   }
   if (bgMap)
   {
      bm.assign(bgMap, bgMap + n);
      ex.backgroundMap = &bm;
   }
   ex.backgroundScale = bgScale;
   ex.minPhotons = minPhotons;
   ex.parallel = parallel != 0;
   ex.accumulate = accumulate != 0;
   std::vector<float> img;
   if (accumulate)
      img.assign(out, out + n);   // a later dye group splats onto the earlier groups' image
   sim::RenderPhotonImage(img, w, hgt, events, frame, pixelNm, 1.3, photonsPerBlink, bg, driftX, driftY, c, globalZ,
                          nullptr, nullptr, &ex);
   std::memcpy(out, img.data(), n * sizeof(float));
}

// CollectGpuEmitters for one frame: the reference's 64-byte records. Returns the count (<= maxOut).
uint32_t ref_collect_gpu_emitters(void* h, const iscu_blink_event* ev, uint32_t nEv, int64_t frame, uint32_t w,
                                  uint32_t hgt, double pixelNm, double photonsPerBlink, double driftX, double driftY,
                                  double globalZ, int kernel, double minPhotons, iscu_gpu_splat_emitter* out,
                                  uint32_t maxOut)
{
   static_assert(sizeof(sim::GpuSplatEmitter) == sizeof(iscu_gpu_splat_emitter), "record layout");
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   const std::vector<sim::BlinkEvent> events = ToEvents(ev, nEv);
   std::vector<sim::GpuSplatEmitter> rec;
   sim::CollectGpuEmitters(events, frame, w, hgt, pixelNm, photonsPerBlink, driftX, driftY, *c, globalZ, nullptr, rec,
                           nullptr, nullptr, kernel, minPhotons);
   const uint32_t n = static_cast<uint32_t>(std::min<size_t>(rec.size(), maxOut));
   std::memcpy(out, rec.data(), n * sizeof(iscu_gpu_splat_emitter));
   return static_cast<uint32_t>(rec.size());
}

// The movie loop of one blink group: per frame RenderPhotonImage (serial) then ApplyNoiseChain (serial), frames in
// parallel on the reference's pool (FluorescenceMovie::Render, ScopeMovie.cpp:7267 and :7649). Events are bucketed
// per frame first (BucketEventsByFrame, SMLMSimulation.cpp:203). Returns the seconds spent in the frame loop.
double ref_render_movie(void* h, const iscu_blink_event* ev, uint32_t nEv, uint32_t frame0, uint32_t nFrames,
                        uint32_t w, uint32_t hgt, double pixelNm, double photonsPerBlink, double bg,
                        const iscu_camera* cam, const float* off, const float* gain, const float* rn, uint32_t seed,
                        float* outPhotons, uint16_t* outAdu)
{
   const auto* c = static_cast<sim::PsfKernelCache*>(h);
   const std::vector<sim::BlinkEvent> events = ToEvents(ev, nEv);
   Maps m;
   FillMaps(m, w, hgt, off, gain, rn);
   const sim::CameraNoiseParams cp = ToCamera(*cam);
   const size_t n = static_cast<size_t>(w) * hgt;
   const auto t0 = std::chrono::steady_clock::now();
   // Buckets over [frame0, frame0 + nFrames): events shifted so the bucket index is the batch frame.
   std::vector<sim::BlinkEvent> shifted = events;
   for (auto& e : shifted)
   {
      e.tStart -= frame0;
      e.tEnd -= frame0;
   }
   const auto buckets = sim::BucketEventsByFrame(shifted, nFrames);
   sim::ParallelFor(nFrames, [&](unsigned k) {
      std::vector<sim::BlinkEvent> fe;
      fe.reserve(buckets[k].size());
      for (uint32_t i : buckets[k])
         fe.push_back(events[i]);
      std::vector<float> img;
      sim::RenderPhotonImage(img, w, hgt, fe, static_cast<long>(frame0 + k), pixelNm, 1.3, photonsPerBlink, bg, 0.0,
                             0.0, c, 0.0);
      std::vector<uint16_t> adu;
      sim::ApplyNoiseChain(img, adu, w, hgt, cp, m.off, m.gain, m.rn, seed, frame0 + k, false, 0);
      if (outPhotons)
         std::memcpy(outPhotons + k * n, img.data(), n * sizeof(float));
      if (outAdu)
         std::memcpy(outAdu + k * n, adu.data(), n * sizeof(uint16_t));
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The multi-colour frame loop: each dye group (events whose slot is g, rendered with caches[g]) splatted in group
// order onto one image per frame -- the first group over the background, the later ones with
// RenderExtras::accumulate, as the movie engine renders its dye groups (ScopeMovie.cpp:7059-7110) -- then the noise
// chain. Frames in parallel on the reference's pool. Returns seconds.
double ref_render_movie_groups(void* const* caches, int nGroups, const iscu_blink_event* ev, uint32_t nEv,
                               uint32_t frame0, uint32_t nFrames, uint32_t w, uint32_t hgt, double pixelNm,
                               double photonsPerBlink, double bg, const iscu_camera* cam, const float* off,
                               const float* gain, const float* rn, uint32_t seed, float* outPhotons, uint16_t* outAdu)
{
   std::vector<std::vector<sim::BlinkEvent>> groupEvents(nGroups);
   for (uint32_t i = 0; i < nEv; ++i)
      if (ev[i].slot >= 0 && ev[i].slot < nGroups)
      {
         const std::vector<sim::BlinkEvent> one = ToEvents(ev + i, 1);
         groupEvents[ev[i].slot].push_back(one[0]);
      }
   Maps m;
   FillMaps(m, w, hgt, off, gain, rn);
   const sim::CameraNoiseParams cp = ToCamera(*cam);
   const size_t n = static_cast<size_t>(w) * hgt;
   const auto t0 = std::chrono::steady_clock::now();
   std::vector<std::vector<std::vector<uint32_t>>> buckets(nGroups);
   for (int g = 0; g < nGroups; ++g)
   {
      std::vector<sim::BlinkEvent> shifted = groupEvents[g];
      for (auto& e : shifted)
      {
         e.tStart -= frame0;
         e.tEnd -= frame0;
      }
      buckets[g] = sim::BucketEventsByFrame(shifted, nFrames);
   }
   sim::ParallelFor(nFrames, [&](unsigned k) {
      std::vector<float> img;
      for (int g = 0; g < nGroups; ++g)
      {
         std::vector<sim::BlinkEvent> fe;
         fe.reserve(buckets[g][k].size());
         for (uint32_t i : buckets[g][k])
            fe.push_back(groupEvents[g][i]);
         sim::RenderExtras ex;
         ex.accumulate = g > 0;
         sim::RenderPhotonImage(img, w, hgt, fe, static_cast<long>(frame0 + k), pixelNm, 1.3, photonsPerBlink, bg,
                                0.0, 0.0, static_cast<const sim::PsfKernelCache*>(caches[g]), 0.0, nullptr, nullptr,
                                &ex);
      }
      std::vector<uint16_t> adu;
      sim::ApplyNoiseChain(img, adu, w, hgt, cp, m.off, m.gain, m.rn, seed, frame0 + k, false, 0);
      if (outPhotons)
         std::memcpy(outPhotons + k * n, img.data(), n * sizeof(float));
      if (outAdu)
         std::memcpy(outAdu + k * n, adu.data(), n * sizeof(uint16_t));
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// sim::DriftTrajectory with the given settings: xyz[3 f + (0, 1, 2)] nm.
void ref_drift_trajectory(long seed, long frames, double frameSec, const double* p, int zDirection, double* xyz)
{
   sim::DriftSettings s;
   s.xyNmPerSqrtSec = p[0];
   s.zNmPerSqrtSec = p[1];
   s.xySpeedNmPerSec = p[2];
   s.zSpeedNmPerSec = p[3];
   s.xyAngleDeg = p[4];
   s.zDirection = zDirection;
   s.angleWanderDeg = p[5];
   s.zAngleWanderDeg = p[6];
   s.speedWanderPct = p[7];
   s.wanderTimeSec = p[8];
   const std::vector<sim::DriftNm> t = sim::DriftTrajectory(seed, frames, frameSec, s);
   for (size_t f = 0; f < t.size(); ++f)
   {
      xyz[3 * f] = t[f].x;
      xyz[3 * f + 1] = t[f].y;
      xyz[3 * f + 2] = t[f].z;
   }
}

// sim::BuildIlluminationField: returns the number of floats written (0 for flat).
size_t ref_illumination_field(unsigned w, unsigned h, int profile, double fwhmPct, float* out, double* meanFactor)
{
   const std::vector<float> f =
      sim::BuildIlluminationField(w, h, static_cast<sim::IllumProfile>(profile), fwhmPct, meanFactor);
   std::memcpy(out, f.data(), f.size() * sizeof(float));
   return f.size();
}

double ref_background_fade_scale(double t, double decay) { return sim::BackgroundFadeScale(t, decay); }

// One dye's blinks overlapping [t0, t1) as the world core schedules them (core/src/dyes.cpp): dSTORM / PALM through
// LabelSchedule run without a horizon (then filtered), DNA-PAINT through PersistentBlinks. kin: 6 doubles
// (activation rate, on, off, bleach probability, photon CV, initial on); hist: nSeg start times and 6 nSeg kinetics
// (0 segments: none). out: (tOn, tOff, brightness) rows, at most cap; returns the number of rows.
int ref_dye_blinks(int mode, const double* kin, const double* histStart, const double* histKin, int nSeg, uint32_t h1,
                   int32_t k, int32_t n, double t0, double t1, double* out, int cap)
{
   auto kinOf = [](const double* v) {
      isc::Kinetics q;
      q.activationRatePerSec = v[0];
      q.onSec = v[1];
      q.offSec = v[2];
      q.bleachProb = v[3];
      q.photonCV = v[4];
      q.initialOnSec = v[5];
      return q;
   };
   isc::Label label;
   label.mode = static_cast<isc::LabelMode>(mode);
   label.kin = kinOf(kin);
   isc::KineticsHistory hist;
   for (int s = 0; s < nSeg; ++s)
   {
      hist.tStart.push_back(histStart[s]);
      hist.kin.push_back(kinOf(histKin + 6 * s));
   }
   const isc::KineticsHistory* h = nSeg > 0 ? &hist : nullptr;
   std::vector<isc::Blink> blinks;
   if (label.mode == isc::LabelMode::DnaPaint)
      isc::PersistentBlinks(h1, k, n, label.kin, t0, t1, blinks, h);
   else
      isc::LabelSchedule(h1, k, n, label, &blinks, nullptr, INFINITY, h);
   int m = 0;
   for (const isc::Blink& b : blinks)
   {
      if (!(b.tOn < t1) || !(b.tOff > t0))
         continue;
      if (m < cap && out)
      {
         out[3 * m] = b.tOn;
         out[3 * m + 1] = b.tOff;
         out[3 * m + 2] = b.brightness;
      }
      ++m;
   }
   return m;
}

// The same over n dyes (iscu_dye records), in parallel on the reference's thread pool (sim::ParallelFor, as the
// world schedules its dye blocks on its pool): counts[i] = dye i's rows; returns the wall seconds of the work.
double ref_dye_blinks_batch(int mode, const double* kin, const double* histStart, const double* histKin, int nSeg,
                            const iscu_dye* dyes, uint32_t n, double t0, double t1, uint32_t* counts)
{
   const auto start = std::chrono::steady_clock::now();
   const unsigned chunks = std::max(1u, std::min(n, 4096u));
   sim::ParallelFor(chunks, [&](unsigned c) {
      const uint32_t lo = static_cast<uint32_t>(static_cast<uint64_t>(n) * c / chunks);
      const uint32_t hi = static_cast<uint32_t>(static_cast<uint64_t>(n) * (c + 1) / chunks);
      for (uint32_t i = lo; i < hi; ++i)
         counts[i] = static_cast<uint32_t>(ref_dye_blinks(mode, kin, histStart, histKin, nSeg, dyes[i].h1, dyes[i].k,
                                                          dyes[i].n, t0, t1, nullptr, 0));
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

// The core's DyeH1 (dyes.cpp:175-178): H1 of microtubule mtIndex of cell (cx, cy).
uint32_t ref_dye_h1(uint32_t seed, int32_t cx, int32_t cy, int mtIndex) { return isc::DyeH1(seed, cx, cy, mtIndex); }

// RenderShiftedImages (WidefieldRender.cpp:2905-2935) on WidefieldImages made from given spectra (nCh channels of
// ny x (nx/2 + 1) complex each: the persistent one, then nCh - 1 bleach ones) at a near focus (spec0) and, when
// spec1 is given, a far one, weight w; bleach coefficients a (nCh - 1); the images' sub-cell pose (fracX, fracY) and
// the frame's drift (dx, dy) cells; the FOV window (x0, y0, cw, ch) at up cells per pixel. cam (+=).
void ref_shifted_images(unsigned nx, unsigned ny, const float* spec0, const float* spec1, int nCh, double w,
                        const double* a, double fracX, double fracY, double dx, double dy, unsigned x0, unsigned y0,
                        unsigned cw, unsigned ch, unsigned up, float* cam)
{
   auto fft = std::make_shared<const sim::RealFft2d>(nx, ny);
   const size_t n = fft->SpecSize();
   auto make = [&](const float* spec, sim::WidefieldImages& im) {
      const auto* c = reinterpret_cast<const sim::cfloat*>(spec);
      im.cw = cw;
      im.ch = ch;
      im.upscale = up;
      im.specPersistent.assign(c, c + n);
      for (int k = 1; k < nCh; ++k)
         im.specBleach.emplace_back(c + k * n, c + (k + 1) * n);
      im.fft = fft;
      im.fovX0 = x0;
      im.fovY0 = y0;
      im.fracX = fracX;
      im.fracY = fracY;
   };
   sim::WidefieldImages i0, i1;
   make(spec0, i0);
   if (spec1)
      make(spec1, i1);
   std::vector<float> img(cam, cam + static_cast<size_t>(cw / up) * (ch / up));
   sim::RenderShiftedImages(i0, spec1 ? &i1 : nullptr, w, std::vector<double>(a, a + nCh - 1), dx, dy, img);
   std::copy(img.begin(), img.end(), cam);
}

// The reference's widefield scene on a dense persistent dye grid: WidefieldScene::GridSpecFor / UpdateFromGrid /
// FocusSeries (WidefieldRender.cpp:891, :1180, :2845) with KernelWidefieldPsf(kernel, upscale) (:263-330) under a
// FlatIllumination wider than any margin, unit frame dose and collection efficiency 1 (a cell's value is its dye
// count: the mean-field image of one structure), each focus's images binned by WidefieldImages::Render (:547) into a
// width x height camera frame.
struct RefWfScene
{
   sim::WidefieldSceneSpec spec;
   sim::FlatIllumination pattern{1e6, 1e6};
   std::unique_ptr<sim::KernelWidefieldPsf> psf;
   sim::WidefieldScene scene;
};

static sim::WidefieldSceneSpec WfSpec(int upscale, double capUm, double pixelUm, unsigned width, unsigned height,
                                      double originXUm, double originYUm, double marginUm, double zPlaneNm)
{
   sim::WidefieldSceneSpec spec;
   spec.originXUm = originXUm;
   spec.originYUm = originYUm;
   spec.width = width;
   spec.height = height;
   spec.pixelUm = pixelUm;
   spec.grid.upscale = upscale;
   spec.grid.zPlaneNm = zPlaneNm;
   spec.marginUm = marginUm;
   spec.kernelCapUm = capUm;
   spec.unitDose = 1.0;
   spec.eta = 1.0;
   spec.bleachingMask = 0;
   spec.persistentMask = 1;
   return spec;
}

// The grid such a scene renders on: grid4 = (nx, ny, FOV cell x0, FOV cell y0).
void ref_wf_grid(int upscale, double pixelUm, unsigned width, unsigned height, double originXUm, double originYUm,
                 double marginUm, double zPlaneNm, unsigned* grid4)
{
   const auto spec = WfSpec(upscale, 1.0, pixelUm, width, height, originXUm, originYUm, marginUm, zPlaneNm);
   unsigned fx = 0, fy = 0;
   const sim::WidefieldGridSpec g = sim::WidefieldScene::GridSpecFor(sim::FlatIllumination(1e6, 1e6), spec, &fx, &fy);
   grid4[0] = g.nx;
   grid4[1] = g.ny;
   grid4[2] = fx;
   grid4[3] = fy;
}

// The scene over kernel h and counts (nzd x ny x nx of the grid above; plane i at world plane k0 + i), focused at
// focus0; gpuMode: power-of-two FFTs, no coarse bands (WidefieldScene::SetGpuMode). info3 = (FFT nx, FFT ny, kernel
// radius). Null (the error in ref_last_error) on a failure.
void* ref_wf_scene_create(void* h, int upscale, double capUm, double pixelUm, unsigned width, unsigned height,
                          double originXUm, double originYUm, double marginUm, double zPlaneNm, long k0, unsigned nzd,
                          const float* counts, double focus0, int gpuMode, unsigned* info3)
{
   auto s = std::make_unique<RefWfScene>();
   s->spec = WfSpec(upscale, capUm, pixelUm, width, height, originXUm, originYUm, marginUm, zPlaneNm);
   s->spec.focusWorldUm = focus0;
   const sim::WidefieldGridSpec g = sim::WidefieldScene::GridSpecFor(s->pattern, s->spec);
   sim::WidefieldDyeGrid grid;
   grid.spec = g;
   grid.k0 = k0;
   grid.nz = nzd;
   grid.persistent.assign(counts, counts + static_cast<size_t>(nzd) * g.nx * g.ny);
   double total = 0.0;
   for (float v : grid.persistent)
      total += v;
   grid.nPersistent = static_cast<long>(total + 0.5);
   s->psf = std::make_unique<sim::KernelWidefieldPsf>(*static_cast<const sim::PsfKernelCache*>(h), upscale);
   s->scene.SetGpuMode(gpuMode != 0);
   std::string err;
   if (!s->scene.UpdateFromGrid(grid, s->pattern, s->spec, *s->psf, err))
   {
      g_err = err;
      return nullptr;
   }
   info3[0] = s->scene.FftSizeX();
   info3[1] = s->scene.FftSizeY();
   info3[2] = static_cast<unsigned>(s->scene.KernelRadius());
   return s.release();
}

// FocusSeries at nFoci foci (world um), each focus's camera frame (width x height, Render from 0) into out. Returns
// the wall seconds of the series and the renders, or -1 (the error in ref_last_error).
double ref_wf_scene_series(void* sc, const double* foci, unsigned nFoci, float* out)
{
   auto* s = static_cast<RefWfScene*>(sc);
   const auto t0 = std::chrono::steady_clock::now();
   std::vector<sim::WidefieldImages> images;
   std::string err;
   if (!s->scene.FocusSeries(std::vector<double>(foci, foci + nFoci), images, err))
   {
      g_err = err;
      return -1.0;
   }
   const size_t frame = static_cast<size_t>(s->spec.width) * s->spec.height;
   sim::ParallelFor(nFoci, [&](unsigned i) {
      std::vector<float> cam(frame, 0.0f);
      images[i].Render({}, cam);
      std::copy(cam.begin(), cam.end(), out + i * frame);
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ref_wf_scene_destroy(void* sc) { delete static_cast<RefWfScene*>(sc); }

// PlanSplat with the Fft placement (PsfGeneratorBridge.cpp:1441-1456) for an emitter at (x, y) px on plane z of
// kernel cache h: its shifted block sums (bw x bw floats) into sums and (x0, y0, bx, by) into st4. Returns bw, or 0
// when PlanSplat refuses.
int ref_plan_splat_fft(void* h, double x, double y, int z, float* sums, int* st4)
{
   const auto* c = static_cast<const sim::PsfKernelCache*>(h);
   sim::SplatPlan plan;
   if (!sim::PlanSplat(*c, z, x, y, 1.0, sim::PsfInterpMode::Fft, plan, false))
      return 0;
   std::copy(plan.shiftedSums.begin(), plan.shiftedSums.end(), sums);
   st4[0] = plan.st.x0;
   st4[1] = plan.st.y0;
   st4[2] = plan.st.bx;
   st4[3] = plan.st.by;
   return c->blockSumWidth;
}

// The same for n emitters (x, y, z), emitters in parallel on the reference's pool; wall seconds.
double ref_plan_splat_fft_batch(void* h, const double* xy, const int* z, uint32_t n)
{
   const auto* c = static_cast<const sim::PsfKernelCache*>(h);
   const auto t0 = std::chrono::steady_clock::now();
   const unsigned chunks = std::max(1u, std::min(n, 256u));
   sim::ParallelFor(chunks, [&](unsigned k) {
      for (uint32_t i = static_cast<uint32_t>(static_cast<uint64_t>(n) * k / chunks);
           i < static_cast<uint32_t>(static_cast<uint64_t>(n) * (k + 1) / chunks); ++i)
      {
         sim::SplatPlan plan;
         sim::PlanSplat(*c, z[i], xy[2 * i], xy[2 * i + 1], 1.0, sim::PsfInterpMode::Fft, plan, false);
      }
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// sim::AppendCsvNumber (CsvNumber.cpp) of n values in format fmt: into 48-byte fields (NUL-padded) and lengths.
void ref_csv_numbers(const double* v, uint32_t n, const char* fmt, char* fields, uint8_t* lens)
{
   for (uint32_t i = 0; i < n; ++i)
   {
      std::string s;
      sim::AppendCsvNumber(s, v[i], fmt);
      std::memset(fields + static_cast<size_t>(i) * 48, 0, 48);
      std::memcpy(fields + static_cast<size_t>(i) * 48, s.data(), s.size());
      lens[i] = static_cast<uint8_t>(s.size());
   }
}

// A numeric table formatted as GroundTruth's Rows does it (GroundTruth.cpp:80-111: chunks of 16384 rows on the
// thread pool, each row's cells by AppendCsvNumber -- or, for "%d", std::to_chars of the value -- joined by ',' and
// ended by '\n'), columns column-major; the text into out (capacity cap), returns its length (or the length needed).
size_t ref_csv_table(const double* cols, uint32_t nRows, uint32_t nCols, const char* const* fmts, char* out,
                     size_t cap)
{
   const size_t kChunk = 16384;
   const size_t chunks = (nRows + kChunk - 1) / kChunk;
   std::vector<std::string> parts(chunks);
   sim::ParallelFor(static_cast<unsigned>(chunks), [&](unsigned c) {
      std::string& s = parts[c];
      const size_t a = c * kChunk, b = std::min<size_t>(nRows, a + kChunk);
      for (size_t r = a; r < b; ++r)
         for (uint32_t k = 0; k < nCols; ++k)
         {
            const double v = cols[static_cast<size_t>(k) * nRows + r];
            if (std::strcmp(fmts[k], "%d") == 0)
            {
               char t[24];
               const std::to_chars_result e = std::to_chars(t, t + sizeof t, static_cast<long long>(v));
               s.append(t, e.ptr);
            }
            else
               sim::AppendCsvNumber(s, v, fmts[k]);
            s += k + 1 < nCols ? ',' : '\n';
         }
   });
   size_t n = 0;
   for (const std::string& s : parts)
   {
      if (n + s.size() <= cap)
         std::memcpy(out + n, s.data(), s.size());
      n += s.size();
   }
   return n;
}

// The CLI's movie writer (cli/tiff_writer.h, header-only, included from where it lies): open, pages, row strips,
// close. n_px: the samples px holds (the writer reads w x h of them only when the page is written).
void* ref_tiff_open(const char* path, uint64_t expected, int big) { return new TiffWriter(path, expected, big != 0); }
uint64_t ref_tiff_bytes(uint64_t w, uint64_t h, uint64_t pages, uint64_t bps, uint64_t desc)
{
   return TiffWriter::Bytes(w, h, pages, bps, desc);
}
int ref_tiff_page_u16(void* t, const uint16_t* px, size_t n_px, uint32_t w, uint32_t hgt, const char* desc)
{
   return static_cast<TiffWriter*>(t)->Page(std::vector<uint16_t>(px, px + n_px), w, hgt, desc ? desc : "") ? 1 : 0;
}
int ref_tiff_page_f32(void* t, const float* px, size_t n_px, uint32_t w, uint32_t hgt, const char* desc)
{
   return static_cast<TiffWriter*>(t)->Page(std::vector<float>(px, px + n_px), w, hgt, desc ? desc : "") ? 1 : 0;
}
int ref_tiff_page_rows(void* t, const uint16_t* px, uint32_t rows, uint32_t w, uint32_t hgt, const char* desc)
{
   return static_cast<TiffWriter*>(t)->PageRows(px, rows, w, hgt, desc ? desc : "") ? 1 : 0;
}
int ref_tiff_rows(void* t, uint64_t page, uint32_t y0, uint32_t rows, const uint16_t* px)
{
   return static_cast<TiffWriter*>(t)->Rows(page, y0, rows, px) ? 1 : 0;
}
int ref_tiff_big(void* t) { return static_cast<TiffWriter*>(t)->big() ? 1 : 0; }
// The writer's message ("" when nothing went wrong), into out (cap bytes).
void ref_tiff_error(void* t, char* out, size_t cap)
{
   std::snprintf(out, cap, "%s", static_cast<TiffWriter*>(t)->error().c_str());
}
int ref_tiff_close(void* t)
{
   auto* w = static_cast<TiffWriter*>(t);
   const bool ok = w->Close();
   delete w;
   return ok ? 1 : 0;
}

// sim::BinnedBlinkRenderer (BinnedBlinks.cpp): Setup on the kernel cache h (null: the Gaussian of sigmaPx), then for
// frames k < nFrames Render of emitters [frames[k].em_start, + em_count) (iscu_emitter: position, photons, z index in
// plane & 0xFFFF) into img[k * w * hgt ..] (+=), frames in parallel on the reference's thread pool as its movie loop
// runs them (one frame per worker, its FFT lines serial). u and R out (nullable). Returns the wall seconds of the
// renders, or -1 when Setup refuses.
double ref_binned_render(void* h, double sigmaPx, unsigned w, unsigned hgt, int upscale, const iscu_emitter* em,
                         const iscu_frame* frames, uint32_t nFrames, float* img, int* uOut, int* rOut)
{
   sim::BinnedBlinkRenderer r;
   if (!r.Setup(static_cast<const sim::PsfKernelCache*>(h), sigmaPx, w, hgt, upscale))
      return -1.0;
   if (uOut)
      *uOut = r.Upscale();
   if (rOut)
      *rOut = r.RadiusCells();
   const size_t px = static_cast<size_t>(w) * hgt;
   const auto start = std::chrono::steady_clock::now();
   sim::ParallelFor(nFrames, [&](unsigned k) {
      std::vector<sim::FrameEmitter> list;
      list.reserve(frames[k].em_count);
      for (uint32_t i = frames[k].em_start; i < frames[k].em_start + frames[k].em_count; ++i)
         list.push_back({em[i].x_px, em[i].y_px, em[i].photons, 1.0, em[i].plane & 0xFFFF});
      std::vector<float> frame(img + k * px, img + (k + 1) * px);
      r.Render(list, frame);
      std::copy(frame.begin(), frame.end(), img + k * px);
   });
   return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

} // extern "C"
