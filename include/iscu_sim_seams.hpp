// iscu_sim_seams.hpp -- libiscu.so behind two of the render engine's own C++ seams (header-only, C++17). Include it in
// a build of the reference's Simulation sources (their directory on the include path, libiscu.so linked):
//
//   iscu_sim::ComputePsfKernelCacheGpu  -- ComputePsfKernelCache (PsfGeneratorBridge.h:317) for the GibsonLanniZernike
//       model with the stack built on the B200: the cache is filled as BuildZernikePsfKernelCache fills it
//       (ZernikePsf.cpp:382-415) and handed its planes through PsfKernelCache::SetData (PsfGeneratorBridge.cpp:1122),
//       so every consumer of a PsfKernelCache (the CPU splat, the halo cut, the widefield kernel, a GPU host) keeps
//       working unchanged;
//   iscu_sim::WidefieldAcceleratorCuda  -- a sim::WidefieldAccelerator (WidefieldRender.h:342-359) over the focus-job
//       engine (iscu_wf_job_*): WidefieldScene::SetAccelerator(&accel) (WidefieldRender.h:615) or
//       FluorescenceMovie::Begin(spec, gpuMode, err, &accel) (ScopeMovie.h:433) hand it the scene's focus work.
//
// Errors follow the engine's convention: bool plus std::string& err, no exceptions across the seam.
#pragma once

#include "PsfGeneratorBridge.h"
#include "SMLMZernike.h"
#include "WidefieldRender.h"
#include "iscu.h"

#include <string>
#include <utility>
#include <vector>

namespace iscu_sim {

// A GibsonLanniZernike request as the C ABI's (the Zernike string parsed as the engine parses it).
inline bool ToIscuRequest(const sim::PsfGeneratorRequest& q, iscu_psf_request& r, std::string& err)
{
   if (q.model != sim::PsfModelKind::GibsonLanniZernike)
   {
      err = "the B200 PSF builder computes the GibsonLanniZernike model only";
      return false;
   }
   bool ok = true;
   const sim::ZernikeCoefficients z = sim::ParseZernikeCoefficients(q.zernikeCoefficients, ok);
   if (!ok)
   {
      err = "Zernike coefficients: need 15 or 28 numbers";
      return false;
   }
   r = iscu_psf_request{};
   r.wavelength_nm = q.wavelengthNm;
   r.na = q.na;
   r.immersion_index = q.immersionIndex;
   r.sample_index = q.sampleIndex;
   r.working_distance_um = q.workingDistanceUm;
   r.sample_depth_nm = q.sampleDepthNm;
   r.pixel_size_nm = q.pixelSizeNm;
   for (size_t j = 0; j < sim::kNumZernike && j < 28; ++j)
      r.zernike[j] = z[j];
   r.mask_double_helix = q.maskType == sim::PsfMaskType::DoubleHelix ? 1 : 0;
   r.mask_modes = q.maskModes;
   r.mask_waist = q.maskWaist;
   r.oversampling = q.oversampling;
   r.kernel_half_width_px = q.kernelHalfWidthPx;
   r.nz = q.nz;
   r.pupil_samples = q.pupilSamples;
   r.z_step_nm = q.zStepNm;
   r.interp = static_cast<int32_t>(q.interpMode);
   return true;
}

// The stack of a GibsonLanniZernike request built on the context's B200 (chirp-Z and sum-1 planes on the device,
// through kernel slot `slot`, which it overwrites), handed to outCache as BuildZernikePsfKernelCache does: the
// geometry fields, then SetData with the planes (the splat's block sums are made from them on first use). The stack
// equals ComputePsfKernelCache's within 1e-5 of each plane's maximum. False (outCache left invalid) with err set.
inline bool ComputePsfKernelCacheGpu(iscu_ctx* ctx, const sim::PsfGeneratorRequest& req, sim::PsfKernelCache& outCache,
                                     std::string& err, int slot = ISCU_MAX_KERNELS - 1, int method = ISCU_CZT_FP32)
{
   outCache = sim::PsfKernelCache();
   iscu_psf_request r;
   if (!ToIscuRequest(req, r, err))
      return false;
   int32_t size = 0, nz = 0, os = 0, bw = 0;
   if (iscu_kernel_build(ctx, slot, &r, method) != ISCU_OK ||
       iscu_kernel_info(ctx, slot, &size, &nz, &os, &bw) != ISCU_OK)
   {
      err = iscu_last_error();
      return false;
   }
   std::vector<float> all(static_cast<size_t>(nz) * size * size);
   if (iscu_kernel_get_planes(ctx, slot, all.data()) != ISCU_OK)
   {
      err = iscu_last_error();
      return false;
   }
   sim::PsfKernelPlanes d;
   d.planes.resize(static_cast<size_t>(nz));
   const size_t plane = static_cast<size_t>(size) * size;
   for (int z = 0; z < nz; ++z)
      d.planes[static_cast<size_t>(z)].assign(all.begin() + z * plane, all.begin() + (z + 1) * plane);
   outCache.oversampling = os;
   outCache.halfWidthOversampled = (size - 1) / 2;
   outCache.sizeOversampled = size;
   outCache.nz = nz;
   outCache.zStepNm = req.zStepNm;
   outCache.interpMode = req.interpMode;
   outCache.blockSumWidth = bw;
   outCache.SetData(std::move(d));
   outCache.valid = true;
   return true;
}

// sim::WidefieldAccelerator on the B200: the scene's plane spectra stay resident on the device by key (HasPlane),
// its kernels' spectra by plane index, within one geometry; Images runs a job's channels (iscu_wf_job_images).
class WidefieldAcceleratorCuda : public sim::WidefieldAccelerator
{
public:
   // budgetBytes: the device bytes the plane spectra may take (0: a quarter of the device).
   explicit WidefieldAcceleratorCuda(iscu_ctx* ctx, uint64_t budgetBytes = 0)
   {
      if (iscu_wf_job_create(ctx, budgetBytes, &job_) != ISCU_OK)
         error_ = iscu_last_error();
   }
   ~WidefieldAcceleratorCuda() override { iscu_wf_job_destroy(job_); }
   WidefieldAcceleratorCuda(const WidefieldAcceleratorCuda&) = delete;
   WidefieldAcceleratorCuda& operator=(const WidefieldAcceleratorCuda&) = delete;

   bool Ok(std::string& err) const
   {
      err = error_;
      return job_ != nullptr;
   }
   bool HasPlane(unsigned long long geometry, unsigned long long key) const override
   {
      return job_ && iscu_wf_job_has_plane(job_, geometry, key) == 1;
   }
   bool Fits(unsigned long long geometry, unsigned NX, unsigned NY, size_t planes) override
   {
      return job_ && iscu_wf_job_fits(job_, geometry, NX, NY, planes) == 1;
   }
   bool Images(const sim::WidefieldGpuJob& job, std::vector<std::vector<float>>& out, std::string& err) override
   {
      if (!job_)
      {
         err = error_;
         return false;
      }
      std::vector<iscu_wf_job_kernel> kernels;
      for (const auto& k : job.kernels)
         kernels.push_back({k.p, 0, reinterpret_cast<const float*>(k.spec->data())});
      std::vector<iscu_wf_job_plane> planes;
      for (const auto& p : job.planes)
         planes.push_back({p.key, p.cells.data(), p.values.data(), static_cast<uint32_t>(p.cells.size()), 0});
      std::vector<iscu_wf_job_dep> deps;
      std::vector<uint32_t> start(1, 0);
      for (const auto& ch : job.channels)
      {
         for (const auto& d : ch)
            deps.push_back({d.key, d.p0, d.p1, d.w0, d.w1, d.two ? 1 : 0, 0});
         start.push_back(static_cast<uint32_t>(deps.size()));
      }
      iscu_wf_job_desc desc{};
      desc.nx_fft = job.NX;
      desc.ny_fft = job.NY;
      desc.nx = job.nx;
      desc.ny = job.ny;
      desc.fov_x0 = job.fovX0;
      desc.fov_y0 = job.fovY0;
      desc.cw = job.cw;
      desc.ch = job.ch;
      desc.frac_x = job.fracX;
      desc.frac_y = job.fracY;
      desc.geometry = job.geometry;
      desc.kernels = kernels.data();
      desc.n_kernels = static_cast<uint32_t>(kernels.size());
      desc.planes = planes.data();
      desc.n_planes = static_cast<uint32_t>(planes.size());
      desc.deps = deps.data();
      desc.channel_start = start.data();
      desc.n_channels = static_cast<uint32_t>(job.channels.size());
      out.assign(job.channels.size(), std::vector<float>(static_cast<size_t>(job.cw) * job.ch));
      std::vector<float*> ptrs;
      for (auto& v : out)
         ptrs.push_back(v.data());
      if (iscu_wf_job_images(job_, &desc, ptrs.data()) != ISCU_OK)
      {
         err = iscu_last_error();
         out.clear();
         return false;
      }
      return true;
   }

private:
   iscu_wf_job* job_ = nullptr;
   std::string error_;
};

} // namespace iscu_sim
