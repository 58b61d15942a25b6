// iscu_gpusim.hpp -- the engine's C++ GPU seams over libiscu.so's C ABI (header-only, C++17).
//
// iscu_sim::GpuSimulator keeps the method names, arguments and error convention (bool + std::string& err, no
// exceptions) of sim::GpuSimulator (adapter/inSiliScope/Simulation/GpuSimD3D11.h:61-111), so the engine's callers
// (SMLMImageGeneration.cpp:251-268, LiveAhead.cpp:254) keep their code when a build links this instead of the
// Direct3D 11 one; the kernel stacks are given as their planes (what a PsfKernelCache holds) rather than as the
// reference's cache objects. The exact path (the CPU renderer's bits), blink events to frames in one call, is
// iscu_render_events on the same context (GpuSimulator::context()).
#pragma once

#include "iscu.h"

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace iscu_sim {

// sim::CameraNoiseParams (SMLMNoise.h:35-50): gain in photons (electrons) per ADU.
struct CameraNoiseParams
{
   double quantumEfficiency = 1.0;
   double darkCurrentElectrons = 0.0;
   double gainPhotonsPerAdu = 1.0;
   double readNoiseElectrons = 0.0;
   bool emccd = false;
   int bitDepth = 16;
   double emGain = 1.0;
   double cicElectrons = 0.0;
};

// What the splat reads of a sim::PsfKernelCache: its planes (nz x size x size, sum 1 each), oversampling, z pitch,
// interpolation (iscu_interp) and halo threshold (<= 0: none).
struct KernelPlanes
{
   std::vector<float> planes;
   int size = 0, nz = 0, oversampling = 1, interp = ISCU_INTERP_CUBIC;
   double zStepNm = 0.0, haloThreshold = 0.0;
};

// sim::GpuSplatEmitter (GpuSimD3D11.h:50-59): the same 64 bytes.
using GpuSplatEmitter = iscu_gpu_splat_emitter;

inline iscu_camera ToCamera(const CameraNoiseParams& c)
{
   iscu_camera k{};
   k.quantum_efficiency = c.quantumEfficiency;
   k.dark_electrons = c.darkCurrentElectrons;
   k.gain = c.gainPhotonsPerAdu;
   k.read_noise_e = c.readNoiseElectrons;
   k.emccd = c.emccd ? 1 : 0;
   k.bit_depth = c.bitDepth;
   k.em_gain = c.emGain;
   k.cic_electrons = c.cicElectrons;
   return k;
}

// A context and its failure message, shared by the classes below.
class Context
{
public:
   explicit Context(iscu_ctx* c) : ctx_(c) {}
   ~Context() { iscu_destroy(ctx_); }
   Context(const Context&) = delete;
   Context& operator=(const Context&) = delete;
   iscu_ctx* get() const { return ctx_; }
   static bool Ok(int rc, std::string& err)
   {
      if (rc == ISCU_OK)
         return true;
      err = iscu_last_error();
      return false;
   }

private:
   iscu_ctx* ctx_;
};

class GpuSimulator
{
public:
   static constexpr size_t kMaxKernels = ISCU_MAX_KERNELS;

   // nullptr if no sm_100 device; outInfo names the device on success, the reason on failure.
   static std::unique_ptr<GpuSimulator> Create(std::string& outInfo, int device = 0)
   {
      iscu_ctx* c = nullptr;
      if (iscu_create(device, &c) != ISCU_OK)
      {
         outInfo = iscu_last_error();
         return nullptr;
      }
      outInfo = "libiscu (CUDA, sm_100a) on device " + std::to_string(device);
      return std::unique_ptr<GpuSimulator>(new GpuSimulator(c));
   }

   // Each kernel's planes into slot k (block sums and halo spans are built on the device).
   bool SetKernels(const std::vector<const KernelPlanes*>& kernels, std::string& outError)
   {
      if (kernels.size() > kMaxKernels)
      {
         outError = "at most 4 kernels";
         return false;
      }
      for (size_t k = 0; k < kernels.size(); ++k)
      {
         const KernelPlanes* p = kernels[k];
         if (!p || p->planes.size() != static_cast<size_t>(p->nz) * p->size * p->size)
         {
            outError = "kernel " + std::to_string(k) + ": planes do not match nz x size x size";
            return false;
         }
         const int s = static_cast<int>(k);
         if (!Context::Ok(iscu_kernel_set_planes(ctx_.get(), s, p->planes.data(), p->size, p->nz, p->oversampling,
                                                 p->zStepNm, p->interp),
                          outError) ||
             !Context::Ok(iscu_kernel_set_halo(ctx_.get(), s, p->haloThreshold), outError))
            return false;
      }
      return true;
   }

   bool SetStatic(unsigned width, unsigned height, const std::vector<float>& offset, const std::vector<float>& gain,
                  const std::vector<float>& readNoise, const std::vector<float>& background, double flatBg,
                  const CameraNoiseParams& cam, std::string& outError)
   {
      const size_t n = static_cast<size_t>(width) * height;
      for (const std::vector<float>* v : {&offset, &gain, &readNoise, &background})
         if (!v->empty() && v->size() != n)
         {
            outError = "a static map is neither empty nor width * height long";
            return false;
         }
      auto ptr = [](const std::vector<float>& v) { return v.empty() ? nullptr : v.data(); };
      cam_ = cam;
      width_ = width;
      height_ = height;
      return Context::Ok(iscu_set_static(ctx_.get(), width, height, 0, ptr(offset), ptr(gain), ptr(readNoise),
                                         ptr(background), nullptr, flatBg),
                         outError);
   }

   bool RenderFrame(const std::vector<GpuSplatEmitter>& emitters, const CameraNoiseParams& cam,
                    double backgroundScale, uint32_t noiseSeed, uint32_t frame, std::vector<uint16_t>& out,
                    std::string& outError, const std::vector<float>* extra = nullptr)
   {
      std::vector<uint16_t>* outs[1] = {&out};
      std::vector<const std::vector<float>*> ex{extra};
      return RenderFrames({emitters}, {frame}, {backgroundScale}, cam, noiseSeed,
                          std::vector<std::vector<uint16_t>*>(outs, outs + 1), outError, extra ? &ex : nullptr);
   }

   bool RenderFrames(const std::vector<std::vector<GpuSplatEmitter>>& emitters, const std::vector<uint32_t>& frames,
                     const std::vector<double>& backgroundScales, const CameraNoiseParams& cam, uint32_t noiseSeed,
                     const std::vector<std::vector<uint16_t>*>& outs, std::string& outError,
                     const std::vector<const std::vector<float>*>* extras = nullptr)
   {
      const size_t nf = frames.size(), px = static_cast<size_t>(width_) * height_;
      if (emitters.size() != nf || backgroundScales.size() != nf || outs.size() != nf ||
          (extras && extras->size() != nf))
      {
         outError = "emitters, frames, background scales, outputs and extras must have one entry per frame";
         return false;
      }
      std::vector<GpuSplatEmitter> rec;
      std::vector<iscu_frame> table(nf);
      std::vector<float> ex;
      bool anyExtra = false;
      if (extras)
         for (const std::vector<float>* e : *extras)
            anyExtra = anyExtra || e != nullptr;
      if (anyExtra)
         ex.assign(nf * px, 0.0f);
      for (size_t k = 0; k < nf; ++k)
      {
         table[k] = iscu_frame{static_cast<uint32_t>(rec.size()), static_cast<uint32_t>(emitters[k].size()),
                               frames[k], 0u, backgroundScales[k]};
         rec.insert(rec.end(), emitters[k].begin(), emitters[k].end());
         if (anyExtra && (*extras)[k])
         {
            if ((*extras)[k]->size() != px)
            {
               outError = "an extra image is not width * height long";
               return false;
            }
            std::copy((*extras)[k]->begin(), (*extras)[k]->end(), ex.begin() + k * px);
         }
      }
      std::vector<uint16_t> adu(nf * px);
      const iscu_camera c = ToCamera(cam);
      if (!Context::Ok(iscu_render_gpu_records(ctx_.get(), rec.data(), static_cast<uint32_t>(rec.size()),
                                               table.data(), static_cast<uint32_t>(nf), anyExtra ? ex.data() : nullptr,
                                               &c, noiseSeed, adu.data()),
                       outError))
         return false;
      for (size_t k = 0; k < nf; ++k)
         outs[k]->assign(adu.begin() + k * px, adu.begin() + (k + 1) * px);
      return true;
   }

   size_t MaxBatchFrames() const { return 65535; }

   iscu_ctx* context() const { return ctx_.get(); }

private:
   explicit GpuSimulator(iscu_ctx* c) : ctx_(c) {}
   Context ctx_;
   CameraNoiseParams cam_;
   unsigned width_ = 0, height_ = 0;
};

} // namespace iscu_sim
