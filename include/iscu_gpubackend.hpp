// sim::GpuBackend (WidefieldGpuHost.h:42-77) over libiscu's named-kernel backend (iscu_buffer_*, iscu_dispatch), so
// that the reference's own GPU hosts -- SplatGpuHost (SplatGpu.h:40-75, the blink splat + noise) and WidefieldGpuHost
// (WidefieldGpuHost.h:79-114, the widefield focus spectra and frames) -- run unmodified on a B200:
//
//    std::string err;
//    std::shared_ptr<iscu_sim::CudaGpuBackend> be = iscu_sim::CudaGpuBackend::Create(0, err);
//    std::unique_ptr<sim::SplatGpuHost> splat = sim::MakeSplatGpuHost(be, err);   // runs its self-check
//    sim::SetDefaultBlinkSplatGpu([be](std::string& info) { return sim::MakeSplatGpuHost(be, info); });
//
// Header-only; include it where the reference's Simulation directory is on the include path (WidefieldGpuHost.h) and
// link libiscu. The reference's conventions hold: bool + err, no exceptions across the seam, the backend's
// recursive mutex serializes its hosts (each call also takes the context's own lock).
#pragma once

#include "WidefieldGpuHost.h"
#include "iscu.h"

#include <cstdint>
#include <memory>
#include <string>

namespace iscu_sim {

class CudaGpuBackend final : public sim::GpuBackend
{
public:
   // A backend on CUDA device `device` (an sm_100 GPU); nullptr (err = why) when there is none.
   static std::shared_ptr<CudaGpuBackend> Create(int device, std::string& err)
   {
      iscu_ctx* ctx = nullptr;
      if (iscu_create(device, &ctx) != ISCU_OK)
      {
         err = iscu_last_error();
         return nullptr;
      }
      std::shared_ptr<CudaGpuBackend> be(new CudaGpuBackend(std::make_shared<Device>(ctx)));
      be->name = "libiscu CUDA sm_100a, device " + std::to_string(device);
      return be;
   }

   BufPtr Make(size_t bytes, const void* data, std::string& err) override
   {
      iscu_buffer* b = nullptr;
      if (iscu_buffer_create(dev_->ctx, bytes, data, &b) != ISCU_OK)
      {
         err = iscu_last_error();
         return nullptr;
      }
      return std::make_shared<CudaBuffer>(dev_, b);
   }

   bool Write(Buffer& b, size_t offset, const void* data, size_t bytes, std::string& err) override
   {
      iscu_buffer* d = Of(b, err);
      return d && Ok(iscu_buffer_write(d, offset, data, bytes), err);
   }

   bool Copy(Buffer& dst, Buffer& src, size_t bytes, std::string& err) override
   {
      iscu_buffer* d = Of(dst, err);
      iscu_buffer* s = d ? Of(src, err) : nullptr;
      return s && Ok(iscu_buffer_copy(d, s, bytes), err);
   }

   bool Dispatch(const char* kernel, const uint32_t* params, size_t nParams, Buffer* const* bufs, size_t nBufs,
                 unsigned x, unsigned y, unsigned z, std::string& err) override
   {
      iscu_buffer* b[8] = {};
      if (nBufs > 8)
      {
         err = "more than 8 buffers";
         return false;
      }
      for (size_t i = 0; i < nBufs; ++i)
         if (!bufs[i] || !(b[i] = Of(*bufs[i], err)))
            return false;
      return Ok(iscu_dispatch(dev_->ctx, kernel, params, nParams, b, nBufs, x, y, z), err);
   }

   bool ReadBack(Buffer& src, size_t bytes, void* dst, std::string& err) override
   {
      iscu_buffer* s = Of(src, err);
      return s && Ok(iscu_buffer_read(s, bytes, dst), err);
   }

   bool ReadBackLow16(Buffer& src, size_t words, uint16_t* dst, std::string& err) override
   {
      iscu_buffer* s = Of(src, err);
      return s && Ok(iscu_buffer_read_low16(s, words, dst), err);
   }

   // A binding is addressed by 32-bit word indices.
   size_t MaxBinding() const override { return size_t(1) << 32; }

   iscu_ctx* context() const { return dev_->ctx; }

private:
   // The context, alive while the backend or any of its buffers is.
   struct Device
   {
      iscu_ctx* ctx;
      explicit Device(iscu_ctx* c) : ctx(c) {}
      ~Device() { iscu_destroy(ctx); }
   };
   struct CudaBuffer final : Buffer
   {
      std::shared_ptr<Device> dev;
      iscu_buffer* buf;
      CudaBuffer(std::shared_ptr<Device> d, iscu_buffer* b) : dev(std::move(d)), buf(b) { bytes = iscu_buffer_bytes(b); }
      ~CudaBuffer() override { iscu_buffer_destroy(buf); }
   };

   explicit CudaGpuBackend(std::shared_ptr<Device> d) : dev_(std::move(d)) {}

   static iscu_buffer* Of(Buffer& b, std::string& err)
   {
      CudaBuffer* c = dynamic_cast<CudaBuffer*>(&b);
      if (!c)
      {
         err = "a buffer made by another backend";
         return nullptr;
      }
      return c->buf;
   }
   static bool Ok(int rc, std::string& err)
   {
      if (rc == ISCU_OK)
         return true;
      err = iscu_last_error();
      return false;
   }

   std::shared_ptr<Device> dev_;
};

} // namespace iscu_sim
