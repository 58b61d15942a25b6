// Internal declarations shared by the translation units of libiscu.so (not part of the ABI).
#pragma once

#include "../../include/iscu.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace iscu {

// ------------------------------------------------------------------ errors
void SetError(const std::string& msg);
void ClearError();
int Fail(int code, const std::string& msg);
int CudaFail(cudaError_t e, const char* what);

#define ISCU_CK(call)                                                                                                 \
   do                                                                                                                 \
   {                                                                                                                  \
      cudaError_t e_ = (call);                                                                                        \
      if (e_ != cudaSuccess)                                                                                          \
         return ::iscu::CudaFail(e_, #call);                                                                          \
   } while (0)

// Checks a launch just issued (configuration errors show at once; faults at the next synchronization).
#define ISCU_CK_LAUNCH(ctx, what)                                                                                     \
   do                                                                                                                 \
   {                                                                                                                  \
      (ctx)->launches.fetch_add(1, std::memory_order_relaxed);                                                        \
      cudaError_t e_ = cudaGetLastError();                                                                            \
      if (e_ != cudaSuccess)                                                                                          \
         return ::iscu::CudaFail(e_, what);                                                                           \
   } while (0)

// ------------------------------------------------------------------ device buffers
// A device allocation owned by the context (freed with it).
struct DevBuf
{
   void* p = nullptr;
   size_t bytes = 0;
   DevBuf() = default;
   DevBuf(const DevBuf&) = delete;
   DevBuf& operator=(const DevBuf&) = delete;
   ~DevBuf() { Free(); }
   void Free()
   {
      if (p)
         cudaFree(p);
      p = nullptr;
      bytes = 0;
   }
   // Grows to at least n bytes (contents not kept).
   cudaError_t Reserve(size_t n)
   {
      if (n <= bytes && p)
         return cudaSuccess;
      Free();
      cudaError_t e = cudaMalloc(&p, n ? n : 16);
      if (e == cudaSuccess)
         bytes = n;
      return e;
   }
   template <class T> T* as() const { return static_cast<T*>(p); }
};

// Page-locked host staging (grows; contents not kept).
struct PinnedBuf
{
   void* p = nullptr;
   size_t bytes = 0;
   PinnedBuf() = default;
   PinnedBuf(const PinnedBuf&) = delete;
   PinnedBuf& operator=(const PinnedBuf&) = delete;
   ~PinnedBuf()
   {
      if (p)
         cudaFreeHost(p);
   }
   cudaError_t Reserve(size_t n)
   {
      if (n <= bytes && p)
         return cudaSuccess;
      if (p)
         cudaFreeHost(p);
      p = nullptr;
      bytes = 0;
      cudaError_t e = cudaHostAlloc(&p, n ? n : 16, cudaHostAllocDefault);
      if (e == cudaSuccess)
         bytes = n;
      return e;
   }
   template <class T> T* as() const { return static_cast<T*>(p); }
};

// ------------------------------------------------------------------ kernel stacks (device view)
// What the splat reads of one kernel stack. Passed by value to the kernels.
struct KernelView
{
   const float* sums = nullptr;     // nz planes of bw x bw block sums, row-major
   const double* sums64 = nullptr;  // the same values widened to float64 (the render's general path)
   // The float64 block sums split by oversampling phase, zero-padded: phase[z][qy][qx][ky][kx] =
   // sums[z][ky os + qy - padLo][kx os + qx - padLo] (0 outside the bw x bw array). A cubic splat's tap (j, i) of
   // neighbouring camera pixels then sits in neighbouring words of one phase plane.
   const double* phase = nullptr;
   int nb = 0, padLo = 0;
   const int16_t* spanLo = nullptr; // halo cut: [z * (2 camRad + 1) + dy + camRad]; nullptr: the whole square
   const int16_t* spanHi = nullptr;
   const int32_t* radius2 = nullptr;
   int os = 1, size = 0, nz = 0, bw = 0, camRad = 0, interp = 2;
   double kc = 0.0;                 // (size - 1) / 2
};

struct KernelSlot
{
   bool valid = false;
   int size = 0, nz = 0, os = 1, bw = 0, halfOv = 0, interp = 2;
   double zStepNm = 0.0;
   DevBuf planes;    // nz * size * size
   DevBuf sums;      // nz * bw * bw
   DevBuf sums64;    // nz * bw * bw float64 copies of sums
   DevBuf phase;     // nz * os * os * nb * nb float64, the phase-split padded sums
   int nb = 0, padLo = 0;
   DevBuf spanLo, spanHi, radius2;
   bool halo = false;
   double haloThreshold = 0.0;
   std::vector<int32_t> radius2Host;
   KernelView View() const
   {
      KernelView v;
      v.sums = sums.as<float>();
      v.sums64 = sums64.as<double>();
      v.phase = phase.as<double>();
      v.nb = nb;
      v.padLo = padLo;
      v.spanLo = halo ? spanLo.as<int16_t>() : nullptr;
      v.spanHi = halo ? spanHi.as<int16_t>() : nullptr;
      v.radius2 = halo ? radius2.as<int32_t>() : nullptr;
      v.os = os;
      v.size = size;
      v.nz = nz;
      v.bw = bw;
      v.camRad = halfOv / os;
      v.interp = interp;
      v.kc = (size - 1) / 2.0;
      return v;
   }
   // sim::PsfKernelCache::NearestZIndex (PsfGeneratorBridge.cpp:40-61).
   int NearestZIndex(double zUm, bool* clamped) const;
};

// ------------------------------------------------------------------ camera (device view)
struct CameraView
{
   double qe = 1.0, dark = 0.0, gain = 1.0, readNoise = 0.0;
   int emccd = 0;
   double maxAdu = 65535.0, emGain = 1.0, cic = 0.0;
};
CameraView MakeCameraView(const iscu_camera& c);

struct StaticView
{
   const float* offset = nullptr;
   const float* gain = nullptr;
   const float* readNoise = nullptr;
   const float* background = nullptr;
   const float* illum = nullptr;
   double flatBg = 0.0;
   uint32_t width = 0, height = 0, pixelBase = 0;
};

// Device scratch of the two-pass render (render_contrib.cu): per-emitter setup records, the (slot, plane, tap
// origin) groups, and every emitter's float contribution to each pixel of its square.
struct ContribScratch
{
   DevBuf rec, grec, keys, list, contrib, ctr;
};

// One I/O slot of the event render (iscu_render_events[_async]): the batch's device staging (events, bucket and
// per-frame arrays, the collected emitters and frames, the counts, the frames rendered), its counts read back into
// page-locked memory, and the events ordering upload -> render -> download.
struct EventIo
{
   bool busy = false;              // enqueued, not yet waited for
   DevBuf events, buckets, emitters, frames, counts, photons, adu;
   PinnedBuf hostCounts;           // {n kept (uint32 in a uint64), n clamped (int64)}
   cudaEvent_t uploaded = nullptr, rendered = nullptr, downloaded = nullptr;
   cudaGraphExec_t launches = nullptr;   // the batch's collection and render, re-captured and updated per batch
};

} // namespace iscu

// ------------------------------------------------------------------ the context
struct iscu_ctx
{
   int device = 0;
   cudaStream_t stream = nullptr;
   std::recursive_mutex mu;
   std::atomic<uint64_t> launches{0};
   int smCount = 0;
   int renderConfig = 0;           // render kernel form (iscu_render_set_config)
   iscu::DevBuf dOrder;            // persistent render: frame order + work counter
   iscu::ContribScratch contrib;   // two-pass render scratch
   // render pass timing (iscu_render_set_timing): 4 events per timed call (start, after grouping, after
   // contributions, end)
   bool renderTiming = false;
   std::vector<cudaEvent_t> renderMarks;
   size_t renderCalls = 0;
   size_t contribLimit = 0;        // most bytes the two-pass render's contributions may take (0: a quarter of HBM)
   iscu::KernelSlot kernels[ISCU_MAX_KERNELS];
   // camera statics
   bool haveStatic = false;
   uint32_t width = 0, height = 0, pixelBase = 0;
   double flatBg = 0.0;
   iscu::DevBuf offset, gain, readNoise, background, illum;
   bool haveOffset = false, haveGain = false, haveReadNoise = false, haveBackground = false, haveIllum = false;
   std::vector<float> illumHost;   // the illumination field, for host-side emitter collection
   // staging for the host-pointer entry points
   iscu::DevBuf dEmitters, dFrames, dPhotons, dAdu, dExtras, dScratch;
   iscu::DevBuf dCollect;          // device emitter collection: kept emitters per frame
   iscu::DevBuf dLow16;            // the named-kernel backend's narrowed read-back (iscu_buffer_read_low16)
   iscu::DevBuf dSchedule;         // blink schedules: the history, per-dye counts and first rows
   // the event render's I/O slots (the last one is the blocking call's) and its copy streams (created on first use)
   iscu::EventIo eventIo[ISCU_EVENT_IO_SLOTS + 1];
   cudaStream_t upload = nullptr, download = nullptr;
   // movie files from device frames (iscu_tiff_pages_dev): two page-locked halves, kept for the context's writers
   iscu::PinnedBuf fileStage[2];
   iscu::DevBuf dCsv;              // CSV tables: row lengths and block offsets
   iscu::DevBuf dFftPlace;         // Fft-placement frames: each emitter's shifted block sums and origin
   cudaEvent_t fileCopied[2] = {nullptr, nullptr};
   iscu::StaticView Static() const
   {
      iscu::StaticView s;
      s.offset = haveOffset ? offset.as<float>() : nullptr;
      s.gain = haveGain ? gain.as<float>() : nullptr;
      s.readNoise = haveReadNoise ? readNoise.as<float>() : nullptr;
      s.background = haveBackground ? background.as<float>() : nullptr;
      s.illum = haveIllum ? illum.as<float>() : nullptr;
      s.flatBg = flatBg;
      s.width = width;
      s.height = height;
      s.pixelBase = pixelBase;
      return s;
   }
};

namespace iscu {

// Launchers implemented in the .cu files (ctx->mu held by the caller).
int LaunchPcg4d(iscu_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n);
int LaunchCounterUniforms(iscu_ctx* ctx, uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix,
                          uint32_t perPixel, double* out);
int LaunchNoiseFrames(iscu_ctx* ctx, const float* photons, uint32_t nFrames, const uint32_t* frames,
                      const CameraView& cam, uint32_t seed, uint16_t* adu);
// CollectFrameEmitters for a batch on the device (collect.cu): out gets the kept emitters (at most maxOut written;
// eventIndex, nullable, their events' indices),
// frames the table, *nOut the count kept (may pass maxOut), *nClamped += the clamped z planes (nullable). gapped: frame
// f's emitters at the start of its candidate slots (bucketStart[f] - bucketStart[0] on), the rest of the slots
// zero-photon records, in one launch; *nOut must be zero beforehand.
int LaunchCollect(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t nEvents,
                  const uint32_t* bucketIndex, const uint32_t* bucketStart, int64_t frame0, uint32_t nFrames,
                  double pixelNm, double perBlink, const double* driftX, const double* driftY, const double* globalZ,
                  const double* bgScale, const float* illum, double minPhotons, iscu_emitter* out,
                  uint32_t* eventIndex, uint32_t maxOut, iscu_frame* frames, uint32_t* nOut, int64_t* nClamped,
                  bool gapped = false);
// The render's timing marks of the current call (nullptr when timing is off or the stream is capturing): 4 events.
cudaEvent_t* RenderMarks(iscu_ctx* ctx);
// Emitter runs of the frames beyond nEmitters are cut at nEmitters.
int LaunchRenderFrames(iscu_ctx* ctx, const iscu_emitter* ems, uint32_t nEmitters, const iscu_frame* frames,
                       uint32_t nFrames, const CameraView* cam, uint32_t seed, float* photons, uint16_t* adu);
// The persistent render's scratch: frames heaviest first, then the work counter (zeroed).
size_t OrderBytes(uint32_t nFrames);
int LaunchFrameOrder(iscu_ctx* ctx, const iscu_frame* frames, uint32_t nFrames, uint32_t* orderBuf);
// Grows the two-pass render's scratch for nEm emitters (no launches; what a graph capture needs done before).
// ISCU_ERR_LIMIT when the contributions would pass the context's limit.
int ReserveContrib(iscu_ctx* ctx, uint32_t nEm, ContribScratch& sc);
// The two-pass render (tile config 0..5 of its gather pass). ISCU_ERR_LIMIT when its contributions would pass the
// context's limit; nothing is launched then.
int LaunchContribRender(iscu_ctx* ctx, int tileConfig, const iscu_emitter* ems, uint32_t nEmitters,
                        const iscu_frame* frames, uint32_t nFrames, const CameraView* cam, uint32_t seed,
                        float* photons, uint16_t* adu, uint32_t* orderBuf, ContribScratch& scratch);
int LaunchRenderGpuRecords(iscu_ctx* ctx, const iscu_gpu_splat_emitter* ems, const iscu_frame* frames,
                           uint32_t nFrames, const float* extras, const CameraView* cam, uint32_t seed,
                           uint16_t* adu);
int LaunchBlockSums(iscu_ctx* ctx, const float* planes, int n, int os, int nz, float* sums);
int LaunchSumsToDouble(iscu_ctx* ctx, const float* in, size_t n, double* out);
// The phase-split layout's geometry for a bw x bw block-sum plane at oversampling os: a low margin padLo >= 4 (a
// multiple of os) and nb words per phase row, covering [-padLo, bw + 4) in sum coordinates.
inline void PhaseGeometry(int bw, int os, int& padLo, int& nb)
{
   padLo = os * ((4 + os - 1) / os);
   nb = (padLo + bw + 4 + os - 1) / os;
}
int LaunchPhaseSplit(iscu_ctx* ctx, const float* sums, int nz, int bw, int os, int padLo, int nb, double* out);
int LaunchNormalizePlanes(iscu_ctx* ctx, float* planes, int planeElems, int nPlanes);
// defocusM: each PSF's defocus in metres (the reference's resAxialM * (z - (nz - 1) / 2) for a stack's plane z).
int BuildPsfLibrary(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t nSets, const uint32_t* setOfPsf,
                    const double* defocusM, uint32_t nPsf, int32_t size, int32_t normalize, int32_t method,
                    float* out);
// KernelWidefieldPsf::Kernel's cells (binned.cu): plane p's cell (dx, dy), |dx|, |dy| <= R, is the float64 sum of the
// n x n oversampled plane over [s0 + dy r, +r) x [s0 + dx r, +r) clipped to it, as float; out nz x (2R+1)^2.
int LaunchCellKernels(iscu_ctx* ctx, const float* planes, int n, int nz, int r, int s0, int R, float* out);
// The halo cut of a slot's stack from its device block sums (halo.cu); threshold <= 0: none.
int BuildHalo(iscu_ctx* ctx, KernelSlot& k, double threshold);
// Copies a cut slot's spans (nz (2 camRad + 1) each) and per-plane radius2 (nz) to host memory.
int GetHaloSpans(iscu_ctx* ctx, const KernelSlot& k, int16_t* lo, int16_t* hi, int32_t* radius2);

// PSF geometry helpers (ZernikePsf.cpp:118-158).
struct PsfGeometry
{
   int size = 0, nz = 0, os = 1, halfOv = 0, M = 0;
   double resLateralNm = 0.0;
};
bool GeometryFor(const iscu_psf_request& r, PsfGeometry& g, std::string& err);

} // namespace iscu
