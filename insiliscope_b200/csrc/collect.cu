// Emitter collection on sm_100a: CollectFrameEmitters (adapter/inSiliScope/Simulation/SMLMSimulation.cpp:55-101,
// with the blink-min-photons filter of RenderPhotonImage) for a batch of frames, from blink events resident in HBM,
// into the render's emitter array and frame table -- the host restatement in capi.cpp (CollectFrame) on the device,
// with the same float64 operations in the same order.
//
// Order matters (a frame's emitters are splatted in event order), so the batch is compacted in three launches:
// a CTA per frame counts the events it keeps, one CTA turns the counts into the frame table, and a CTA per frame
// writes its emitters at its table offset, ranks inside a chunk from warp ballots. The event render, which reads a
// frame's emitters only through its table entry, takes them uncompacted in one launch (CollectGappedKernel).
//
// Compiled with --fmad=false, as the host code is compiled with -ffp-contract=off.

#include "iscu_internal.h"

#include <algorithm>
#include <cstdint>

namespace iscu {

namespace {

constexpr int kCT = 256;

struct CollectArgs
{
   const iscu_blink_event* events;
   uint32_t nEvents;
   const uint32_t* bucketIndex;   // nullable: candidate j is events[j]
   const uint32_t* bucketStart;   // nFrames + 1
   int64_t frame0;
   uint32_t nFrames;
   uint32_t width, height;
   double pixelNm, perBlink, minPhotons;
   const double* driftX;          // per frame, nullable
   const double* driftY;
   const double* globalZ;
   const double* bgScale;
   const float* illum;            // width * height, nullable
   int32_t callSlot;              // -1: each event's own slot
   int valid[ISCU_MAX_KERNELS];
   int nz[ISCU_MAX_KERNELS];
   double zStepNm[ISCU_MAX_KERNELS];
   iscu_emitter* out;
   uint32_t* eventIndex;          // nullable: each kept emitter's event index (ground-truth rows)
   uint32_t maxOut;
   iscu_frame* frames;
   uint32_t* keptPerFrame;
   uint32_t* nOut;
   unsigned long long* nClamped;  // nullable
};

// The candidate range of frame f (a decreasing offset reads as empty).
__device__ __forceinline__ void Bucket(const CollectArgs& a, uint32_t f, uint32_t& j0, uint32_t& j1)
{
   j0 = a.bucketStart[f];
   j1 = a.bucketStart[f + 1];
   if (j1 < j0)
      j1 = j0;
}

// The emitter of candidate j in frame f, as CollectFrame computes it; false when the event is not splatted in the
// frame (no overlap, below min photons, an empty kernel slot, an index outside the events).
__device__ bool EmitterOf(const CollectArgs& a, uint32_t f, uint32_t j, iscu_emitter& em, bool& clamped,
                          uint32_t& idx)
{
   clamped = false;
   idx = a.bucketIndex ? a.bucketIndex[j] : j;
   if (idx >= a.nEvents)
      return false;
   const iscu_blink_event e = a.events[idx];
   const int32_t slot = a.callSlot >= 0 ? a.callSlot : e.slot;
   if (slot < 0 || slot >= ISCU_MAX_KERNELS || !a.valid[slot])
      return false;
   const int64_t frame = a.frame0 + f;
   // std::min / std::max as the host writes them
   const double fHi = static_cast<double>(frame + 1), fLo = static_cast<double>(frame);
   const double tEnd = e.t_end < fHi ? e.t_end : fHi;
   const double tStart = fLo < e.t_start ? e.t_start : fLo;
   double ov = tEnd - tStart;
   if (ov <= 0.0)
      return false;
   if (ov > 1.0)
      ov = 1.0;
   const double sitePxX = e.x_um * 1000.0 / a.pixelNm;
   const double sitePxY = e.y_um * 1000.0 / a.pixelNm;
   const double xPx = sitePxX + (a.driftX ? a.driftX[f] : 0.0);
   const double yPx = sitePxY + (a.driftY ? a.driftY[f] : 0.0);
   double photons = a.perBlink * ov;
   if (e.brightness != 1.0)
      photons *= e.brightness;
   if (e.excite != 1.0)
      photons *= e.excite;
   if (a.illum)
   {
      // IlluminationAt (SMLMBackground.cpp:42-54): bilinear at the undrifted site
      const double wm = static_cast<double>(a.width - 1), hm = static_cast<double>(a.height - 1);
      double xi = sitePxX < wm ? sitePxX : wm;
      xi = 0.0 < xi ? xi : 0.0;
      double yi = sitePxY < hm ? sitePxY : hm;
      yi = 0.0 < yi ? yi : 0.0;
      const unsigned fx0 = static_cast<unsigned>(floor(xi)), fy0 = static_cast<unsigned>(floor(yi));
      const unsigned x0 = fx0 < a.width - 1 ? fx0 : a.width - 1;
      const unsigned y0 = fy0 < a.height - 1 ? fy0 : a.height - 1;
      const unsigned x1 = x0 + 1 < a.width - 1 ? x0 + 1 : a.width - 1;
      const unsigned y1 = y0 + 1 < a.height - 1 ? y0 + 1 : a.height - 1;
      const double fx = xi - x0, fy = yi - y0;
      const auto at = [&](unsigned x, unsigned y) {
         return static_cast<double>(a.illum[static_cast<size_t>(y) * a.width + x]);
      };
      photons *= (at(x0, y0) * (1 - fx) + at(x1, y0) * fx) * (1 - fy) + (at(x0, y1) * (1 - fx) + at(x1, y1) * fx) * fy;
   }
   // NearestZIndex (PsfGeneratorBridge.cpp:40-61)
   int z = 0;
   const int nz = a.nz[slot];
   const double zStep = a.zStepNm[slot];
   if (nz > 1 && zStep > 0.0)
   {
      const double zUm = e.z_nm / 1000.0 - (a.globalZ ? a.globalZ[f] : 0.0);
      const double idxF = zUm * 1000.0 / zStep + (nz - 1) / 2.0;
      long long zi = llround(idxF);
      if (zi < 0)
      {
         zi = 0;
         clamped = true;
      }
      if (zi >= nz)
      {
         zi = nz - 1;
         clamped = true;
      }
      z = static_cast<int>(zi);
   }
   if (a.minPhotons > 0.0 && photons < a.minPhotons)
      return false;
   em.x_px = xPx;
   em.y_px = yPx;
   em.photons = photons;
   em.plane = z | (slot << 16);
   em.reserved = 0;
   return true;
}

__global__ void __launch_bounds__(kCT) CollectCountKernel(CollectArgs a)
{
   const uint32_t f = blockIdx.x;
   uint32_t j0, j1;
   Bucket(a, f, j0, j1);
   uint32_t kept = 0;
   for (uint32_t c = j0; c < j1; c += kCT)
   {
      const uint32_t j = c + threadIdx.x;
      bool keep = false;
      if (j < j1)
      {
         iscu_emitter em;
         bool cl;
         uint32_t idx;
         keep = EmitterOf(a, f, j, em, cl, idx);
      }
      kept += static_cast<uint32_t>(__syncthreads_count(keep));
   }
   if (threadIdx.x == 0)
      a.keptPerFrame[f] = kept;
}

// One CTA of 1024 threads: the frame table (em_start = exclusive sum of the kept counts) and the total.
__global__ void __launch_bounds__(1024) CollectTableKernel(CollectArgs a)
{
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __shared__ uint32_t sw[32];
   __shared__ uint32_t carry;
   if (threadIdx.x == 0)
      carry = 0;
   __syncthreads();
   for (uint32_t f0 = 0; f0 < a.nFrames; f0 += 1024)
   {
      const uint32_t f = f0 + threadIdx.x;
      const uint32_t c = f < a.nFrames ? a.keptPerFrame[f] : 0u;
      uint32_t x = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1)
      {
         const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
         if (lane >= d)
            x += y;
      }
      if (lane == 31)
         sw[warp] = x;
      __syncthreads();
      if (warp == 0)
      {
         uint32_t y = sw[lane];
#pragma unroll
         for (int d = 1; d < 32; d <<= 1)
         {
            const uint32_t z = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d)
               y += z;
         }
         sw[lane] = y;
      }
      __syncthreads();
      const uint32_t ex = carry + (warp ? sw[warp - 1] : 0u) + x - c;
      if (f < a.nFrames)
      {
         iscu_frame fr;
         fr.em_start = ex;
         fr.em_count = c;
         fr.frame = static_cast<uint32_t>(a.frame0 + f);
         fr.reserved = 0;
         fr.bg_scale = a.bgScale ? a.bgScale[f] : 1.0;
         a.frames[f] = fr;
      }
      __syncthreads();
      if (threadIdx.x == 1023)
         carry = ex + c;
      __syncthreads();
   }
   if (threadIdx.x == 0)
      *a.nOut = carry;
}

__global__ void __launch_bounds__(kCT) CollectWriteKernel(CollectArgs a)
{
   const uint32_t f = blockIdx.x;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __shared__ uint32_t sWarp[kCT / 32];
   uint32_t j0, j1;
   Bucket(a, f, j0, j1);
   uint32_t pos = a.frames[f].em_start;
   unsigned long long clampedSum = 0;
   for (uint32_t c = j0; c < j1; c += kCT)
   {
      const uint32_t j = c + threadIdx.x;
      bool keep = false, cl = false;
      iscu_emitter em;
      uint32_t idx = 0;
      if (j < j1)
      {
         keep = EmitterOf(a, f, j, em, cl, idx);
         clampedSum += cl ? 1ull : 0ull;
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, keep);
      if (lane == 0)
         sWarp[warp] = __popc(ballot);
      __syncthreads();
      uint32_t base = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kCT / 32; ++w)
      {
         base += w < warp ? sWarp[w] : 0u;
         total += sWarp[w];
      }
      if (keep)
      {
         const uint32_t o = pos + base + __popc(ballot & ((1u << lane) - 1u));
         if (o < a.maxOut)
         {
            a.out[o] = em;
            if (a.eventIndex)
               a.eventIndex[o] = idx;
         }
      }
      pos += total;
      __syncthreads();
   }
   if (a.nClamped)
   {
      for (int d = 16; d > 0; d >>= 1)
         clampedSum += __shfl_down_sync(0xffffffffu, clampedSum, d);
      if (lane == 0 && clampedSum)
         atomicAdd(a.nClamped, clampedSum);
   }
}

// The event render's collection in one launch: a CTA per frame writes its kept emitters, in event order, at the start
// of the frame's own candidate slots [bucketStart[f] - bucketStart[0], bucketStart[f + 1] - bucketStart[0]), fills the
// rest of those slots with zero-photon records (every render form skips them), and writes its frame table entry; the
// total kept goes to nOut by atomics. The render reads a frame's emitters from its table entry, so the gaps change no
// addition: the frames are the compacted batch's, bit for bit.
__global__ void __launch_bounds__(kCT) CollectGappedKernel(CollectArgs a)
{
   const uint32_t f = blockIdx.x;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   __shared__ uint32_t sWarp[kCT / 32];
   uint32_t j0, j1;
   Bucket(a, f, j0, j1);
   const uint32_t first = j0 - a.bucketStart[0], end = j1 - a.bucketStart[0];
   uint32_t pos = first;
   unsigned long long clampedSum = 0;
   for (uint32_t c = j0; c < j1; c += kCT)
   {
      const uint32_t j = c + threadIdx.x;
      bool keep = false, cl = false;
      iscu_emitter em;
      uint32_t idx = 0;
      if (j < j1)
      {
         keep = EmitterOf(a, f, j, em, cl, idx);
         clampedSum += cl ? 1ull : 0ull;
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, keep);
      if (lane == 0)
         sWarp[warp] = __popc(ballot);
      __syncthreads();
      uint32_t base = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kCT / 32; ++w)
      {
         base += w < warp ? sWarp[w] : 0u;
         total += sWarp[w];
      }
      if (keep)
      {
         const uint32_t o = pos + base + __popc(ballot & ((1u << lane) - 1u));
         if (o < a.maxOut)
         {
            a.out[o] = em;
            if (a.eventIndex)
               a.eventIndex[o] = idx;
         }
      }
      pos += total;
      __syncthreads();
   }
   iscu_emitter none;
   none.x_px = 0.0;
   none.y_px = 0.0;
   none.photons = 0.0;
   none.plane = 0;
   none.reserved = 0;
   for (uint32_t o = pos + threadIdx.x; o < end && o < a.maxOut; o += kCT)
      a.out[o] = none;
   if (threadIdx.x == 0)
   {
      iscu_frame fr;
      fr.em_start = first;
      fr.em_count = pos - first;
      fr.frame = static_cast<uint32_t>(a.frame0 + f);
      fr.reserved = 0;
      fr.bg_scale = a.bgScale ? a.bgScale[f] : 1.0;
      a.frames[f] = fr;
      if (pos > first)
         atomicAdd(a.nOut, pos - first);
   }
   if (a.nClamped)
   {
      for (int d = 16; d > 0; d >>= 1)
         clampedSum += __shfl_down_sync(0xffffffffu, clampedSum, d);
      if (lane == 0 && clampedSum)
         atomicAdd(a.nClamped, clampedSum);
   }
}

} // namespace

int LaunchCollect(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t nEvents,
                  const uint32_t* bucketIndex, const uint32_t* bucketStart, int64_t frame0, uint32_t nFrames,
                  double pixelNm, double perBlink, const double* driftX, const double* driftY, const double* globalZ,
                  const double* bgScale, const float* illum, double minPhotons, iscu_emitter* out,
                  uint32_t* eventIndex, uint32_t maxOut, iscu_frame* frames, uint32_t* nOut, int64_t* nClamped,
                  bool gapped)
{
   if (nFrames == 0)
   {
      ISCU_CK(cudaMemsetAsync(nOut, 0, sizeof(uint32_t), ctx->stream));
      return ISCU_OK;
   }
   CollectArgs a;
   a.events = events;
   a.nEvents = nEvents;
   a.bucketIndex = bucketIndex;
   a.bucketStart = bucketStart;
   a.frame0 = frame0;
   a.nFrames = nFrames;
   a.width = ctx->width;
   a.height = ctx->height;
   a.pixelNm = pixelNm;
   a.perBlink = perBlink;
   a.minPhotons = minPhotons;
   a.driftX = driftX;
   a.driftY = driftY;
   a.globalZ = globalZ;
   a.bgScale = bgScale;
   a.illum = illum;
   a.callSlot = slot;
   for (int s = 0; s < ISCU_MAX_KERNELS; ++s)
   {
      const KernelSlot& k = ctx->kernels[s];
      a.valid[s] = k.valid ? 1 : 0;
      a.nz[s] = k.nz;
      a.zStepNm[s] = k.zStepNm;
   }
   a.out = out;
   a.eventIndex = eventIndex;
   a.maxOut = maxOut;
   a.frames = frames;
   ISCU_CK(ctx->dCollect.Reserve(static_cast<size_t>(nFrames) * sizeof(uint32_t)));
   a.keptPerFrame = ctx->dCollect.as<uint32_t>();
   a.nOut = nOut;
   a.nClamped = reinterpret_cast<unsigned long long*>(nClamped);
   if (gapped)
   {
      // nOut is zeroed by the caller (the event render clears its counts with the upload)
      CollectGappedKernel<<<nFrames, kCT, 0, ctx->stream>>>(a);
      ISCU_CK_LAUNCH(ctx, "CollectGappedKernel");
      return ISCU_OK;
   }
   CollectCountKernel<<<nFrames, kCT, 0, ctx->stream>>>(a);
   ISCU_CK_LAUNCH(ctx, "CollectCountKernel");
   CollectTableKernel<<<1, 1024, 0, ctx->stream>>>(a);
   ISCU_CK_LAUNCH(ctx, "CollectTableKernel");
   CollectWriteKernel<<<nFrames, kCT, 0, ctx->stream>>>(a);
   ISCU_CK_LAUNCH(ctx, "CollectWriteKernel");
   return ISCU_OK;
}


// The event render of one batch, enqueued in I/O slot io (the iscu_render_events[_async] contract): host events,
// bucket and per-frame arrays up on the upload stream, CollectFrameEmitters + render + noise on the context's stream,
// frames and counts down on the download stream. Returns with the work in flight; io.busy marks it.
int EnqueueRenderEvents(iscu_ctx* ctx, EventIo& io, int32_t slot, const iscu_blink_event* events, uint32_t nEvents,
                        const uint32_t* bucketIndex, const uint32_t* bucketStart, int64_t frame0, uint32_t nFrames,
                        double pixelNm, double perBlink, const double* driftX, const double* driftY,
                        const double* globalZ, const double* bgScale, int32_t useIllum, double minPhotons,
                        const iscu_camera* cam, uint32_t seed, float* photons, uint16_t* adu)
{
   if ((nFrames && !bucketStart) || (nEvents && !events))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (cam && !adu)
      return Fail(ISCU_ERR_ARG, "a camera needs an ADU output");
   if (slot < -1 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (-1..3)");
   if (nFrames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   if (io.busy)
      return Fail(ISCU_ERR_STATE, "the I/O slot's batch has not been waited for");
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   if (slot >= 0 && !ctx->kernels[slot].valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
   ISCU_CK(cudaStreamIsCapturing(ctx->stream, &capturing));
   if (capturing != cudaStreamCaptureStatusNone)
      return Fail(ISCU_ERR_STATE, "the event render copies from host memory: not inside a stream capture");
   for (uint32_t f = 0; f < nFrames; ++f)
      if (bucketStart[f + 1] < bucketStart[f])
         return Fail(ISCU_ERR_ARG, "bucket offsets must not decrease");
   const uint32_t nIdx = nFrames ? bucketStart[nFrames] : 0;   // the index list (or the events) covers [0, nIdx)
   const uint32_t nCand = nFrames ? bucketStart[nFrames] - bucketStart[0] : 0;
   if (!bucketIndex && nIdx > nEvents)
      return Fail(ISCU_ERR_ARG, "buckets reach past the events");
   if (!ctx->upload)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking));
   if (!ctx->download)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->download, cudaStreamNonBlocking));
   for (cudaEvent_t* e : {&io.uploaded, &io.rendered, &io.downloaded})
      if (!*e)
         ISCU_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
   ISCU_CK(io.hostCounts.Reserve(16));
   // the slot's device staging: events, bucket arrays, per-frame arrays, the batch's emitters and frames, the outputs
   const size_t px = static_cast<size_t>(ctx->width) * ctx->height * nFrames;
   const size_t evB = static_cast<size_t>(nEvents) * sizeof(iscu_blink_event);
   const size_t idxB = bucketIndex ? static_cast<size_t>(nIdx) * sizeof(uint32_t) : 0;
   const size_t bsB = (static_cast<size_t>(nFrames) + 1) * sizeof(uint32_t);
   const size_t perFrameB = static_cast<size_t>(nFrames) * sizeof(double);
   const size_t perFrameAt = (idxB + bsB + 7) & ~size_t(7);
   ISCU_CK(io.events.Reserve(std::max<size_t>(evB, 16)));
   ISCU_CK(io.buckets.Reserve(perFrameAt + 4 * perFrameB + 16));
   ISCU_CK(io.emitters.Reserve(std::max<size_t>(static_cast<size_t>(nCand) * sizeof(iscu_emitter), 16)));
   ISCU_CK(io.frames.Reserve(std::max<size_t>(static_cast<size_t>(nFrames) * sizeof(iscu_frame), 16)));
   ISCU_CK(io.counts.Reserve(16));
   if (photons)
      ISCU_CK(io.photons.Reserve(std::max<size_t>(px * sizeof(float), 16)));
   if (adu)
      ISCU_CK(io.adu.Reserve(std::max<size_t>(px * sizeof(uint16_t), 16)));
   char* b = io.buckets.as<char>();
   uint32_t* dIdx = bucketIndex ? reinterpret_cast<uint32_t*>(b) : nullptr;
   uint32_t* dBs = reinterpret_cast<uint32_t*>(b + idxB);
   double* dPerFrame = reinterpret_cast<double*>(b + perFrameAt);
   const double* hostPerFrame[4] = {driftX, driftY, globalZ, bgScale};
   const double* devPerFrame[4] = {nullptr, nullptr, nullptr, nullptr};
   uint32_t* dN = io.counts.as<uint32_t>();
   int64_t* dClamped = reinterpret_cast<int64_t*>(io.counts.as<char>() + 8);

   // upload: the slot's buffers are free (its last batch was waited for), so the copies need wait on nothing
   cudaStream_t up = ctx->upload;
   if (evB)
      ISCU_CK(cudaMemcpyAsync(io.events.p, events, evB, cudaMemcpyHostToDevice, up));
   if (idxB)
      ISCU_CK(cudaMemcpyAsync(dIdx, bucketIndex, idxB, cudaMemcpyHostToDevice, up));
   if (nFrames)
      ISCU_CK(cudaMemcpyAsync(dBs, bucketStart, bsB, cudaMemcpyHostToDevice, up));
   for (int k = 0; k < 4; ++k)
      if (hostPerFrame[k] && nFrames)
      {
         ISCU_CK(cudaMemcpyAsync(dPerFrame + static_cast<size_t>(k) * nFrames, hostPerFrame[k], perFrameB,
                                 cudaMemcpyHostToDevice, up));
         devPerFrame[k] = dPerFrame + static_cast<size_t>(k) * nFrames;
      }
   ISCU_CK(cudaMemsetAsync(io.counts.p, 0, 16, up));
   ISCU_CK(cudaEventRecord(io.uploaded, up));

   // collection, render and noise on the context's stream, after the upload and after everything enqueued before.
   // They are captured into a graph and replayed through the slot's executable (updated in place from each batch's
   // capture, made again when the launches' shape changes): the same kernels with fewer gaps between them. What the
   // launches would allocate is reserved first, since a capture may not allocate.
   cudaStream_t s = ctx->stream;
   ISCU_CK(cudaStreamWaitEvent(s, io.uploaded, 0));
   if (nFrames)
   {
      CameraView cv;
      if (cam)
         cv = MakeCameraView(*cam);
      ISCU_CK(ctx->dCollect.Reserve(static_cast<size_t>(nFrames) * sizeof(uint32_t)));
      ISCU_CK(ctx->dOrder.Reserve(OrderBytes(nFrames)));
      if (ctx->renderConfig >= 12)
      {
         const int rr = ReserveContrib(ctx, nCand, ctx->contrib);
         if (rr == ISCU_ERR_LIMIT)
            ClearError();   // the render falls back to the one-pass form of the same tile
         else if (rr != ISCU_OK)
            return rr;
      }
      ISCU_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int rc = LaunchCollect(ctx, slot, io.events.as<iscu_blink_event>(), nEvents, dIdx, dBs, frame0, nFrames,
                             pixelNm, perBlink, devPerFrame[0], devPerFrame[1], devPerFrame[2], devPerFrame[3],
                             useIllum && ctx->haveIllum ? ctx->illum.as<float>() : nullptr, minPhotons,
                             io.emitters.as<iscu_emitter>(), nullptr, nCand, io.frames.as<iscu_frame>(), dN,
                             dClamped, true);
      if (rc == ISCU_OK)
         rc = LaunchRenderFrames(ctx, io.emitters.as<iscu_emitter>(), nCand, io.frames.as<iscu_frame>(), nFrames,
                                 cam ? &cv : nullptr, seed, photons ? io.photons.as<float>() : nullptr,
                                 adu ? io.adu.as<uint16_t>() : nullptr);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (rc != ISCU_OK || ec != cudaSuccess)
      {
         if (graph)
            cudaGraphDestroy(graph);
         if (rc != ISCU_OK)
            return rc;
         ISCU_CK(ec);
      }
      bool updated = false;
      if (io.launches)
      {
         cudaGraphExecUpdateResultInfo info;
         updated = cudaGraphExecUpdate(io.launches, graph, &info) == cudaSuccess;
         if (!updated)
         {
            cudaGetLastError();   // a refused update leaves no sticky error; the executable is made again
            cudaGraphExecDestroy(io.launches);
            io.launches = nullptr;
         }
      }
      cudaError_t ei = cudaSuccess;
      if (!updated)
         ei = cudaGraphInstantiate(&io.launches, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess)
      {
         io.launches = nullptr;
         ISCU_CK(ei);
      }
      ISCU_CK(cudaGraphLaunch(io.launches, s));
   }
   ISCU_CK(cudaEventRecord(io.rendered, s));

   // download: the frames and the counts, after the render
   cudaStream_t down = ctx->download;
   ISCU_CK(cudaStreamWaitEvent(down, io.rendered, 0));
   if (photons && px)
      ISCU_CK(cudaMemcpyAsync(photons, io.photons.p, px * sizeof(float), cudaMemcpyDeviceToHost, down));
   if (adu && px)
      ISCU_CK(cudaMemcpyAsync(adu, io.adu.p, px * sizeof(uint16_t), cudaMemcpyDeviceToHost, down));
   ISCU_CK(cudaMemcpyAsync(io.hostCounts.p, io.counts.p, 16, cudaMemcpyDeviceToHost, down));
   ISCU_CK(cudaEventRecord(io.downloaded, down));
   io.busy = true;
   return ISCU_OK;
}

// Waits for slot io's batch; its counts into *nEmitters (nullable) and += *nClamped (nullable). The slot is idle after.
int WaitRenderEvents(EventIo& io, uint32_t* nEmitters, int64_t* nClamped)
{
   if (!io.busy)
      return Fail(ISCU_ERR_STATE, "no batch in the I/O slot");
   io.busy = false;
   ISCU_CK(cudaEventSynchronize(io.downloaded));
   const uint64_t* c = io.hostCounts.as<uint64_t>();
   if (nEmitters)
      *nEmitters = static_cast<uint32_t>(c[0]);
   if (nClamped)
      *nClamped += static_cast<int64_t>(c[1]);
   return ISCU_OK;
}

} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_collect_emitters_dev(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events_dev, uint32_t n_events,
                              const uint32_t* bucket_index_dev, const uint32_t* bucket_start_dev, int64_t frame0,
                              uint32_t n_frames, double pixel_size_nm, double photons_per_blink,
                              const double* drift_x_px_dev, const double* drift_y_px_dev,
                              const double* global_z_offset_um_dev, const double* bg_scale_dev, const float* illum_dev,
                              double min_photons, iscu_emitter* out_dev, uint32_t* event_index_dev,
                              uint32_t max_out, iscu_frame* frames_out_dev, uint32_t* n_out_dev,
                              int64_t* n_clamped_dev)
{
   if (!ctx || !n_out_dev || (n_frames && (!bucket_start_dev || !frames_out_dev)) || (n_events && !events_dev) ||
       (max_out && !out_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (slot < -1 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (-1..3)");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static): the frame size is unknown");
   if (slot >= 0 && !ctx->kernels[slot].valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   return LaunchCollect(ctx, slot, events_dev, n_events, bucket_index_dev, bucket_start_dev, frame0, n_frames,
                        pixel_size_nm, photons_per_blink, drift_x_px_dev, drift_y_px_dev, global_z_offset_um_dev,
                        bg_scale_dev, illum_dev, min_photons, out_dev, event_index_dev, max_out, frames_out_dev,
                        n_out_dev, n_clamped_dev);
}

int iscu_render_events(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t n_events,
                       const uint32_t* bucket_index, const uint32_t* bucket_start, int64_t frame0, uint32_t n_frames,
                       double pixel_size_nm, double photons_per_blink, const double* drift_x_px,
                       const double* drift_y_px, const double* global_z_offset_um, const double* bg_scale,
                       int32_t use_illum, double min_photons, const iscu_camera* cam, uint32_t seed, float* photons,
                       uint16_t* adu, uint32_t* n_emitters, int64_t* n_clamped)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null argument");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   EventIo& io = ctx->eventIo[ISCU_EVENT_IO_SLOTS];   // the blocking call's own slot
   int rc = EnqueueRenderEvents(ctx, io, slot, events, n_events, bucket_index, bucket_start, frame0, n_frames,
                                pixel_size_nm, photons_per_blink, drift_x_px, drift_y_px, global_z_offset_um,
                                bg_scale, use_illum, min_photons, cam, seed, photons, adu);
   if (rc != ISCU_OK)
      return rc;
   return WaitRenderEvents(io, n_emitters, n_clamped);
}

int iscu_render_events_async(iscu_ctx* ctx, int32_t io_slot, int32_t slot, const iscu_blink_event* events,
                             uint32_t n_events, const uint32_t* bucket_index, const uint32_t* bucket_start,
                             int64_t frame0, uint32_t n_frames, double pixel_size_nm, double photons_per_blink,
                             const double* drift_x_px, const double* drift_y_px, const double* global_z_offset_um,
                             const double* bg_scale, int32_t use_illum, double min_photons, const iscu_camera* cam,
                             uint32_t seed, float* photons, uint16_t* adu)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null argument");
   if (io_slot < 0 || io_slot >= ISCU_EVENT_IO_SLOTS)
      return Fail(ISCU_ERR_ARG, "I/O slot out of range (0..3)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   return EnqueueRenderEvents(ctx, ctx->eventIo[io_slot], slot, events, n_events, bucket_index, bucket_start,
                              frame0, n_frames, pixel_size_nm, photons_per_blink, drift_x_px, drift_y_px,
                              global_z_offset_um, bg_scale, use_illum, min_photons, cam, seed, photons, adu);
}

int iscu_render_events_wait(iscu_ctx* ctx, int32_t io_slot, uint32_t* n_emitters, int64_t* n_clamped)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null argument");
   if (io_slot < 0 || io_slot >= ISCU_EVENT_IO_SLOTS)
      return Fail(ISCU_ERR_ARG, "I/O slot out of range (0..3)");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   return WaitRenderEvents(ctx->eventIo[io_slot], n_emitters, n_clamped);
}

} // extern "C"
