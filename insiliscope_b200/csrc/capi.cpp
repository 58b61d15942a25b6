// The extern "C" surface of libiscu.so (include/iscu.h): argument checks, context state, host staging and the
// host-side steps the reference also runs on the CPU (camera map generation, emitter collection, halo spans).
//
// Built with -ffp-contract=off: the host arithmetic restated here (CollectFrameEmitters, the camera maps,
// NearestZIndex) must round exactly as the reference's does.

#include "iscu_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <vector>

namespace iscu {

namespace {
thread_local std::string g_error;
}

void SetError(const std::string& msg) { g_error = msg; }
void ClearError() { g_error.clear(); }
int Fail(int code, const std::string& msg)
{
   g_error = msg;
   return code;
}
int CudaFail(cudaError_t e, const char* what)
{
   g_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
   return ISCU_ERR_CUDA;
}

CameraView MakeCameraView(const iscu_camera& c)
{
   CameraView v;
   v.qe = c.quantum_efficiency;
   v.dark = c.dark_electrons;
   v.gain = c.gain;
   v.readNoise = c.read_noise_e;
   v.emccd = c.emccd ? 1 : 0;
   // ApplyNoiseChain's EMCCD constants (SMLMNoise.cpp:162-164).
   v.maxAdu = std::ldexp(1.0, std::min(16, std::max(1, static_cast<int>(c.bit_depth)))) - 1.0;
   v.emGain = std::max(1.0, c.em_gain);
   v.cic = c.cic_electrons;
   return v;
}

int KernelSlot::NearestZIndex(double zUm, bool* clamped) const
{
   if (clamped)
      *clamped = false;
   if (nz <= 1 || zStepNm <= 0.0)
      return 0;
   const double idxF = zUm * 1000.0 / zStepNm + (nz - 1) / 2.0;
   int idx = static_cast<int>(std::lround(idxF));
   if (idx < 0)
   {
      idx = 0;
      if (clamped)
         *clamped = true;
   }
   if (idx >= nz)
   {
      idx = nz - 1;
      if (clamped)
         *clamped = true;
   }
   return idx;
}

namespace {

struct Lock
{
   std::lock_guard<std::recursive_mutex> g;
   explicit Lock(iscu_ctx* c) : g(c->mu) { ClearError(); }
};

int CheckSlot(iscu_ctx* ctx, int32_t slot, bool needValid)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   if (slot < 0 || slot >= ISCU_MAX_KERNELS)
      return Fail(ISCU_ERR_ARG, "kernel slot out of range (0..3)");
   if (needValid && !ctx->kernels[slot].valid)
      return Fail(ISCU_ERR_STATE, "no kernel stack in slot " + std::to_string(slot));
   return ISCU_OK;
}

int UploadMap(iscu_ctx* ctx, DevBuf& buf, bool& have, const float* host, size_t n)
{
   have = host != nullptr;
   if (!host)
      return ISCU_OK;
   ISCU_CK(buf.Reserve(n * sizeof(float)));
   ISCU_CK(cudaMemcpyAsync(buf.p, host, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
   return ISCU_OK;
}

// The sensor's static maps draw from one std::mt19937_64 stream: the offset map's w h standard normals, then the
// gain map's, then the read-noise map's -- the order in which the reference generates them (SMLMNoise.cpp:89-140,
// called offset, gain, read noise by SplatGpu.cpp:500-502). Normal number j is made from engine outputs 2j and 2j + 1
// taken as uniforms in [0, 1) (std::generate_canonical, what std::uniform_real_distribution(0, 1) returns) by the
// direct Box-Muller form sqrt(-2 ln a) cos(2 pi b), a raised to 1e-300 (GaussianRng, SMLMNoise.cpp:17-35). A window
// of rows keeps a slice of each map: the engine jumps over the outputs of the pixels left out with discard().
class SensorNormalStream
{
public:
   explicit SensorNormalStream(uint64_t seed) : eng_(seed) {}
   // Normal number j of the stream; j may not decrease from one call to the next.
   double Normal(uint64_t j)
   {
      const uint64_t at = 2 * j;
      if (at > used_)
      {
         eng_.discard(at - used_);
         used_ = at;
      }
      const double a = Uniform();
      const double b = Uniform();
      return std::sqrt(-2.0 * std::log(a < 1e-300 ? 1e-300 : a)) * std::cos(kTwoPi * b);
   }

private:
   static constexpr double kTwoPi = 2.0 * 3.14159265358979323846;   // exact doubling of the double nearest pi
   double Uniform()
   {
      ++used_;
      return std::generate_canonical<double, std::numeric_limits<double>::digits>(eng_);
   }
   std::mt19937_64 eng_;
   uint64_t used_ = 0;
};

} // namespace

} // namespace iscu

using namespace iscu;

extern "C" {

const char* iscu_last_error(void) { return g_error.c_str(); }

int iscu_abi_version(void) { return ISCU_ABI_VERSION; }

int iscu_create(int device, iscu_ctx** out)
{
   ClearError();
   if (!out)
      return Fail(ISCU_ERR_ARG, "null output pointer");
   *out = nullptr;
   int n = 0;
   cudaError_t e = cudaGetDeviceCount(&n);
   if (e != cudaSuccess || n == 0)
      return Fail(ISCU_ERR_NODEV, "no CUDA device");
   if (device < 0 || device >= n)
      return Fail(ISCU_ERR_ARG, "device index out of range");
   cudaDeviceProp prop;
   ISCU_CK(cudaGetDeviceProperties(&prop, device));
   if (prop.major != 10)
      return Fail(ISCU_ERR_NODEV, std::string("not an sm_100 device: ") + prop.name);
   ISCU_CK(cudaSetDevice(device));
   std::unique_ptr<iscu_ctx> c(new iscu_ctx());
   c->device = device;
   c->smCount = prop.multiProcessorCount;
   ISCU_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
   *out = c.release();
   return ISCU_OK;
}

void iscu_destroy(iscu_ctx* ctx)
{
   if (!ctx)
      return;
   cudaSetDevice(ctx->device);
   cudaStreamSynchronize(ctx->stream);
   for (cudaStream_t c : {ctx->upload, ctx->download})
      if (c)
         cudaStreamSynchronize(c);
   for (cudaEvent_t e : ctx->renderMarks)
      cudaEventDestroy(e);
   for (iscu::EventIo& io : ctx->eventIo)
   {
      for (cudaEvent_t e : {io.uploaded, io.rendered, io.downloaded})
         if (e)
            cudaEventDestroy(e);
      if (io.launches)
         cudaGraphExecDestroy(io.launches);
   }
   for (cudaEvent_t e : ctx->fileCopied)
      if (e)
         cudaEventDestroy(e);
   cudaStream_t streams[3] = {ctx->stream, ctx->upload, ctx->download};
   delete ctx;
   for (cudaStream_t c : streams)
      if (c)
         cudaStreamDestroy(c);
}

int iscu_synchronize(iscu_ctx* ctx)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   Lock l(ctx);
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   for (cudaStream_t c : {ctx->upload, ctx->download})
      if (c)
         ISCU_CK(cudaStreamSynchronize(c));
   ISCU_CK(cudaGetLastError());
   return ISCU_OK;
}

void* iscu_stream(iscu_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

uint64_t iscu_launch_count(iscu_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

// ------------------------------------------------------------------------------------------ RNG
int iscu_pcg4d_dev(iscu_ctx* ctx, const uint32_t* in4_dev, uint32_t* out4_dev, size_t n)
{
   if (!ctx || (n && (!in4_dev || !out4_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   Lock l(ctx);
   return LaunchPcg4d(ctx, in4_dev, out4_dev, n);
}

int iscu_counter_uniforms_dev(iscu_ctx* ctx, uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix,
                              uint32_t per_pixel, double* out_dev)
{
   if (!ctx || (npix && per_pixel && !out_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   Lock l(ctx);
   return LaunchCounterUniforms(ctx, seed, frame, pixel0, npix, per_pixel, out_dev);
}

// ------------------------------------------------------------------------------------------ camera
int iscu_set_static(iscu_ctx* ctx, uint32_t width, uint32_t height, uint32_t pixel_base, const float* offset,
                    const float* gain, const float* read_noise, const float* background, const float* illum,
                    double flat_bg)
{
   if (!ctx)
      return Fail(ISCU_ERR_ARG, "null context");
   if (width == 0 || height == 0 || width > 65536 || height > 65536)
      return Fail(ISCU_ERR_ARG, "frame size out of range (1..65536)");
   Lock l(ctx);
   const size_t n = static_cast<size_t>(width) * height;
   ctx->haveStatic = false;
   int rc;
   if ((rc = UploadMap(ctx, ctx->offset, ctx->haveOffset, offset, n)) != ISCU_OK ||
       (rc = UploadMap(ctx, ctx->gain, ctx->haveGain, gain, n)) != ISCU_OK ||
       (rc = UploadMap(ctx, ctx->readNoise, ctx->haveReadNoise, read_noise, n)) != ISCU_OK ||
       (rc = UploadMap(ctx, ctx->background, ctx->haveBackground, background, n)) != ISCU_OK ||
       (rc = UploadMap(ctx, ctx->illum, ctx->haveIllum, illum, n)) != ISCU_OK)
      return rc;
   if (illum)
      ctx->illumHost.assign(illum, illum + n);
   else
      ctx->illumHost.clear();
   ctx->width = width;
   ctx->height = height;
   ctx->pixelBase = pixel_base;
   ctx->flatBg = flat_bg;
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   ctx->haveStatic = true;
   return ISCU_OK;
}

int iscu_generate_camera_maps(uint32_t width, uint32_t height, uint64_t seed, double offset_mean_adu,
                              double offset_std_adu, double gain_nominal, double gain_std_fraction,
                              double read_noise_nominal, double read_noise_std_fraction, uint32_t keep_y0,
                              uint32_t keep_rows, float* offset, float* gain, float* read_noise)
{
   ClearError();
   if (width == 0 || height == 0)
      return Fail(ISCU_ERR_ARG, "map size must be > 0");
   const uint64_t n = static_cast<uint64_t>(width) * height;
   uint32_t y0 = 0, rows = height;
   if (keep_rows)
   {
      y0 = std::min(keep_y0, height);
      rows = std::min(keep_rows, height - y0);
   }
   const uint64_t first = static_cast<uint64_t>(y0) * width, count = static_cast<uint64_t>(rows) * width;
   SensorNormalStream s(seed);
   // The offset map (PixelOffsetMap::Generate, SMLMNoise.cpp:89-102): normals [0, n).
   for (uint64_t i = 0; i < count; ++i)
   {
      const float v = static_cast<float>(offset_mean_adu + offset_std_adu * s.Normal(first + i));
      if (offset)
         offset[i] = v;
   }
   // The gain map (PixelGainMap::Generate, SMLMNoise.cpp:119-140): normals [n, 2n), floored at 4 % of the nominal.
   const double gainFloor = 0.04 * gain_nominal;
   for (uint64_t i = 0; i < count; ++i)
   {
      const double v = gain_nominal * (1.0 + gain_std_fraction * s.Normal(n + first + i));
      if (gain)
         gain[i] = static_cast<float>(std::max(v, gainFloor));
   }
   // The read-noise map (PixelReadNoiseMap::Generate, SMLMNoise.cpp:104-117): normals [2n, 3n), not below 0.
   for (uint64_t i = 0; i < count; ++i)
   {
      const double v = read_noise_nominal * (1.0 + read_noise_std_fraction * s.Normal(2 * n + first + i));
      if (read_noise)
         read_noise[i] = static_cast<float>(std::max(v, 0.0));
   }
   return ISCU_OK;
}

int iscu_noise_frames_dev(iscu_ctx* ctx, const float* photons_dev, uint32_t n_frames, const uint32_t* frames_dev,
                          const iscu_camera* cam, uint32_t seed, uint16_t* adu_dev)
{
   if (!ctx || !cam || (n_frames && (!photons_dev || !frames_dev || !adu_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   Lock l(ctx);
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   return LaunchNoiseFrames(ctx, photons_dev, n_frames, frames_dev, MakeCameraView(*cam), seed, adu_dev);
}

// ------------------------------------------------------------------------------------------ PSF
int iscu_psf_geometry(const iscu_psf_request* req, int32_t* size, int32_t* nz, int32_t* pupil_samples)
{
   ClearError();
   if (!req)
      return Fail(ISCU_ERR_ARG, "null request");
   PsfGeometry g;
   std::string err;
   if (!GeometryFor(*req, g, err))
      return Fail(ISCU_ERR_ARG, err);
   if (size)
      *size = g.size;
   if (nz)
      *nz = g.nz;
   if (pupil_samples)
      *pupil_samples = g.M;
   return ISCU_OK;
}

int iscu_psf_library_dev(iscu_ctx* ctx, const iscu_psf_request* sets, uint32_t n_sets, const uint32_t* set_of_psf,
                         const double* defocus_nm, uint32_t n_psf, int32_t size, int32_t normalize, int32_t method,
                         float* out_dev)
{
   if (!ctx || (n_psf && (!sets || !set_of_psf || !defocus_nm || !out_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (method != ISCU_CZT_FP32 && method != ISCU_CZT_TF32X3 && method != ISCU_CZT_F16X3)
      return Fail(ISCU_ERR_ARG, "unknown chirp-Z method");
   if (size < 0 || size > 1024)
      return Fail(ISCU_ERR_ARG, "plane size out of range (0..1024)");
   Lock l(ctx);
   std::vector<double> defocusM(n_psf);
   for (uint32_t i = 0; i < n_psf; ++i)
      defocusM[i] = defocus_nm[i] * 1E-9;
   return BuildPsfLibrary(ctx, sets, n_sets, set_of_psf, defocusM.data(), n_psf, size, normalize, method, out_dev);
}

// ------------------------------------------------------------------------------------------ kernel slots
static int FinishKernelSlot(iscu_ctx* ctx, KernelSlot& k)
{
   k.bw = k.size + k.os - 1;
   ISCU_CK(k.sums.Reserve(static_cast<size_t>(k.nz) * k.bw * k.bw * sizeof(float)));
   const size_t nSums = static_cast<size_t>(k.nz) * k.bw * k.bw;
   ISCU_CK(k.sums64.Reserve(nSums * sizeof(double)));
   PhaseGeometry(k.bw, k.os, k.padLo, k.nb);
   ISCU_CK(k.phase.Reserve(static_cast<size_t>(k.nz) * k.os * k.os * k.nb * k.nb * sizeof(double)));
   int rc = LaunchBlockSums(ctx, k.planes.as<float>(), k.size, k.os, k.nz, k.sums.as<float>());
   if (rc == ISCU_OK)
      rc = LaunchSumsToDouble(ctx, k.sums.as<float>(), nSums, k.sums64.as<double>());
   if (rc == ISCU_OK)
      rc = LaunchPhaseSplit(ctx, k.sums.as<float>(), k.nz, k.bw, k.os, k.padLo, k.nb, k.phase.as<double>());
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   k.halo = false;
   k.valid = true;
   return ISCU_OK;
}

int iscu_kernel_build(iscu_ctx* ctx, int32_t slot, const iscu_psf_request* req, int32_t method)
{
   int rc = CheckSlot(ctx, slot, false);
   if (rc != ISCU_OK)
      return rc;
   if (!req)
      return Fail(ISCU_ERR_ARG, "null request");
   Lock l(ctx);
   PsfGeometry g;
   std::string err;
   if (!GeometryFor(*req, g, err))
      return Fail(ISCU_ERR_ARG, err);
   KernelSlot& k = ctx->kernels[slot];
   k.valid = false;
   k.size = g.size;
   k.nz = g.nz;
   k.os = g.os;
   k.halfOv = g.halfOv;
   k.interp = req->interp;
   k.zStepNm = req->z_step_nm;
   ISCU_CK(k.planes.Reserve(static_cast<size_t>(k.nz) * k.size * k.size * sizeof(float)));
   // Plane z at resAxialM * (z - (nz - 1) / 2) (ZernikePsf.cpp:237).
   const double resAxialM = req->z_step_nm * 1E-9;
   std::vector<uint32_t> setOf(static_cast<size_t>(k.nz), 0u);
   std::vector<double> defocusM(static_cast<size_t>(k.nz));
   for (int z = 0; z < k.nz; ++z)
      defocusM[static_cast<size_t>(z)] = resAxialM * (z - (k.nz - 1.0) / 2.0);
   rc = BuildPsfLibrary(ctx, req, 1, setOf.data(), defocusM.data(), static_cast<uint32_t>(k.nz), k.size, 1, method,
                        k.planes.as<float>());
   if (rc != ISCU_OK)
      return rc;
   return FinishKernelSlot(ctx, k);
}

int iscu_kernel_set_planes(iscu_ctx* ctx, int32_t slot, const float* planes, int32_t size, int32_t nz,
                           int32_t oversampling, double z_step_nm, int32_t interp)
{
   int rc = CheckSlot(ctx, slot, false);
   if (rc != ISCU_OK)
      return rc;
   if (!planes || size < 3 || nz < 1 || oversampling < 1 || size % 2 == 0 || size > 8193)
      return Fail(ISCU_ERR_ARG, "kernel planes: need odd size >= 3, nz >= 1, oversampling >= 1");
   if ((size - 1) / 2 % oversampling != 0)
      return Fail(ISCU_ERR_ARG, "kernel planes: half width must be a multiple of the oversampling");
   if (interp < ISCU_INTERP_NEAREST || interp > ISCU_INTERP_CUBIC)
      return Fail(ISCU_ERR_ARG, "kernel planes: interp must be nearest, linear or cubic");
   Lock l(ctx);
   KernelSlot& k = ctx->kernels[slot];
   k.valid = false;
   k.size = size;
   k.nz = nz;
   k.os = oversampling;
   k.halfOv = (size - 1) / 2;
   k.interp = interp;
   k.zStepNm = z_step_nm;
   const size_t bytes = static_cast<size_t>(nz) * size * size * sizeof(float);
   ISCU_CK(k.planes.Reserve(bytes));
   ISCU_CK(cudaMemcpyAsync(k.planes.p, planes, bytes, cudaMemcpyHostToDevice, ctx->stream));
   return FinishKernelSlot(ctx, k);
}

int iscu_kernel_set_halo(iscu_ctx* ctx, int32_t slot, double threshold)
{
   int rc = CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   Lock l(ctx);
   return BuildHalo(ctx, ctx->kernels[slot], threshold);
}

int iscu_kernel_get_halo(iscu_ctx* ctx, int32_t slot, int16_t* lo, int16_t* hi, int32_t* radius2)
{
   int rc = CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   if (!lo || !hi || !radius2)
      return Fail(ISCU_ERR_ARG, "null argument");
   Lock l(ctx);
   const KernelSlot& k = ctx->kernels[slot];
   if (!k.halo)
      return Fail(ISCU_ERR_STATE, "slot " + std::to_string(slot) + " has no halo cut");
   return GetHaloSpans(ctx, k, lo, hi, radius2);
}

int iscu_kernel_info(iscu_ctx* ctx, int32_t slot, int32_t* size, int32_t* nz, int32_t* oversampling,
                     int32_t* block_sum_width)
{
   int rc = CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   const KernelSlot& k = ctx->kernels[slot];
   if (size)
      *size = k.size;
   if (nz)
      *nz = k.nz;
   if (oversampling)
      *oversampling = k.os;
   if (block_sum_width)
      *block_sum_width = k.bw;
   return ISCU_OK;
}

int iscu_kernel_get_planes(iscu_ctx* ctx, int32_t slot, float* out)
{
   int rc = CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   if (!out)
      return Fail(ISCU_ERR_ARG, "null output");
   Lock l(ctx);
   const KernelSlot& k = ctx->kernels[slot];
   ISCU_CK(cudaMemcpyAsync(out, k.planes.p, static_cast<size_t>(k.nz) * k.size * k.size * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

int iscu_kernel_get_block_sums(iscu_ctx* ctx, int32_t slot, float* out)
{
   int rc = CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   if (!out)
      return Fail(ISCU_ERR_ARG, "null output");
   Lock l(ctx);
   const KernelSlot& k = ctx->kernels[slot];
   ISCU_CK(cudaMemcpyAsync(out, k.sums.p, static_cast<size_t>(k.nz) * k.bw * k.bw * sizeof(float),
                           cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

// ------------------------------------------------------------------------------------------ splat + noise
int iscu_render_frames_dev(iscu_ctx* ctx, const iscu_emitter* emitters_dev, uint32_t n_emitters,
                           const iscu_frame* frames_dev, uint32_t n_frames, const iscu_camera* cam, uint32_t seed,
                           float* photons_dev, uint16_t* adu_dev)
{
   if (!ctx || (n_frames && !frames_dev) || (n_emitters && !emitters_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (cam && !adu_dev)
      return Fail(ISCU_ERR_ARG, "a camera needs an ADU output");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   Lock l(ctx);
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   CameraView cv;
   if (cam)
      cv = MakeCameraView(*cam);
   return LaunchRenderFrames(ctx, emitters_dev, n_emitters, frames_dev, n_frames, cam ? &cv : nullptr, seed,
                             photons_dev, adu_dev);
}

int iscu_render_frames(iscu_ctx* ctx, const iscu_emitter* emitters, uint32_t n_emitters, const iscu_frame* frames,
                       uint32_t n_frames, const iscu_camera* cam, uint32_t seed, float* photons, uint16_t* adu)
{
   if (!ctx || (n_frames && !frames) || (n_emitters && !emitters))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (cam && !adu)
      return Fail(ISCU_ERR_ARG, "a camera needs an ADU output");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   Lock l(ctx);
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   for (uint32_t k = 0; k < n_frames; ++k)
      if (static_cast<uint64_t>(frames[k].em_start) + frames[k].em_count > n_emitters)
         return Fail(ISCU_ERR_ARG, "frame " + std::to_string(k) + ": emitters beyond the array");
   const size_t px = static_cast<size_t>(ctx->width) * ctx->height * n_frames;
   const size_t emB = static_cast<size_t>(n_emitters) * sizeof(iscu_emitter), frB = n_frames * sizeof(iscu_frame);
   ISCU_CK(ctx->dEmitters.Reserve(emB));
   ISCU_CK(ctx->dFrames.Reserve(frB));
   if (photons)
      ISCU_CK(ctx->dPhotons.Reserve(px * sizeof(float)));
   if (adu)
      ISCU_CK(ctx->dAdu.Reserve(px * sizeof(uint16_t)));
   ISCU_CK(cudaMemcpyAsync(ctx->dEmitters.p, emitters, emB, cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(ctx->dFrames.p, frames, frB, cudaMemcpyHostToDevice, ctx->stream));
   CameraView cv;
   if (cam)
      cv = MakeCameraView(*cam);
   int rc = LaunchRenderFrames(ctx, ctx->dEmitters.as<iscu_emitter>(), n_emitters, ctx->dFrames.as<iscu_frame>(),
                               n_frames, cam ? &cv : nullptr, seed, photons ? ctx->dPhotons.as<float>() : nullptr,
                               adu ? ctx->dAdu.as<uint16_t>() : nullptr);
   if (rc != ISCU_OK)
      return rc;
   if (photons)
      ISCU_CK(cudaMemcpyAsync(photons, ctx->dPhotons.p, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
   if (adu)
      ISCU_CK(cudaMemcpyAsync(adu, ctx->dAdu.p, px * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

int iscu_render_gpu_records(iscu_ctx* ctx, const iscu_gpu_splat_emitter* emitters, uint32_t n_emitters,
                            const iscu_frame* frames, uint32_t n_frames, const float* extras, const iscu_camera* cam,
                            uint32_t seed, uint16_t* adu)
{
   if (!ctx || !cam || !adu || (n_frames && !frames) || (n_emitters && !emitters))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (n_frames > 65535)
      return Fail(ISCU_ERR_LIMIT, "at most 65535 frames per call");
   Lock l(ctx);
   if (!ctx->haveStatic)
      return Fail(ISCU_ERR_STATE, "no camera statics (iscu_set_static)");
   for (uint32_t k = 0; k < n_frames; ++k)
      if (static_cast<uint64_t>(frames[k].em_start) + frames[k].em_count > n_emitters)
         return Fail(ISCU_ERR_ARG, "frame " + std::to_string(k) + ": emitters beyond the array");
   const size_t px = static_cast<size_t>(ctx->width) * ctx->height * n_frames;
   const size_t emB = static_cast<size_t>(n_emitters) * sizeof(iscu_gpu_splat_emitter);
   const size_t frB = n_frames * sizeof(iscu_frame);
   ISCU_CK(ctx->dScratch.Reserve(emB));
   ISCU_CK(ctx->dFrames.Reserve(frB));
   ISCU_CK(ctx->dAdu.Reserve(px * sizeof(uint16_t)));
   if (extras)
      ISCU_CK(ctx->dExtras.Reserve(px * sizeof(float)));
   ISCU_CK(cudaMemcpyAsync(ctx->dScratch.p, emitters, emB, cudaMemcpyHostToDevice, ctx->stream));
   ISCU_CK(cudaMemcpyAsync(ctx->dFrames.p, frames, frB, cudaMemcpyHostToDevice, ctx->stream));
   if (extras)
      ISCU_CK(cudaMemcpyAsync(ctx->dExtras.p, extras, px * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
   const CameraView cv = MakeCameraView(*cam);
   int rc = LaunchRenderGpuRecords(ctx, ctx->dScratch.as<iscu_gpu_splat_emitter>(), ctx->dFrames.as<iscu_frame>(),
                                   n_frames, extras ? ctx->dExtras.as<float>() : nullptr, &cv, seed,
                                   ctx->dAdu.as<uint16_t>());
   if (rc != ISCU_OK)
      return rc;
   ISCU_CK(cudaMemcpyAsync(adu, ctx->dAdu.p, px * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

// ------------------------------------------------------------------------------------------ emitter collection
} // extern "C"

namespace iscu {
namespace {

// One frame's emitters (CollectFrameEmitters, SMLMSimulation.cpp:55-101, then the blink-min-photons filter,
// :152-156) from the events ev(j) for j in [j0, j1), appended to out[n ..]. Returns ISCU_ERR_LIMIT when out is full.
template <class EventAt>
int CollectFrame(const KernelSlot* kernels, int32_t callSlot, EventAt ev, uint32_t j0, uint32_t j1, int64_t frame,
                 uint32_t width, uint32_t height, double pixel_size_nm, double photons_per_blink, double drift_x_px,
                 double drift_y_px, double global_z_offset_um, const float* illum, double min_photons,
                 iscu_emitter* out, uint32_t max_out, uint32_t& n, int64_t* n_clamped)
{
   for (uint32_t j = j0; j < j1; ++j)
   {
      const iscu_blink_event& e = ev(j);
      const int32_t slot = callSlot >= 0 ? callSlot : e.slot;
      if (slot < 0 || slot >= ISCU_MAX_KERNELS || !kernels[slot].valid)
         return Fail(ISCU_ERR_STATE, "event " + std::to_string(j) + ": no kernel stack in its slot");
      const KernelSlot& k = kernels[slot];
      double ov = std::min(static_cast<double>(frame + 1), e.t_end) - std::max(static_cast<double>(frame), e.t_start);
      if (ov <= 0.0)
         continue;
      if (ov > 1.0)
         ov = 1.0;
      const double sitePxX = e.x_um * 1000.0 / pixel_size_nm;
      const double sitePxY = e.y_um * 1000.0 / pixel_size_nm;
      const double xPx = sitePxX + drift_x_px;
      const double yPx = sitePxY + drift_y_px;
      double photons = photons_per_blink * ov;
      if (e.brightness != 1.0)
         photons *= e.brightness;
      if (e.excite != 1.0)
         photons *= e.excite;
      if (illum)
      {
         // IlluminationAt (SMLMBackground.cpp:42-54): bilinear at the undrifted site.
         const double xi = std::max(0.0, std::min(static_cast<double>(width - 1), sitePxX));
         const double yi = std::max(0.0, std::min(static_cast<double>(height - 1), sitePxY));
         const unsigned x0 = std::min(width - 1, static_cast<unsigned>(std::floor(xi)));
         const unsigned y0 = std::min(height - 1, static_cast<unsigned>(std::floor(yi)));
         const unsigned x1 = std::min(width - 1, x0 + 1), y1 = std::min(height - 1, y0 + 1);
         const double fx = xi - x0, fy = yi - y0;
         auto at = [&](unsigned x, unsigned y) { return static_cast<double>(illum[static_cast<size_t>(y) * width + x]); };
         photons *= (at(x0, y0) * (1 - fx) + at(x1, y0) * fx) * (1 - fy) + (at(x0, y1) * (1 - fx) + at(x1, y1) * fx) * fy;
      }
      bool clamped = false;
      const int z = k.NearestZIndex(e.z_nm / 1000.0 - global_z_offset_um, &clamped);
      if (clamped && n_clamped)
         ++*n_clamped;
      if (min_photons > 0.0 && photons < min_photons)
         continue;
      if (n >= max_out)
         return Fail(ISCU_ERR_LIMIT, "emitter output array too small");
      out[n].x_px = xPx;
      out[n].y_px = yPx;
      out[n].photons = photons;
      out[n].plane = z | (slot << 16);
      out[n].reserved = 0;
      ++n;
   }
   return ISCU_OK;
}

} // namespace
} // namespace iscu

extern "C" {

int iscu_collect_frame_emitters(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, uint32_t n_events,
                                int64_t frame, uint32_t width, uint32_t height, double pixel_size_nm,
                                double photons_per_blink, double drift_x_px, double drift_y_px,
                                double global_z_offset_um, const float* illum, double min_photons,
                                iscu_emitter* out, uint32_t max_out, uint32_t* n_out, int64_t* n_clamped)
{
   int rc = slot == -1 ? (ctx ? ISCU_OK : Fail(ISCU_ERR_ARG, "null context")) : CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   if ((n_events && !events) || !n_out || (max_out && !out) || width == 0 || height == 0)
      return Fail(ISCU_ERR_ARG, "null argument or empty frame");
   uint32_t n = 0;
   rc = CollectFrame(ctx->kernels, slot, [&](uint32_t j) -> const iscu_blink_event& { return events[j]; }, 0,
                     n_events, frame, width, height, pixel_size_nm, photons_per_blink, drift_x_px, drift_y_px,
                     global_z_offset_um, illum, min_photons, out, max_out, n, n_clamped);
   *n_out = n;
   return rc;
}

int iscu_collect_emitters(iscu_ctx* ctx, int32_t slot, const iscu_blink_event* events, const uint32_t* bucket_index,
                          const uint32_t* bucket_start, int64_t frame0, uint32_t n_frames, uint32_t width,
                          uint32_t height, double pixel_size_nm, double photons_per_blink, const double* drift_x_px,
                          const double* drift_y_px, const double* global_z_offset_um, const double* bg_scale,
                          const float* illum, double min_photons, iscu_emitter* out, uint32_t max_out,
                          iscu_frame* frames_out, uint32_t* n_out, int64_t* n_clamped)
{
   int rc = slot == -1 ? (ctx ? ISCU_OK : Fail(ISCU_ERR_ARG, "null context")) : CheckSlot(ctx, slot, true);
   if (rc != ISCU_OK)
      return rc;
   if (!bucket_start || !n_out || (n_frames && !frames_out) || (max_out && !out) || width == 0 || height == 0)
      return Fail(ISCU_ERR_ARG, "null argument or empty frame");
   if (bucket_start[n_frames] > bucket_start[0] && !events)
      return Fail(ISCU_ERR_ARG, "null events");
   const KernelSlot* k = ctx->kernels;
   uint32_t n = 0;
   for (uint32_t f = 0; f < n_frames; ++f)
   {
      if (bucket_start[f + 1] < bucket_start[f])
         return Fail(ISCU_ERR_ARG, "bucket offsets must not decrease");
      const uint32_t first = n;
      auto at = [&](uint32_t j) -> const iscu_blink_event& { return events[bucket_index ? bucket_index[j] : j]; };
      rc = CollectFrame(k, slot, at, bucket_start[f], bucket_start[f + 1], frame0 + f, width, height, pixel_size_nm,
                        photons_per_blink, drift_x_px ? drift_x_px[f] : 0.0, drift_y_px ? drift_y_px[f] : 0.0,
                        global_z_offset_um ? global_z_offset_um[f] : 0.0, illum, min_photons, out, max_out, n,
                        n_clamped);
      if (rc != ISCU_OK)
         return rc;
      frames_out[f].em_start = first;
      frames_out[f].em_count = n - first;
      frames_out[f].frame = static_cast<uint32_t>(frame0 + f);
      frames_out[f].reserved = 0;
      frames_out[f].bg_scale = bg_scale ? bg_scale[f] : 1.0;
   }
   *n_out = n;
   return ISCU_OK;
}

} // extern "C"
