// The named-kernel backend (iscu_buffer_*, iscu_dispatch): sim::GpuBackend (WidefieldGpuHost.h:42-77) on CUDA, so that
// the reference's SplatGpuHost (SplatGpu.cpp) and WidefieldGpuHost (WidefieldGpuHost.cpp) run unmodified on the device.
//
// The kernels compute what the reference's WGSL sources define for them (SplatGpu.wgsl splat_frames; WidefieldGpu.wgsl
// wf_clear, wf_scatter, wf_fft, wf_split, wf_mac, wf_expand, wf_crop, wf_frame): the same bindings, parameter words,
// dispatch geometry (one CUDA block per workgroup: 256 threads, or 16 x 16 as 256 with x fastest) and float32
// arithmetic. Where the result is defined only up to rounding the B200 form is its own: wf_fft is a Stockham autosort
// radix-2 transform ping-ponging between two shared-memory arrays (no bit-reversed load), reading the host's twiddle
// table. Integer index arithmetic wraps in 32 bits as WGSL's u32/i32 does.
//
// Robust access, as WebGPU guarantees it: every buffer is passed with its word count, a read out of range gives 0 and a
// write out of range is dropped; loop counts read from buffers are capped by the buffers' sizes (a tile's emitter
// list, a channel's dependency list) or by the WGSL's own caps (Knuth's 1,000 steps, Marsaglia-Tsang's 1,000 tries),
// and a splat record's tap count by its four weights. So no dispatch, however malformed its buffers, faults or hangs.
#include "iscu_internal.h"
#include "counter_rng.cuh"

#include <cuda_fp16.h>

#include <cstring>
#include <string>

struct iscu_buffer
{
   iscu_ctx* ctx = nullptr;
   void* p = nullptr;
   size_t bytes = 0;   // a multiple of 4
};

namespace iscu {
namespace {

constexpr uint32_t kNone = 0xffffffffu;

// A bound storage buffer: 32-bit words and their count.
struct Words
{
   uint32_t* w;
   uint64_t n;
   __device__ __forceinline__ uint32_t Ld(uint32_t i) const { return i < n ? w[i] : 0u; }
   __device__ __forceinline__ float LdF(uint32_t i) const { return __uint_as_float(Ld(i)); }
   __device__ __forceinline__ void St(uint32_t i, uint32_t v) const
   {
      if (i < n)
         w[i] = v;
   }
   // element e of an array of vec2<f32> / vec2<u32> / vec4<u32> (an element out of range reads as zeros)
   __device__ __forceinline__ float2 Ld2(uint32_t e) const
   {
      const uint64_t a = 2ull * e;
      return a + 1 < n ? make_float2(__uint_as_float(w[a]), __uint_as_float(w[a + 1])) : make_float2(0.f, 0.f);
   }
   __device__ __forceinline__ uint2 Ld2u(uint32_t e) const
   {
      const uint64_t a = 2ull * e;
      return a + 1 < n ? make_uint2(w[a], w[a + 1]) : make_uint2(0u, 0u);
   }
   __device__ __forceinline__ uint4 Ld4u(uint32_t e) const
   {
      const uint64_t a = 4ull * e;
      return a + 3 < n ? make_uint4(w[a], w[a + 1], w[a + 2], w[a + 3]) : make_uint4(0u, 0u, 0u, 0u);
   }
   __device__ __forceinline__ void St2(uint32_t e, float2 v) const
   {
      const uint64_t a = 2ull * e;
      if (a + 1 < n)
      {
         w[a] = __float_as_uint(v.x);
         w[a + 1] = __float_as_uint(v.y);
      }
   }
   __device__ __forceinline__ void St2Part(uint32_t e, int comp, float v) const
   {
      const uint64_t a = 2ull * e;
      if (a + 1 < n)
         w[a + comp] = __float_as_uint(v);
   }
   // how many words lie at or after word i (0 past the end)
   __device__ __forceinline__ uint64_t Room(uint32_t i) const { return i < n ? n - i : 0; }
};

// The 64-byte parameter block (binding 0).
struct Block
{
   uint32_t p[16];
   __host__ __device__ float F(int i) const
   {
      float f;
      memcpy(&f, &p[i], 4);
      return f;
   }
};

// 32-bit wrapping signed arithmetic (WGSL's i32).
__device__ __forceinline__ int32_t WAdd(int32_t a, int32_t b)
{
   return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
}
__device__ __forceinline__ int32_t WSub(int32_t a, int32_t b)
{
   return static_cast<int32_t>(static_cast<uint32_t>(a) - static_cast<uint32_t>(b));
}
__device__ __forceinline__ int32_t WMul(int32_t a, int32_t b)
{
   return static_cast<int32_t>(static_cast<uint32_t>(a) * static_cast<uint32_t>(b));
}
__device__ __forceinline__ int32_t WAbs(int32_t a) { return a < 0 ? WSub(0, a) : a; }   // abs(i32 min) = i32 min

__device__ __forceinline__ float2 CMul(float2 a, float2 b)
{
   return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 Conj(float2 a) { return make_float2(a.x, -a.y); }

// ----------------------------------------------------------------------------- the float32 noise chain of the WGSL
// The counter stream of (seed, frame, pixel) in float32 (SplatGpu.wgsl / WidefieldGpu.wgsl uniform01): one pcg4d per
// four words, uniform = (f32(x >> 9) + 0.5) * 2^-23 (exact in float32); then Box-Muller, Knuth Poisson (normal
// approximation above 60), Marsaglia-Tsang Gamma and the sCMOS / EMCCD ADU formulas, all in float32.
struct F32Stream
{
   uint32_t seed, frame, pix, ctr;
   uint32_t q0, q1, q2, q3;
   int k;
   __device__ F32Stream(uint32_t s, uint32_t f, uint32_t p) : seed(s), frame(f), pix(p), ctr(0), q0(0), q1(0), q2(0),
                                                            q3(0), k(4)
   {
   }
   __device__ __forceinline__ float Uniform()
   {
      if (k == 4)
      {
         q0 = seed;
         q1 = frame;
         q2 = pix;
         q3 = ctr;
         Pcg4d(q0, q1, q2, q3);
         ++ctr;
         k = 0;
      }
      const uint32_t x = q0;
      q0 = q1;
      q1 = q2;
      q2 = q3;
      ++k;
      return (static_cast<float>(x >> 9) + 0.5f) * 1.1920928955078125e-7f;
   }
   __device__ float Gauss()
   {
      const float r = sqrtf(-2.0f * logf(Uniform()));
      return r * cosf(6.2831853071795864f * Uniform());
   }
   __device__ float Poisson(float l)
   {
      if (l > 60.0f)
         return fmaxf(0.0f, floorf(l + sqrtf(l) * Gauss() + 0.5f));
      if (!(l > 0.0f))
         return 0.0f;
      const float L = expf(-l);
      int n = 0;
      float p = 1.0f;
      do
      {
         ++n;
         p *= Uniform();
      } while (p > L && n < 1000);
      return static_cast<float>(n - 1);
   }
   __device__ float Gamma(float kk)
   {
      const float d = kk - 1.0f / 3.0f;
      const float c = 1.0f / sqrtf(9.0f * d);
      for (int it = 0; it < 1000; ++it)
      {
         const float x = Gauss();
         const float t = 1.0f + c * x;
         if (t <= 0.0f)
            continue;
         const float v = t * t * t;
         const float w = Uniform();
         if (w < 1.0f - 0.0331f * x * x * x * x)
            return d * v;
         if (logf(w) < 0.5f * x * x + d * (1.0f - v + logf(v)))
            return d * v;
      }
      return d;
   }
};

// Camera parameters of a dispatch (the block words of splat_frames 4..9 / wf_frame 8..13).
struct F32Camera
{
   uint32_t emccd;
   float qe, dark, cic, emGain, maxAdu;
};

// px: offset ADU, gain photons/ADU, read noise e-, (background).
__device__ __forceinline__ uint32_t NoiseAdu(F32Stream& rng, float photons, float4 px, const F32Camera& cam)
{
   float adu;
   if (cam.emccd != 0u)
   {
      const float ne = rng.Poisson(photons * cam.qe + cam.dark + cam.cic);
      float o = 0.0f;
      if (ne > 0.0f)
         o = rng.Gamma(ne);
      adu = floorf(px.x + (o + (px.z / cam.emGain) * rng.Gauss()) / px.y + 0.5f);
      adu = fminf(fmaxf(adu, 0.0f), cam.maxAdu);
   }
   else
   {
      const float ne = rng.Poisson(photons * cam.qe + cam.dark);
      adu = px.x + (ne + px.z * rng.Gauss()) / px.y;
      adu = floorf(fminf(fmaxf(adu, 0.0f), 65535.0f) + 0.5f);
   }
   return __float2uint_rz(adu);   // saturating; NaN -> 0
}

// ----------------------------------------------------------------------------- splat_frames (SplatGpu.wgsl)
// Block words: W, H, NFrames, Seed, Emccd, Qe, Dark, Cic, EmGain, MaxAdu, PixBase, SpanAt, EmAt. Buffers: S0..S3 (block
// sums), Stat (4 words per pixel, then the halo spans from SpanAt), Dyn (kernel table, frames, emitters, extras, tile
// lists), Out (one word of ADU per pixel and frame).
struct SplatRecord   // GpuSplatEmitter (GpuSimD3D11.h:50-59), 16 words
{
   int32_t x0, y0, bx, by, plane, nt;
   float photons;
   int32_t cutR2;
   float wx[4], wy[4];
};

__device__ __forceinline__ float Taps(const Words& S, uint32_t base, int32_t r0, int32_t c0, int32_t bw,
                                      const SplatRecord& em, int nt)
{
   float s = 0.0f;
   for (int j = 0; j < nt; ++j)
   {
      const int32_t r = WAdd(r0, j);
      if (r < 0 || r >= bw)
         continue;
      float row = 0.0f;
      for (int i = 0; i < nt; ++i)
      {
         const int32_t c = WAdd(c0, i);
         if (c >= 0 && c < bw)
            row += em.wx[i] * S.LdF(base + static_cast<uint32_t>(WAdd(WMul(r, bw), c)));
      }
      s += em.wy[j] * row;
   }
   return s;
}

constexpr uint32_t kChunk = 256;

__global__ void __launch_bounds__(256) SplatFramesKernel(Block P, Words S0, Words S1, Words S2, Words S3, Words Stat,
                                                         Words Dyn, Words Out)
{
   __shared__ SplatRecord sEm[kChunk];
   __shared__ uint32_t sStart, sCount;
   const uint32_t li = threadIdx.x;
   const uint32_t X = blockIdx.x * 16u + (li & 15u), Y = blockIdx.y * 16u + (li >> 4);
   const uint32_t W = P.p[0], H = P.p[1];
   const bool inside = X < W && Y < H;
   const uint32_t i = Y * W + X;
   float4 px = make_float4(0.f, 0.f, 1.f, 0.f);
   if (inside)
      px = make_float4(Stat.LdF(4u * i), Stat.LdF(4u * i + 1u), Stat.LdF(4u * i + 2u), Stat.LdF(4u * i + 3u));
   const uint32_t fa = 32u + 8u * blockIdx.z;
   if (li == 0)
   {
      const uint32_t tileAt = Dyn.Ld(fa + 5u);
      const uint32_t t = blockIdx.y * ((W + 15u) / 16u) + blockIdx.x;
      const uint32_t a = Dyn.Ld(tileAt + t);
      uint32_t count = Dyn.Ld(tileAt + t + 1u) - a;
      if (count > Dyn.Room(a))   // the list lies in Dyn
         count = static_cast<uint32_t>(Dyn.Room(a));
      sStart = a;
      sCount = count;
   }
   __syncthreads();
   const uint32_t emCount = sCount, listStart = sStart;
   const uint32_t frame = Dyn.Ld(fa + 2u);
   const float bgScale = Dyn.LdF(fa + 3u);
   const uint32_t extra = Dyn.Ld(fa + 4u);
   const uint32_t emAt = P.p[12], spanAt = P.p[11];

   float acc = px.w * bgScale;
   const int32_t Xi = static_cast<int32_t>(X), Yi = static_cast<int32_t>(Y);
   for (uint32_t e0 = 0; e0 < emCount; e0 += kChunk)
   {
      const uint32_t cnt = min(kChunk, emCount - e0);
      if (li < cnt)
      {
         const uint32_t a = emAt + 16u * Dyn.Ld(listStart + e0 + li);
         SplatRecord r;
         r.x0 = static_cast<int32_t>(Dyn.Ld(a));
         r.y0 = static_cast<int32_t>(Dyn.Ld(a + 1u));
         r.bx = static_cast<int32_t>(Dyn.Ld(a + 2u));
         r.by = static_cast<int32_t>(Dyn.Ld(a + 3u));
         r.plane = static_cast<int32_t>(Dyn.Ld(a + 4u));
         r.nt = static_cast<int32_t>(Dyn.Ld(a + 5u));
         r.photons = Dyn.LdF(a + 6u);
         r.cutR2 = static_cast<int32_t>(Dyn.Ld(a + 7u));
         for (int k = 0; k < 4; ++k)
         {
            r.wx[k] = Dyn.LdF(a + 8u + k);
            r.wy[k] = Dyn.LdF(a + 12u + k);
         }
         sEm[li] = r;
      }
      __syncthreads();
      if (inside)
         for (uint32_t k = 0; k < cnt; ++k)
         {
            const SplatRecord& em = sEm[k];
            const uint32_t kk = static_cast<uint32_t>(em.plane) >> 16;
            const int32_t camRad = static_cast<int32_t>(Dyn.Ld(4u * kk)), os = static_cast<int32_t>(Dyn.Ld(4u * kk + 1u));
            const int32_t bw = static_cast<int32_t>(Dyn.Ld(4u * kk + 2u)), off = static_cast<int32_t>(Dyn.Ld(4u * kk + 3u));
            const int32_t dx = WSub(Xi, em.x0), dy = WSub(Yi, em.y0);
            if (WAbs(dx) > camRad || WAbs(dy) > camRad)
               continue;
            if (WAdd(WMul(dx, dx), WMul(dy, dy)) > em.cutR2)
               continue;
            const uint32_t stride = Dyn.Ld(16u + 4u * kk), spansOn = Dyn.Ld(17u + 4u * kk);
            const uint32_t span0 = Dyn.Ld(18u + 4u * kk), buf = Dyn.Ld(19u + 4u * kk);
            const uint32_t plane = static_cast<uint32_t>(em.plane) & 0xffffu;
            if (spansOn != 0u)
            {
               const uint32_t sa = spanAt + 2u * (span0 + plane * static_cast<uint32_t>(WAdd(WMul(2, camRad), 1)) +
                                                  static_cast<uint32_t>(WAdd(dy, camRad)));
               if (dx < static_cast<int32_t>(Stat.Ld(sa)) || dx > static_cast<int32_t>(Stat.Ld(sa + 1u)))
                  continue;
            }
            const int32_t r0 = WAdd(WAdd(em.by, WMul(dy, os)), off);
            const int32_t c0 = WAdd(WAdd(em.bx, WMul(dx, os)), off);
            const uint32_t base = plane * stride;
            const int nt = min(max(em.nt, 0), 4);   // four weights per axis
            const Words S{buf == 0u ? S0.w : buf == 1u ? S1.w : buf == 2u ? S2.w : S3.w,
                          buf == 0u ? S0.n : buf == 1u ? S1.n : buf == 2u ? S2.n : S3.n};
            acc += em.photons * Taps(S, base, r0, c0, bw, em, nt);
         }
      __syncthreads();
   }
   if (!inside)
      return;
   if (extra != kNone)
      acc += Dyn.LdF(extra + i);
   F32Stream rng(P.p[3], frame, P.p[10] + i);
   const F32Camera cam{P.p[4], P.F(5), P.F(6), P.F(7), P.F(8), P.F(9)};
   Out.St(blockIdx.z * W * H + i, NoiseAdu(rng, fmaxf(acc, 0.0f), px, cam));
}

// ----------------------------------------------------------------------------- the widefield kernels (WidefieldGpu.wgsl)
__device__ __forceinline__ uint32_t Flat256(uint32_t rowLen)
{
   return blockIdx.x * 256u + threadIdx.x + blockIdx.y * rowLen;
}

// wf_clear: {count, rowLen}; data (vec2<f32>).
__global__ void __launch_bounds__(256) WfClearKernel(Block P, Words data)
{
   const uint32_t i = Flat256(P.p[1]);
   if (i < P.p[0])
      data.St2(i, make_float2(0.f, 0.f));
}

// wf_scatter: {count, nx, NX, planeStride, rowLen}; entries (vec4<u32>: grid slot, cell, value bits, component), data.
__global__ void __launch_bounds__(256) WfScatterKernel(Block P, Words entries, Words data)
{
   const uint32_t i = Flat256(P.p[4]);
   if (i >= P.p[0])
      return;
   const uint4 e = entries.Ld4u(i);
   const uint32_t nx = P.p[1];
   const uint32_t x = e.y % nx, y = e.y / nx;
   const uint32_t idx = e.x * P.p[3] + y * P.p[2] + x;
   data.St2Part(idx, e.w == 0u ? 0 : 1, __uint_as_float(e.z));
}

// wf_fft: {n, logn, elemStride, xfStride, planeStride, inverse, twOff}; data, tw (n / 2 twiddles exp(-2 pi i k / n)
// at twOff). Transform blockIdx.x of plane blockIdx.z, elements base + i * elemStride, in place, no scaling. Stockham
// autosort: stage s (span m = n >> (s + 1), stride 2^s) maps x[q + 2^s p], x[q + 2^s (p + m)] to
// y[q + 2^s 2p] = a + b, y[q + 2^s (2p + 1)] = (a - b) w^(p 2^s); the result lands in natural order.
__global__ void __launch_bounds__(256) WfFftKernel(Block P, Words data, Words tw)
{
   __shared__ float2 buf[2][2048];
   const uint32_t n = P.p[0], logn = P.p[1], elemStride = P.p[2];
   const uint32_t base = blockIdx.z * P.p[4] + blockIdx.x * P.p[3];
   const bool inverse = P.p[5] != 0u;
   const uint32_t twOff = P.p[6];
   for (uint32_t i = threadIdx.x; i < n; i += 256u)
      buf[0][i] = data.Ld2(base + i * elemStride);
   __syncthreads();
   int src = 0;
   const uint32_t half = n >> 1;
   for (uint32_t s = 0; s < logn; ++s)
   {
      const float2* x = buf[src];
      float2* y = buf[src ^ 1];
      const uint32_t mask = (1u << s) - 1u;
      for (uint32_t j = threadIdx.x; j < half; j += 256u)
      {
         const uint32_t q = j & mask, p = j >> s;
         const float2 a = x[j], b = x[j + half];   // q + 2^s p = j; q + 2^s (p + m) = j + n / 2
         float2 w = tw.Ld2(twOff + (j & ~mask));    // exp(-2 pi i p 2^s / n)
         if (inverse)
            w.y = -w.y;
         const uint32_t o = q + (p << (s + 1));
         y[o] = make_float2(a.x + b.x, a.y + b.y);
         y[o + (1u << s)] = CMul(make_float2(a.x - b.x, a.y - b.y), w);
      }
      __syncthreads();
      src ^= 1;
   }
   for (uint32_t i = threadIdx.x; i < n; i += 256u)
      data.St2(base + i * elemStride, buf[src][i]);
}

__device__ __forceinline__ uint32_t PackHalf2(float2 v)
{
   const __half2 h = __floats2half2_rn(v.x, v.y);
   uint32_t u;
   memcpy(&u, &h, 4);
   return u;
}
__device__ __forceinline__ float2 UnpackHalf2(uint32_t u)
{
   __half2 h;
   memcpy(&h, &u, 4);
   return __half22float2(h);
}

// wf_split: {NX, NY, W, SS, PS, pairs}; data, slots (vec4<u32>: slot A, slot B or none, 1/scale A, 1/scale B), spec.
__global__ void __launch_bounds__(256) WfSplitKernel(Block P, Words data, Words slots, Words spec)
{
   const uint32_t kx = blockIdx.x * 16u + (threadIdx.x & 15u), ky = blockIdx.y * 16u + (threadIdx.x >> 4);
   const uint32_t NX = P.p[0], NY = P.p[1], Wd = P.p[2], SS = P.p[3];
   if (kx >= Wd || ky >= NY)
      return;
   const uint32_t z = blockIdx.z, base = z * P.p[4];
   const float2 zk = data.Ld2(base + ky * NX + kx);
   const float2 zm = Conj(data.Ld2(base + ((NY - ky) % NY) * NX + (NX - kx) % NX));
   const uint4 s = slots.Ld4u(z);
   const uint32_t bin = ky * Wd + kx;
   const float2 a = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
   const float sa = __uint_as_float(s.z);
   spec.St(s.x * SS + bin, PackHalf2(make_float2(a.x * sa, a.y * sa)));
   if (s.y != kNone)
   {
      const float2 d = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
      const float sb = __uint_as_float(s.w);
      spec.St(s.y * SS + bin, PackHalf2(make_float2(d.y * sb, -d.x * sb)));   // (Zk - conj Zm) / 2i
   }
}

// wf_mac: {SS, nChan, rowLen}; spec (fp16 pairs), kspec (vec2<f32>), depI (vec4<u32>: plane slot, k0, k1 or none,
// scale bits), depW (vec2<f32>), chans (vec2<u32>: first dep, count), out (vec2<f32>).
__global__ void __launch_bounds__(256) WfMacKernel(Block P, Words spec, Words kspec, Words depI, Words depW,
                                                   Words chans, Words out)
{
   const uint32_t SS = P.p[0];
   const uint32_t bin = Flat256(P.p[2]);
   if (bin >= SS)
      return;
   const uint2 c = chans.Ld2u(blockIdx.z);
   const uint64_t nDeps = depI.n / 4;
   const uint64_t want = static_cast<uint64_t>(c.x) + c.y;
   const uint64_t end = want < nDeps ? want : nDeps;   // the list lies in depI
   float2 acc = make_float2(0.f, 0.f);
   for (uint64_t d = c.x; d < end; ++d)
   {
      const uint4 di = depI.Ld4u(static_cast<uint32_t>(d));
      const float2 dw = depW.Ld2(static_cast<uint32_t>(d));
      const float2 u = UnpackHalf2(spec.Ld(di.x * SS + bin));
      const float sc = __uint_as_float(di.w);
      const float2 a = make_float2(u.x * sc, u.y * sc);
      const float2 k0 = kspec.Ld2(di.y * SS + bin);
      float2 k = make_float2(dw.x * k0.x, dw.x * k0.y);
      if (di.z != kNone)
      {
         const float2 k1 = kspec.Ld2(di.z * SS + bin);
         k = make_float2(k.x + dw.y * k1.x, k.y + dw.y * k1.y);
      }
      const float2 m = CMul(a, k);
      acc = make_float2(acc.x + m.x, acc.y + m.y);
   }
   out.St2(blockIdx.z * SS + bin, acc);
}

// wf_expand: {NX, NY, W, SS, PS, pairs, fracX, fracY}; chan (vec2<f32> half spectra), pairs (vec2<u32>), data.
__global__ void __launch_bounds__(256) WfExpandKernel(Block P, Words chan, Words pairs, Words data)
{
   const uint32_t x = blockIdx.x * 16u + (threadIdx.x & 15u), y = blockIdx.y * 16u + (threadIdx.x >> 4);
   const uint32_t NX = P.p[0], NY = P.p[1], Wd = P.p[2], SS = P.p[3];
   if (x >= NX || y >= NY)
      return;
   const uint2 pr = pairs.Ld2u(blockIdx.z);
   auto halfBin = [&](uint32_t c) -> float2 {
      if (x < Wd)
         return chan.Ld2(c * SS + y * Wd + x);
      return Conj(chan.Ld2(c * SS + ((NY - y) % NY) * Wd + (NX - x)));
   };
   float kx = static_cast<float>(x), ky = static_cast<float>(y);
   if (x > NX / 2u)
      kx = kx - static_cast<float>(NX);
   if (y > NY / 2u)
      ky = ky - static_cast<float>(NY);
   const float ax = 6.2831853071795864f * kx * P.F(6) / static_cast<float>(NX);
   const float ay = 6.2831853071795864f * ky * P.F(7) / static_cast<float>(NY);
   float2 px = make_float2(cosf(ax), sinf(ax));
   if (x == NX / 2u)
      px.y = 0.0f;
   float2 py = make_float2(cosf(ay), sinf(ay));
   if (y == NY / 2u)
      py.y = 0.0f;
   const float2 ph = CMul(px, py);
   const float2 s1 = CMul(halfBin(pr.x), ph);
   float2 z = s1;
   if (pr.y != kNone)
   {
      const float2 s2 = CMul(halfBin(pr.y), ph);
      z = make_float2(s1.x - s2.y, s1.y + s2.x);
   }
   data.St2(blockIdx.z * P.p[4] + y * NX + x, z);
}

// wf_crop: {NX, PS, fovX0, fovY0, cw, ch, scale}; data, pairs, imgs (f32).
__global__ void __launch_bounds__(256) WfCropKernel(Block P, Words data, Words pairs, Words imgs)
{
   const uint32_t gx = blockIdx.x * 16u + (threadIdx.x & 15u), gy = blockIdx.y * 16u + (threadIdx.x >> 4);
   const uint32_t cw = P.p[4], ch = P.p[5];
   if (gx >= cw || gy >= ch)
      return;
   const uint2 pr = pairs.Ld2u(blockIdx.z);
   const float sc = P.F(6);
   const float2 v0 = data.Ld2(blockIdx.z * P.p[1] + (P.p[3] + gy) * P.p[0] + P.p[2] + gx);
   const uint32_t i = gy * cw + gx, cs = cw * ch;
   imgs.St(pr.x * cs + i, __float_as_uint(v0.x * sc));
   if (pr.y != kNone)
      imgs.St(pr.y * cs + i, __float_as_uint(v0.y * sc));
}

// wf_frame: {W, H, cw, u, nB, hasP, nFrames, seed, emccd, qe, dark, cic, emGain, maxAdu}; imgs (f32), coef (f32),
// frames (vec2<u32>: frame id, background scale bits), pix (vec4<f32>: offset, gain, read noise, background), out.
__global__ void __launch_bounds__(256) WfFrameKernel(Block P, Words imgs, Words coef, Words frames, Words pix,
                                                     Words out)
{
   const uint32_t gx = blockIdx.x * 16u + (threadIdx.x & 15u), gy = blockIdx.y * 16u + (threadIdx.x >> 4);
   const uint32_t W = P.p[0], H = P.p[1], cw = P.p[2], u = P.p[3], nB = P.p[4], hasP = P.p[5];
   if (gx >= W || gy >= H || blockIdx.z >= P.p[6])
      return;
   const uint32_t i = gy * W + gx;
   const float4 px = make_float4(pix.LdF(4u * i), pix.LdF(4u * i + 1u), pix.LdF(4u * i + 2u), pix.LdF(4u * i + 3u));
   const uint2 fr = frames.Ld2u(blockIdx.z);
   const uint32_t cs = cw * (H * u);
   const uint32_t nBc = static_cast<uint64_t>(nB) < coef.n ? nB : static_cast<uint32_t>(coef.n);   // coefficients held
   float dyes = 0.0f;
   for (uint32_t sy = 0; sy < u; ++sy)
      for (uint32_t sx = 0; sx < u; ++sx)
      {
         const uint32_t c = (gy * u + sy) * cw + gx * u + sx;
         float v = 0.0f;
         if (hasP != 0u)
            v = imgs.LdF(c);
         for (uint32_t j = 0; j < nBc; ++j)
            v = v + coef.LdF(blockIdx.z * nB + j) * imgs.LdF((hasP + j) * cs + c);
         dyes = dyes + fmaxf(0.0f, v);
      }
   const float photons = fmaxf(px.w * __uint_as_float(fr.y) + dyes, 0.0f);
   F32Stream rng(P.p[7], fr.x, i);
   const F32Camera cam{P.p[8], P.F(9), P.F(10), P.F(11), P.F(12), P.F(13)};
   out.St(blockIdx.z * W * H + i, NoiseAdu(rng, photons, px, cam));
}

// The low 16 bits of n words (ReadBackLow16), on the device.
__global__ void Low16Kernel(const uint32_t* __restrict__ in, size_t n, uint16_t* __restrict__ out)
{
   for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
        i += static_cast<size_t>(gridDim.x) * blockDim.x)
      out[i] = static_cast<uint16_t>(in[i]);
}

// ----------------------------------------------------------------------------- dispatch
enum KernelId
{
   kSplatFrames,
   kWfClear,
   kWfScatter,
   kWfFft,
   kWfSplit,
   kWfMac,
   kWfExpand,
   kWfCrop,
   kWfFrame,
   kKernels
};

struct KernelInfo
{
   const char* name;
   int buffers;
};

constexpr KernelInfo kInfo[kKernels] = {{"splat_frames", 7}, {"wf_clear", 1},  {"wf_scatter", 2},
                                        {"wf_fft", 2},       {"wf_split", 3},  {"wf_mac", 6},
                                        {"wf_expand", 3},    {"wf_crop", 3},   {"wf_frame", 5}};

Words View(const iscu_buffer* b) { return Words{static_cast<uint32_t*>(b->p), b->bytes / 4}; }

// Parameters a kernel cannot run with (the rest is the buffers' business: robust access).
int CheckParams(int id, const Block& P)
{
   switch (id)
   {
   case kWfFft:
   {
      const uint32_t n = P.p[0], logn = P.p[1];
      if (logn < 1 || logn > 11 || n != (1u << logn))
         return Fail(ISCU_ERR_ARG, "wf_fft: n must be 2^logn, 2 <= n <= 2048");
      return ISCU_OK;
   }
   case kWfScatter:
      if (P.p[1] == 0)
         return Fail(ISCU_ERR_ARG, "wf_scatter: nx must be > 0");
      return ISCU_OK;
   case kWfSplit:
   case kWfExpand:
      if (P.p[0] == 0 || P.p[1] == 0)
         return Fail(ISCU_ERR_ARG, "the grid's NX and NY must be > 0");
      return ISCU_OK;
   case kWfFrame:
      if (P.p[3] > 64)
         return Fail(ISCU_ERR_ARG, "wf_frame: upscale above 64");
      if (P.p[4] > 65536)
         return Fail(ISCU_ERR_ARG, "wf_frame: more than 65536 bleach maps");
      return ISCU_OK;
   default:
      return ISCU_OK;
   }
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_buffer_create(iscu_ctx* ctx, size_t bytes, const void* data, iscu_buffer** out)
{
   if (!ctx || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const size_t rounded = ((bytes + 3) / 4) * 4;
   std::unique_ptr<iscu_buffer> b(new iscu_buffer());
   b->ctx = ctx;
   b->bytes = rounded;
   ISCU_CK(cudaMallocAsync(&b->p, rounded ? rounded : 4, ctx->stream));
   if (data && bytes)
   {
      cudaError_t e = cudaMemcpyAsync(b->p, data, bytes, cudaMemcpyHostToDevice, ctx->stream);
      if (e == cudaSuccess && rounded > bytes)
         e = cudaMemsetAsync(static_cast<char*>(b->p) + bytes, 0, rounded - bytes, ctx->stream);
      if (e == cudaSuccess)
         e = cudaStreamSynchronize(ctx->stream);   // the caller's memory is free to reuse on return
      if (e != cudaSuccess)
      {
         cudaFreeAsync(b->p, ctx->stream);
         return CudaFail(e, "iscu_buffer_create upload");
      }
   }
   else if (rounded)
   {
      cudaError_t e = cudaMemsetAsync(b->p, 0, rounded, ctx->stream);
      if (e != cudaSuccess)
      {
         cudaFreeAsync(b->p, ctx->stream);
         return CudaFail(e, "iscu_buffer_create clear");
      }
   }
   *out = b.release();
   return ISCU_OK;
}

void iscu_buffer_destroy(iscu_buffer* buf)
{
   if (!buf)
      return;
   {
      std::lock_guard<std::recursive_mutex> lock(buf->ctx->mu);
      cudaFreeAsync(buf->p, buf->ctx->stream);   // after the work already queued on the stream
   }
   delete buf;
}

size_t iscu_buffer_bytes(const iscu_buffer* buf) { return buf ? buf->bytes : 0; }

int iscu_buffer_write(iscu_buffer* buf, size_t offset, const void* data, size_t bytes)
{
   if (!buf || (bytes && !data))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (offset > buf->bytes || bytes > buf->bytes - offset)
      return Fail(ISCU_ERR_ARG, "write past the buffer's end");
   std::lock_guard<std::recursive_mutex> lock(buf->ctx->mu);
   ClearError();
   if (!bytes)
      return ISCU_OK;
   ISCU_CK(cudaMemcpyAsync(static_cast<char*>(buf->p) + offset, data, bytes, cudaMemcpyHostToDevice,
                           buf->ctx->stream));
   ISCU_CK(cudaStreamSynchronize(buf->ctx->stream));
   return ISCU_OK;
}

int iscu_buffer_copy(iscu_buffer* dst, const iscu_buffer* src, size_t bytes)
{
   if (!dst || !src)
      return Fail(ISCU_ERR_ARG, "null argument");
   if (dst->ctx != src->ctx)
      return Fail(ISCU_ERR_ARG, "buffers of two contexts");
   if (bytes > dst->bytes || bytes > src->bytes)
      return Fail(ISCU_ERR_ARG, "copy past a buffer's end");
   std::lock_guard<std::recursive_mutex> lock(dst->ctx->mu);
   ClearError();
   if (bytes)
      ISCU_CK(cudaMemcpyAsync(dst->p, src->p, bytes, cudaMemcpyDeviceToDevice, dst->ctx->stream));
   return ISCU_OK;
}

int iscu_buffer_read(const iscu_buffer* src, size_t bytes, void* dst)
{
   if (!src || (bytes && !dst))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (bytes > src->bytes)
      return Fail(ISCU_ERR_ARG, "read past the buffer's end");
   std::lock_guard<std::recursive_mutex> lock(src->ctx->mu);
   ClearError();
   if (bytes)
      ISCU_CK(cudaMemcpyAsync(dst, src->p, bytes, cudaMemcpyDeviceToHost, src->ctx->stream));
   ISCU_CK(cudaStreamSynchronize(src->ctx->stream));
   return ISCU_OK;
}

int iscu_buffer_read_low16(const iscu_buffer* src, size_t words, uint16_t* dst)
{
   if (!src || (words && !dst))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (words > src->bytes / 4)
      return Fail(ISCU_ERR_ARG, "read past the buffer's end");
   iscu_ctx* ctx = src->ctx;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (words)
   {
      ISCU_CK(ctx->dLow16.Reserve(words * sizeof(uint16_t)));
      const unsigned blocks = static_cast<unsigned>(std::min<size_t>((words + 255) / 256, 8u * ctx->smCount));
      Low16Kernel<<<blocks, 256, 0, ctx->stream>>>(static_cast<const uint32_t*>(src->p), words,
                                                     ctx->dLow16.as<uint16_t>());
      ISCU_CK_LAUNCH(ctx, "Low16Kernel");
      ISCU_CK(cudaMemcpyAsync(dst, ctx->dLow16.p, words * sizeof(uint16_t), cudaMemcpyDeviceToHost, ctx->stream));
   }
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   return ISCU_OK;
}

int iscu_dispatch(iscu_ctx* ctx, const char* kernel, const uint32_t* params, size_t n_params,
                  iscu_buffer* const* bufs, size_t n_bufs, uint32_t x, uint32_t y, uint32_t z)
{
   if (!ctx || !kernel || (n_params && !params) || (n_bufs && !bufs))
      return Fail(ISCU_ERR_ARG, "null argument");
   int id = 0;
   while (id < kKernels && std::strcmp(kInfo[id].name, kernel) != 0)
      ++id;
   if (id == kKernels)
      return Fail(ISCU_ERR_ARG, std::string("no kernel named ") + kernel);
   if (n_params > 16)
      return Fail(ISCU_ERR_ARG, "a parameter block holds 16 words");
   if (n_bufs != static_cast<size_t>(kInfo[id].buffers))
      return Fail(ISCU_ERR_ARG, std::string(kernel) + " binds " + std::to_string(kInfo[id].buffers) + " buffers, not " +
                                    std::to_string(n_bufs));
   Words w[8];
   for (size_t b = 0; b < n_bufs; ++b)
   {
      if (!bufs[b])
         return Fail(ISCU_ERR_ARG, "null buffer");
      if (bufs[b]->ctx != ctx)
         return Fail(ISCU_ERR_ARG, "a buffer of another context");
      w[b] = View(bufs[b]);
   }
   if (y > 65535 || z > 65535 || x > 0x7fffffffu)
      return Fail(ISCU_ERR_LIMIT, "at most 2^31 - 1 x 65535 x 65535 workgroups");
   Block P;
   std::memset(&P, 0, sizeof P);
   if (n_params)
      std::memcpy(P.p, params, n_params * 4);
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   const int rc = CheckParams(id, P);
   if (rc != ISCU_OK)
      return rc;
   if (x == 0 || y == 0 || z == 0)
      return ISCU_OK;   // an empty dispatch
   const dim3 grid(x, y, z);
   cudaStream_t s = ctx->stream;
   switch (id)
   {
   case kSplatFrames:
      SplatFramesKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2], w[3], w[4], w[5], w[6]);
      break;
   case kWfClear:
      WfClearKernel<<<grid, 256, 0, s>>>(P, w[0]);
      break;
   case kWfScatter:
      WfScatterKernel<<<grid, 256, 0, s>>>(P, w[0], w[1]);
      break;
   case kWfFft:
      WfFftKernel<<<grid, 256, 0, s>>>(P, w[0], w[1]);
      break;
   case kWfSplit:
      WfSplitKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2]);
      break;
   case kWfMac:
      WfMacKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2], w[3], w[4], w[5]);
      break;
   case kWfExpand:
      WfExpandKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2]);
      break;
   case kWfCrop:
      WfCropKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2]);
      break;
   case kWfFrame:
      WfFrameKernel<<<grid, 256, 0, s>>>(P, w[0], w[1], w[2], w[3], w[4]);
      break;
   default:
      break;
   }
   ISCU_CK_LAUNCH(ctx, kernel);
   return ISCU_OK;
}

} // extern "C"
