// The tcgen05 / mbarrier / bulk-copy building blocks of the chirp-Z tensor-core kernels (psf_tc.cu: TF32 x 3;
// psf_tc16.cu: FP16 x 3), and the pupil phasor both compute from the per-set phase tables.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace iscu {
namespace tc {

constexpr uint64_t kWaitNs = 4000000000ull;   // a wait gives up after 4 s

__device__ __forceinline__ uint32_t SmemAddr(const void* p)
{
   return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count)
{
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count));
}

__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void TcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void TcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: canonical K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t addr)
{
   uint64_t d = 0;
   d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);          // start address
   d |= static_cast<uint64_t>(1u) << 16;                       // leading byte offset (unused for this layout)
   d |= static_cast<uint64_t>(1024u >> 4) << 32;               // stride byte offset: 8-row group pitch
   d |= static_cast<uint64_t>(1u) << 46;                       // descriptor version (sm_100)
   d |= static_cast<uint64_t>(2u) << 61;                       // layout: 128-byte swizzle
   return d;
}

__device__ __forceinline__ void Commit(uint64_t* bar)
{
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(bar))
                : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes into v[0..31] (thread = lane).
__device__ __forceinline__ void TmemLoad32(uint32_t taddr, float* v)
{
   uint32_t r[32];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 32; ++i)
      v[i] = __uint_as_float(r[i]);
}

// The pupil phasor of one sample from the phase table: the float64 phase x = base + a opd3F, reduced mod 2 pi as
// x - 2 pi n with n = rint(x / 2 pi) (formed by adding and taking away 1.5 2^52, exact for |x / 2 pi| < 2^51) and
// 2 pi's float64 value (its remaining 2.4e-16 times n is far below float32's resolution for these phases), then the
// float32 sine and cosine of the reduced phase by the special-function unit (absolute error ~4e-7 over [-pi, pi]).
// Branch-free, so a thread's samples interleave: outside the aperture (opd3F < 0) the entry (0, -1) gives a finite
// phase, zeroed at the end.
__device__ __forceinline__ float2 TablePhasor(double2 t, double a)
{
   const double x = fma(a, t.y, t.x);
   const double kRound = 6755399441055744.0;   // 1.5 2^52
   const double n = fma(x, 0.15915494309189533577, kRound) - kRound;
   const float r = static_cast<float>(fma(-n, 6.283185307179586232, x));
   float sn, cs;
   __sincosf(r, &sn, &cs);
   const bool in = t.y >= 0.0;
   return make_float2(in ? cs : 0.f, in ? sn : 0.f);
}

__device__ __forceinline__ void MbarExpectTx(uint64_t* bar, uint32_t bytes)
{
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)), "r"(bytes)
                : "memory");
}

// A bulk copy global -> this CTA's shared memory (no multicast), completing `bytes` on the mbarrier.
__device__ __forceinline__ void BulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   SmemAddr(dst)),
                "l"(src), "r"(bytes), "r"(SmemAddr(bar))
                : "memory");
}

__device__ __forceinline__ uint64_t GlobalNs()
{
   uint64_t t;
   asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
   return t;
}

// Waits for the phase of the given parity to complete. false after kWaitNs, or (err non-null) once *err is set.
// backoff: after a few polls the thread sleeps between polls, leaving its scheduler's issue slots to the warps that
// share it (the MMA thread polls without it: its waits are on the critical path).
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity, const volatile int* err, bool backoff = true)
{
   const uint32_t a = SmemAddr(bar);
   uint64_t t0 = 0;
   for (unsigned it = 0;; ++it)
   {
      uint32_t done;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done)
                   : "r"(a), "r"(parity)
                   : "memory");
      if (done)
         return true;
      if (backoff && it >= 2)
         __nanosleep(it < 16 ? 32 : 128);
      if ((it & 15) == 15)
      {
         if (err && *err)
            return false;
         const uint64_t now = GlobalNs();
         if (t0 == 0)
            t0 = now;
         else if (now - t0 > kWaitNs)
            return false;
      }
   }
}

__device__ __forceinline__ void MbarArrive(uint64_t* bar)
{
   asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

// 16 consecutive TMEM columns of this warp's 32 lanes into v[0..15].
__device__ __forceinline__ void TmemLoad16(uint32_t taddr, float* v)
{
   uint32_t r[16];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 16; ++i)
      v[i] = __uint_as_float(r[i]);
}

// v[0..31] into 32 consecutive TMEM columns of this warp's 32 lanes (thread = lane); the caller waits with
// TmemWaitStore before another thread may rely on them.
__device__ __forceinline__ void TmemStore32(uint32_t taddr, const uint32_t* v)
{
   asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
                "%32};" ::"r"(taddr),
                "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
                "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
                "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
                "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
                : "memory");
}

__device__ __forceinline__ void TmemWaitStore() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

} // namespace tc
} // namespace iscu
