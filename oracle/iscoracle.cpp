// TEST INFRASTRUCTURE -- the oracle. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
// as the checker; the product (insiliscope_b200, libiscu.so) never links, loads or calls it.
//
// A CPU restatement of inSiliScope's image-formation path, written from the reference's algorithm (each function
// cites the reference file:line it follows), compiled with -ffp-contract=off like the reference. Where the reference
// computes in float64 this does too, in the same order, so its integer and float outputs are the reference's bit for
// bit; the PSF is restated as the direct float64 DFT (E = A U A^T) that the reference's Bluestein chirp-Z evaluates.
// Pinned against the reference's golden vectors (spec/golden/ref.txt rng/stream lines), its PSF fixture
// (tests/psf/zernike_ref.bin) and the reference's own functions built here (oracle/_ref): tests/test_oracle.py.
#include "../include/iscu.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

// pcg4d: four 32-bit LCG lanes, two rounds of cross-multiplies around a 16-bit xorshift
// (adapter/inSiliScope/Simulation/SMLMCounterRng.h:37-56; core/src/rng.h:18-33).
void Pcg(uint32_t v[4])
{
   for (int i = 0; i < 4; ++i)
      v[i] = v[i] * 1664525u + 1013904223u;
   v[0] += v[1] * v[3];
   v[1] += v[2] * v[0];
   v[2] += v[0] * v[1];
   v[3] += v[1] * v[2];
   for (int i = 0; i < 4; ++i)
      v[i] ^= v[i] >> 16;
   v[0] += v[1] * v[3];
   v[1] += v[2] * v[0];
   v[2] += v[0] * v[1];
   v[3] += v[1] * v[2];
}

double UnitOf(uint32_t x) { return (static_cast<double>(x >> 9) + 0.5) * (1.0 / 8388608.0); }

// A pixel's uniform stream: hash (seed, frame, pixel, counter), four uniforms per hash (SMLMCounterRng.h:60-91).
struct Stream
{
   uint32_t seed, frame, pixel, counter = 0, word[4] = {0, 0, 0, 0};
   int used = 4;
   Stream(uint32_t s, uint32_t f, uint32_t p) : seed(s), frame(f), pixel(p) {}
   double Next()
   {
      if (used == 4)
      {
         word[0] = seed;
         word[1] = frame;
         word[2] = pixel;
         word[3] = counter++;
         Pcg(word);
         used = 0;
      }
      return UnitOf(word[used++]);
   }
};

// Box-Muller, radius then angle (SMLMCounterRng.h:95-100).
double Normal(Stream& s)
{
   const double u1 = s.Next();
   const double r = std::sqrt(-2.0 * std::log(u1));
   const double u2 = s.Next();
   return r * std::cos(6.283185307179586 * u2);
}

// Knuth below mean 60, rounded normal above, at most 1000 factors (SMLMCounterRng.h:102-118).
double Poisson(double mean, Stream& s)
{
   if (mean > 60.0)
   {
      const double g = Normal(s);
      const double v = std::floor(mean + std::sqrt(mean) * g + 0.5);
      return v > 0.0 ? v : 0.0;
   }
   if (!(mean > 0.0))
      return 0.0;
   const double limit = std::exp(-mean);
   double prod = 1.0;
   int k = 0;
   while (true)
   {
      ++k;
      prod *= s.Next();
      if (!(prod > limit) || k >= 1000)
         break;
   }
   return k - 1.0;
}

// Marsaglia-Tsang Gamma(shape, 1), at most 1000 rounds (SMLMCounterRng.h:120-136).
double GammaDraw(double shape, Stream& s)
{
   const double d = shape - 1.0 / 3.0;
   const double c = 1.0 / std::sqrt(9.0 * d);
   for (int round = 0; round < 1000; ++round)
   {
      const double x = Normal(s);
      const double t = 1.0 + c * x;
      if (t <= 0.0)
         continue;
      const double v = t * t * t;
      const double w = s.Next();
      const double x2 = x * x;
      if (w < 1.0 - 0.0331 * x * x * x * x)
         return d * v;
      if (std::log(w) < 0.5 * x2 + d * (1.0 - v + std::log(v)))
         return d * v;
   }
   return d;
}

// Box-Muller on a std::mt19937_64 for the static maps (SMLMNoise.cpp:17-35).
double MapNormal(std::mt19937_64& g)
{
   std::uniform_real_distribution<double> u(0.0, 1.0);
   double a = u(g);
   if (a < 1e-300)
      a = 1e-300;
   const double b = u(g);
   return std::sqrt(-2.0 * std::log(a)) * std::cos(2.0 * kPi * b);
}

// ------------------------------------------------------------------------------------------ PSF (float64 DFT)
struct Geometry
{
   int size, nz, M, os, halfOv;
   double resLatNm;
};

Geometry Geo(const iscu_psf_request& r)
{
   // ZernikePsf.cpp:118-158.
   Geometry g;
   g.os = std::max(1, r.oversampling);
   const int half = std::max(1, r.kernel_half_width_px);
   g.halfOv = half * g.os;
   g.size = 2 * g.halfOv + 1;
   const int nzw = std::max(3, r.nz);
   g.nz = nzw | 1;
   g.resLatNm = r.pixel_size_nm / g.os;
   if (r.pupil_samples > 0)
      g.M = std::min(1024, std::max(8, static_cast<int>(r.pupil_samples)));
   else
   {
      const double diag = 2.0 * std::sqrt(2.0) * half * r.pixel_size_nm / 1000.0;
      const double m = 4.0 + 2.0 * r.na * diag / (r.wavelength_nm / 1000.0);
      const int need = std::max(64, std::min(512, 4 * static_cast<int>(std::ceil(m / 4.0))));
      int L = 1;
      while (L < need + g.size - 1)
         L *= 2;
      g.M = std::max(need, std::min(512, (L - g.size + 1) / 4 * 4));
   }
   return g;
}

double Choose(int a, int b)
{
   if (b < 0 || b > a)
      return 0.0;
   double r = 1.0;
   for (int i = 0; i < b; ++i)
      r = r * (a - i) / (i + 1);
   return r;
}

// sum_k (-1)^k C(n-k, k) C(n-2k, (n-m)/2 - k) rho^(n-2k): the unnormalized radial term (ZernikePsf.cpp:58-67).
double Radial(int n, int m, double rho)
{
   double r = 0.0;
   for (int k = 0; 2 * k <= n - m; ++k)
      r += (k & 1 ? -1.0 : 1.0) * Choose(n - k, k) * Choose(n - 2 * k, (n - m) / 2 - k) *
           std::pow(rho, static_cast<double>(n - 2 * k));
   return r;
}

// Double-helix phase: arg of sum_p u^l e^{-u^2} L_p^l(2u^2) e^{i l phi}, l = 2p + 1 (ZernikePsf.cpp:80-110).
double HelixPhase(int modes, double waist, double rhoNorm, double phi)
{
   const int np = std::max(2, modes);
   const double u = std::max(0.0, std::min(1.0, rhoNorm)) / std::max(0.2, waist);
   double re = 0.0, im = 0.0;
   for (int p = 0; p < np; ++p)
   {
      const int l = 2 * p + 1;
      double lPrev = 0.0, lCur = 1.0;
      const double x = 2.0 * (u * u);
      for (int k = 0; k < p; ++k)
      {
         const double nxt = ((2 * k + 1 + l - x) * lCur - (k + l) * lPrev) / (k + 1);
         lPrev = lCur;
         lCur = nxt;
      }
      const double amp = std::pow(u, static_cast<double>(l)) * std::exp(-(u * u)) * lCur;
      re += amp * std::cos(l * phi);
      im += amp * std::sin(l * phi);
   }
   return (re == 0.0 && im == 0.0) ? 0.0 : std::atan2(im, re);
}

} // namespace

extern "C" {

// ------------------------------------------------------------------------------------------ RNG
void or_pcg4d(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t* out)
{
   uint32_t v[4] = {a, b, c, d};
   Pcg(v);
   std::memcpy(out, v, sizeof(v));
}

// isc::HashUnit (core/src/rng.h:37-41): the first word of pcg4d(seed, cx, cy, k) as a uniform.
double or_hash_unit(uint32_t seed, int32_t cx, int32_t cy, uint32_t k)
{
   uint32_t v[4] = {seed, static_cast<uint32_t>(cx), static_cast<uint32_t>(cy), k};
   Pcg(v);
   return UnitOf(v[0]);
}

// isc::HashStream (core/src/rng.h:45-52): draw i is HashUnit at counter base*4096 + i (uint32 wrap).
void or_hash_stream(uint32_t seed, int32_t cx, int32_t cy, uint32_t base, uint32_t n, double* out)
{
   for (uint32_t i = 0; i < n; ++i)
      out[i] = or_hash_unit(seed, cx, cy, base * 4096u + i);
}

void or_counter_uniforms(uint32_t seed, uint32_t frame, uint32_t pixel0, uint32_t npix, uint32_t per, double* out)
{
   for (uint32_t i = 0; i < npix; ++i)
   {
      Stream s(seed, frame, pixel0 + i);
      for (uint32_t j = 0; j < per; ++j)
         out[static_cast<size_t>(i) * per + j] = s.Next();
   }
}

// ------------------------------------------------------------------------------------------ camera
// Static maps from one mt19937_64: offset, then gain (floored at 4 % of nominal), then read noise (>= 0); a window
// keeps rows [keepY0, keepY0 + keepRows) but every pixel's two draws are taken (SMLMNoise.cpp:66-140).
void or_camera_maps(uint32_t w, uint32_t h, uint64_t seed, double offMean, double offStd, double gainNom,
                    double gainFrac, double rnNom, double rnFrac, uint32_t keepY0, uint32_t keepRows, float* off,
                    float* gain, float* rn)
{
   std::mt19937_64 g(seed);
   const size_t total = static_cast<size_t>(w) * h;
   size_t lo = 0, hi = total;
   if (keepRows)
   {
      const uint32_t rows = std::min(keepRows, h - std::min(h, keepY0));
      lo = static_cast<size_t>(keepY0) * w;
      hi = lo + static_cast<size_t>(rows) * w;
   }
   for (int map = 0; map < 3; ++map)
      for (size_t i = 0; i < total; ++i)
      {
         const double z = MapNormal(g);
         if (i < lo || i >= hi)
            continue;
         if (map == 0)
            off[i - lo] = static_cast<float>(offMean + offStd * z);
         else if (map == 1)
         {
            const double v = gainNom * (1.0 + gainFrac * z), floorGain = 0.04 * gainNom;
            gain[i - lo] = static_cast<float>(v < floorGain ? floorGain : v);
         }
         else
         {
            const double v = rnNom * (1.0 + rnFrac * z);
            rn[i - lo] = static_cast<float>(v < 0.0 ? 0.0 : v);
         }
      }
}

// The per-pixel noise chain of one frame (SMLMNoise.cpp:142-216): sCMOS Poisson + Gaussian read noise, or EMCCD
// Poisson -> Gamma register -> read noise / EM gain; / gain + offset, rounded and clipped.
void or_noise_chain(const float* photons, uint32_t w, uint32_t h, const iscu_camera* cam, const float* off,
                    const float* gain, const float* rn, uint32_t seed, uint32_t frame, uint32_t pixelBase,
                    uint16_t* out)
{
   const size_t n = static_cast<size_t>(w) * h;
   const double emGain = std::max(1.0, cam->em_gain);
   const int bits = std::min(16, std::max(1, static_cast<int>(cam->bit_depth)));
   const double maxAdu = static_cast<double>((1u << bits) - 1u);
   for (size_t i = 0; i < n; ++i)
   {
      Stream s(seed, frame, static_cast<uint32_t>(i) + pixelBase);
      const double ph = std::max(0.0, static_cast<double>(photons[i]));
      const double g = gain ? static_cast<double>(gain[i]) : cam->gain;
      const double o = off ? static_cast<double>(off[i]) : 0.0;
      const double r = rn ? static_cast<double>(rn[i]) : cam->read_noise_e;
      double adu;
      if (cam->emccd)
      {
         const double ne = Poisson(ph * cam->quantum_efficiency + cam->dark_electrons + cam->cic_electrons, s);
         const double amplified = ne > 0.0 ? GammaDraw(ne, s) : 0.0;
         const double z = Normal(s);
         adu = std::floor(o + (amplified + (r / emGain) * z) / g + 0.5);
         adu = std::min(std::max(adu, 0.0), maxAdu);
      }
      else
      {
         const double ne = Poisson(ph * cam->quantum_efficiency + cam->dark_electrons, s);
         const double z = Normal(s);
         adu = o + (ne + r * z) / g;
         adu = std::floor(std::min(std::max(adu, 0.0), 65535.0) + 0.5);
      }
      out[i] = static_cast<uint16_t>(adu);
   }
}

// ------------------------------------------------------------------------------------------ PSF
int or_psf_geometry(const iscu_psf_request* r, int* size, int* nz, int* M)
{
   const Geometry g = Geo(*r);
   *size = g.size;
   *nz = g.nz;
   *M = g.M;
   return 0;
}

// |E|^2 planes in float64 for the given defocus values (metres; the reference's plane z sits at
// zStep * 1e-9 * (z - (nz-1)/2)). E = A U A^T, A[p][m] = exp(i (kMin + m dk)(x0 + p dx)), the pupil
// U = exp(i (k0 (opd1 + ni (ti - ti0) opd3) + zernike + mask)) inside the aperture (ZernikePsf.cpp:160-337, ChirpZ.h
// :28-142). size <= 0: the request's 2 half os + 1. normalize: each plane / its sum.
void or_psf_planes(const iscu_psf_request* req, int size, const double* defocusM, int n, int normalize, double* out)
{
   const Geometry g = Geo(*req);
   const int M = g.M, P = size > 0 ? size : g.size, c0 = M / 2;
   const double NA = req->na, ni = req->immersion_index, ns = req->sample_index;
   const double k0 = 2.0 * kPi / (req->wavelength_nm * 1e-9);
   const double bMax = std::min(1.0, ns / NA);
   const double kMax = k0 * NA * bMax;
   const double dk = 2.0 * kMax / (M - 4);
   const double kMin = -std::floor(M / 2.0) * dk;
   const double dx = g.resLatNm * 1e-9;
   const double x0 = -((P - 1) / 2.0) * dx;
   const double depth = req->sample_depth_nm * 1e-9;
   const double ti0 = req->working_distance_um * 1e-6;
   // modes: OSA j -> (n, l); m = |l|
   struct Mode { double c; int n, l; };
   std::vector<Mode> modes;
   for (int j = 0; j < 28; ++j)
      if (req->zernike[j] != 0.0)
      {
         int nn = 0;
         while ((nn + 1) * (nn + 2) / 2 <= j)
            ++nn;
         modes.push_back({req->zernike[j], nn, 2 * (j - nn * (nn + 1) / 2) - nn});
      }
   std::vector<char> in(static_cast<size_t>(M) * M, 0);
   std::vector<double> opd1(in.size()), opd3f(in.size()), extra(in.size());
   for (int iy = 0; iy < M; ++iy)
      for (int ix = 0; ix < M; ++ix)
      {
         const double ky = (iy - c0) * dk, kx = (ix - c0) * dk;
         const double kr2 = kx * kx + ky * ky;
         if (kr2 > kMax * kMax)
            continue;
         const size_t q = static_cast<size_t>(iy) * M + ix;
         in[q] = 1;
         const double rho = std::sqrt(kr2) / (k0 * NA), phi = std::atan2(ky, kx);
         const double s1 = NA * rho / ns, s3 = NA * rho / ni;
         opd1[q] = ns * depth * std::sqrt(std::max(0.0, 1.0 - s1 * s1));
         opd3f[q] = std::sqrt(std::max(0.0, 1.0 - s3 * s3));
         double w = 0.0;
         for (const Mode& md : modes)
         {
            const int m = std::abs(md.l);
            const double rn = rho / bMax;
            const double rad = rn <= 1.0 ? Radial(md.n, m, rn) : 0.0;
            w += md.c * rad * (md.l >= 0 ? std::cos(m * phi) : std::sin(m * phi));
         }
         extra[q] = w * (2.0 * kPi) +
                    (req->mask_double_helix ? HelixPhase(req->mask_modes, req->mask_waist, rho / bMax, phi) : 0.0);
      }
   std::vector<std::complex<double>> A(static_cast<size_t>(P) * M);
   for (int p = 0; p < P; ++p)
      for (int m = 0; m < M; ++m)
         A[static_cast<size_t>(p) * M + m] = std::polar(1.0, (kMin + m * dk) * (x0 + p * dx));
   const double focal = depth * (ni / ns);
   std::vector<std::complex<double>> U(static_cast<size_t>(M) * M), T(static_cast<size_t>(P) * M);
   for (int z = 0; z < n; ++z)
   {
      const double dti = ((ti0 - focal) + defocusM[z]) - ti0;
      for (size_t q = 0; q < U.size(); ++q)
         U[q] = in[q] ? std::polar(1.0, k0 * (opd1[q] + ni * dti * opd3f[q]) + extra[q]) : 0.0;
      // T = A U (the transform over ky of every pupil column), then E = T A^T (over kx).
      for (int p = 0; p < P; ++p)
         for (int m = 0; m < M; ++m)
         {
            std::complex<double> acc = 0.0;
            for (int k = 0; k < M; ++k)
               acc += A[static_cast<size_t>(p) * M + k] * U[static_cast<size_t>(k) * M + m];
            T[static_cast<size_t>(p) * M + m] = acc;
         }
      double* plane = out + static_cast<size_t>(z) * P * P;
      double sum = 0.0;
      for (int y = 0; y < P; ++y)
         for (int x = 0; x < P; ++x)
         {
            std::complex<double> acc = 0.0;
            for (int k = 0; k < M; ++k)
               acc += T[static_cast<size_t>(y) * M + k] * A[static_cast<size_t>(x) * M + k];
            plane[static_cast<size_t>(y) * P + x] = std::norm(acc);
            sum += std::norm(acc);
         }
      if (normalize && sum > 0.0)
         for (int i = 0; i < P * P; ++i)
            plane[i] /= sum;
   }
}

// Block sums of each os x os block of kernel cells, blocks starting at -(os-1) .. n-1 on both axes, float64 in the
// reference's order (row sums, then the column sum of those) -> float (PsfGeneratorBridge.cpp:1021-1047).
void or_block_sums(const float* planes, int n, int os, int nz, float* out)
{
   const int bw = n + os - 1;
   for (int z = 0; z < nz; ++z)
   {
      const float* k = planes + static_cast<size_t>(z) * n * n;
      float* o = out + static_cast<size_t>(z) * bw * bw;
      for (int a = 0; a < bw; ++a)
         for (int b = 0; b < bw; ++b)
         {
            double s = 0.0;
            for (int y = std::max(0, a - os + 1); y <= std::min(n - 1, a); ++y)
            {
               double r = 0.0;
               for (int x = std::max(0, b - os + 1); x <= std::min(n - 1, b); ++x)
                  r += static_cast<double>(k[static_cast<size_t>(y) * n + x]);
               s += r;
            }
            o[static_cast<size_t>(a) * bw + b] = static_cast<float>(s);
         }
   }
}

// ------------------------------------------------------------------------------------------ splat
// One frame: background (flat, or map, times illumination, times bgScale), then each emitter (x, y, photons,
// plane|slot<<16 -- slot ignored, one kernel) added in order: per camera pixel of the (2 camRad + 1)^2 square that is
// on the image (and in the halo cut's columns when spans are given), float(photons * sum_j wy_j sum_i wx_i B) with
// the SplatSetup taps (PsfGeneratorBridge.cpp:1382-1422, SplatKernel.inl:51-171, SMLMSimulation.cpp:103-160).
void or_render_frame(const float* sums, int nz, int bw, int os, int size, int interp, const int16_t* spanLo,
                     const int16_t* spanHi, const iscu_emitter* ems, uint32_t nEm, uint32_t w, uint32_t h,
                     double flatBg, const float* bgMap, const float* illum, double bgScale, float* img)
{
   const size_t npx = static_cast<size_t>(w) * h;
   for (size_t i = 0; i < npx; ++i)
   {
      double b = bgMap ? static_cast<double>(bgMap[i]) : flatBg;
      if (illum)
         b *= static_cast<double>(illum[i]);
      img[i] = static_cast<float>(b * bgScale);
   }
   const int camRad = ((size - 1) / 2) / os, off = os - 1;
   const double kc = (size - 1) / 2.0;
   for (uint32_t e = 0; e < nEm; ++e)
   {
      const iscu_emitter& em = ems[e];
      const int z = em.plane & 0xffff;
      if (!(em.photons > 0.0) || em.plane < 0 || z >= nz)
         continue;
      const int x0 = static_cast<int>(std::floor(em.x_px + 0.5)), y0 = static_cast<int>(std::floor(em.y_px + 0.5));
      const double tx = kc + (x0 - em.x_px - 0.5) * os + 0.5, ty = kc + (y0 - em.y_px - 0.5) * os + 0.5;
      double wx[4] = {1, 0, 0, 0}, wy[4] = {1, 0, 0, 0};
      int bx, by, taps;
      if (interp == ISCU_INTERP_NEAREST)
      {
         bx = static_cast<int>(std::floor(tx + 0.5));
         by = static_cast<int>(std::floor(ty + 0.5));
         taps = 1;
      }
      else
      {
         const int fxI = static_cast<int>(std::floor(tx)), fyI = static_cast<int>(std::floor(ty));
         const double fx = tx - fxI, fy = ty - fyI;
         if (interp == ISCU_INTERP_CUBIC)
         {
            // Catmull-Rom weights of the fraction f: taps at -1, 0, 1, 2.
            auto cr = [](double f, double* c) {
               const double f2 = f * f, f3 = f2 * f;
               c[0] = -0.5 * f3 + f2 - 0.5 * f;
               c[1] = 1.5 * f3 - 2.5 * f2 + 1.0;
               c[2] = -1.5 * f3 + 2.0 * f2 + 0.5 * f;
               c[3] = 0.5 * f3 - 0.5 * f2;
            };
            cr(fx, wx);
            cr(fy, wy);
            bx = fxI - 1;
            by = fyI - 1;
            taps = 4;
         }
         else
         {
            wx[0] = 1.0 - fx;
            wx[1] = fx;
            wy[0] = 1.0 - fy;
            wy[1] = fy;
            bx = fxI;
            by = fyI;
            taps = 2;
         }
      }
      const float* B = sums + static_cast<size_t>(z) * bw * bw;
      for (int dy = -camRad; dy <= camRad; ++dy)
      {
         const int Y = y0 + dy;
         if (Y < 0 || Y >= static_cast<int>(h))
            continue;
         int lo = -camRad, hi = camRad;
         if (spanLo)
         {
            lo = std::max(lo, static_cast<int>(spanLo[z * (2 * camRad + 1) + dy + camRad]));
            hi = std::min(hi, static_cast<int>(spanHi[z * (2 * camRad + 1) + dy + camRad]));
         }
         const int r0 = by + dy * os + off;
         for (int dx = lo; dx <= hi; ++dx)
         {
            const int X = x0 + dx;
            if (X < 0 || X >= static_cast<int>(w))
               continue;
            const int c0 = bx + dx * os + off;
            double sum = 0.0;
            for (int j = 0; j < taps; ++j)
            {
               if (r0 + j < 0 || r0 + j >= bw)
                  continue;
               double row = 0.0;
               for (int i = 0; i < taps; ++i)
               {
                  if (c0 + i < 0 || c0 + i >= bw)
                     continue;
                  row += wx[i] * static_cast<double>(B[static_cast<size_t>(r0 + j) * bw + c0 + i]);
               }
               sum += wy[j] * row;
            }
            img[static_cast<size_t>(Y) * w + X] += static_cast<float>(em.photons * sum);
         }
      }
   }
}

// The frame's emitters from its blink events (CollectFrameEmitters, SMLMSimulation.cpp:55-101, minus the
// illumination): overlap with [frame, frame + 1), photons = perBlink * overlap * brightness * excite, position in
// camera pixels plus drift, nearest z plane by lround (PsfGeneratorBridge.cpp:40-61); min_photons drops dim ones.
uint32_t or_collect_frame_emitters(const iscu_blink_event* ev, uint32_t nEv, int64_t frame, double pixelNm,
                                   double perBlink, double driftX, double driftY, double globalZUm, int nz,
                                   double zStepNm, int slot, double minPhotons, iscu_emitter* out)
{
   uint32_t n = 0;
   for (uint32_t i = 0; i < nEv; ++i)
   {
      const double lo = std::max(static_cast<double>(frame), ev[i].t_start);
      const double hi = std::min(static_cast<double>(frame + 1), ev[i].t_end);
      double ov = hi - lo;
      if (ov <= 0.0)
         continue;
      ov = std::min(ov, 1.0);
      double ph = perBlink * ov;
      if (ev[i].brightness != 1.0)
         ph *= ev[i].brightness;
      if (ev[i].excite != 1.0)
         ph *= ev[i].excite;
      int z = 0;
      if (nz > 1 && zStepNm > 0.0)
      {
         const long r = std::lround((ev[i].z_nm / 1000.0 - globalZUm) * 1000.0 / zStepNm + (nz - 1) / 2.0);
         z = static_cast<int>(std::min<long>(std::max<long>(r, 0), nz - 1));
      }
      if (minPhotons > 0.0 && ph < minPhotons)
         continue;
      out[n].x_px = ev[i].x_um * 1000.0 / pixelNm + driftX;
      out[n].y_px = ev[i].y_um * 1000.0 / pixelNm + driftY;
      out[n].photons = ph;
      out[n].plane = z | (slot << 16);
      out[n].reserved = 0;
      ++n;
   }
   return n;
}

} // extern "C"
