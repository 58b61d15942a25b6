// Drives iscu_sim::GpuSimulator (include/iscu_gpusim.hpp) the way the engine drives sim::GpuSimulator: one kernel,
// the static maps, one frame of 64-byte records. Inputs are raw files in argv[1] (written by
// tests/test_gpu_cpp_host.py); the frame goes to argv[1]/adu.u16. Exit 0 on success.
#include "iscu_gpusim.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

template <class T>
static std::vector<T> Read(const std::string& path)
{
   std::ifstream f(path, std::ios::binary);
   std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
   std::vector<T> v(b.size() / sizeof(T));
   if (!v.empty())
      std::copy(b.begin(), b.begin() + v.size() * sizeof(T), reinterpret_cast<char*>(v.data()));
   return v;
}

int main(int argc, char** argv)
{
   if (argc != 20)
   {
      std::fprintf(stderr, "usage: gpusim_main dir size nz os interp zStepNm w h flatBg seed frame bgScale emccd qe "
                           "dark gain readNoise emGain cic\n");
      return 1;
   }
   const std::string dir = argv[1];
   iscu_sim::KernelPlanes k;
   k.planes = Read<float>(dir + "/planes.f32");
   k.size = std::atoi(argv[2]);
   k.nz = std::atoi(argv[3]);
   k.oversampling = std::atoi(argv[4]);
   k.interp = std::atoi(argv[5]);
   k.zStepNm = std::atof(argv[6]);
   const unsigned w = static_cast<unsigned>(std::atoi(argv[7])), h = static_cast<unsigned>(std::atoi(argv[8]));
   const double flatBg = std::atof(argv[9]);
   const uint32_t seed = static_cast<uint32_t>(std::strtoul(argv[10], nullptr, 10));
   const uint32_t frame = static_cast<uint32_t>(std::strtoul(argv[11], nullptr, 10));
   const double bgScale = std::atof(argv[12]);
   iscu_sim::CameraNoiseParams cam;
   cam.emccd = std::atoi(argv[13]) != 0;
   cam.quantumEfficiency = std::atof(argv[14]);
   cam.darkCurrentElectrons = std::atof(argv[15]);
   cam.gainPhotonsPerAdu = std::atof(argv[16]);
   cam.readNoiseElectrons = std::atof(argv[17]);
   cam.emGain = std::atof(argv[18]);
   cam.cicElectrons = std::atof(argv[19]);

   std::string info, err;
   std::unique_ptr<iscu_sim::GpuSimulator> sim = iscu_sim::GpuSimulator::Create(info);
   if (!sim)
   {
      std::fprintf(stderr, "no GPU simulator: %s\n", info.c_str());
      return 2;
   }
   // the error convention: a bad map is refused with a message, nothing thrown
   if (sim->SetStatic(w, h, std::vector<float>(3, 0.f), {}, {}, {}, flatBg, cam, err) || err.empty())
   {
      std::fprintf(stderr, "a wrong-size map was accepted\n");
      return 3;
   }
   err.clear();
   if (!sim->SetKernels({&k}, err))
   {
      std::fprintf(stderr, "SetKernels: %s\n", err.c_str());
      return 4;
   }
   const std::vector<float> offset = Read<float>(dir + "/offset.f32"), gain = Read<float>(dir + "/gain.f32"),
                            rn = Read<float>(dir + "/readnoise.f32");
   if (!sim->SetStatic(w, h, offset, gain, rn, {}, flatBg, cam, err))
   {
      std::fprintf(stderr, "SetStatic: %s\n", err.c_str());
      return 5;
   }
   const std::vector<iscu_sim::GpuSplatEmitter> rec = Read<iscu_sim::GpuSplatEmitter>(dir + "/records.bin");
   std::vector<uint16_t> out;
   if (!sim->RenderFrame(rec, cam, bgScale, seed, frame, out, err))
   {
      std::fprintf(stderr, "RenderFrame: %s\n", err.c_str());
      return 6;
   }
   std::ofstream(dir + "/adu.u16", std::ios::binary)
      .write(reinterpret_cast<const char*>(out.data()), static_cast<std::streamsize>(out.size() * sizeof(uint16_t)));
   std::printf("%s: %zu records, %zu pixels\n", info.c_str(), rec.size(), out.size());
   return 0;
}
