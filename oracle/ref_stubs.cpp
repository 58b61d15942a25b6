// TEST INFRASTRUCTURE: WidefieldRender.cpp names three members of sim::SampleSource that live in SampleSource.cpp,
// which needs the world core (not compiled for the checks). The checks build their widefield scenes from dye grids
// (WidefieldScene::UpdateFromGrid) and never reach a sample source; reaching one aborts.
#include "SampleSource.h"

#include <cstdio>
#include <cstdlib>

namespace sim {

namespace {
[[noreturn]] void NoSampleSource()
{
   std::fprintf(stderr, "a sample source is not part of the checks\n");
   std::abort();
}
} // namespace

int SampleSource::AllStructures() { NoSampleSource(); }
int SampleSource::PersistentMask() const { NoSampleSource(); }
long SampleSource::Density3d(double, double, double, double, double, double, int, int, int, int, float*)
{
   NoSampleSource();
}

} // namespace sim
