// analysis_stubs.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Definitions of the DEM members that live in the reference's CUDA and
// fluid sources (src/device.cu, src/navierstokes.cpp, src/darcy.cpp), so
// that src/sphere.cpp and src/file_io.cpp link into a host program.  The
// analysis harness constructs DEM without CUDA set-up and without fluid, so
// none of these is ever called; each aborts if it were.
#include <cstdio>
#include <cstdlib>

#include "sphere.h"

static void never(const char *what)
{
    std::fprintf(stderr, "analysis harness: %s called\n", what);
    std::abort();
}

void DEM::initializeGPU() { never("initializeGPU"); }
void DEM::allocateGlobalDeviceMemory() { never("allocateGlobalDeviceMemory"); }
void DEM::transferToConstantDeviceMemory() { never("transferToConstantDeviceMemory"); }
void DEM::transferToGlobalDeviceMemory(int) { never("transferToGlobalDeviceMemory"); }
void DEM::initNS() { never("initNS"); }
void DEM::initNSmem() { never("initNSmem"); }
void DEM::initNSmemDev() { never("initNSmemDev"); }
void DEM::initDarcy() { never("initDarcy"); }
void DEM::initDarcyMem() { never("initDarcyMem"); }
void DEM::initDarcyMemDev() { never("initDarcyMemDev"); }
unsigned int DEM::idx(const int, const int, const int) { never("idx"); return 0; }
unsigned int DEM::d_idx(const int, const int, const int) { never("d_idx"); return 0; }
