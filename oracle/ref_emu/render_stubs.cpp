// render_stubs.cpp -- TEST INFRASTRUCTURE ONLY.
//
// DEM::checkForCudaErrors lives in the reference's src/device.cu, which the
// ray-tracer harness does not build; DEM::cameraInit calls it after its
// (here host) copies, where there is no CUDA error to check.
#include "sphere.h"

void DEM::checkForCudaErrors(const char *, const int) {}
