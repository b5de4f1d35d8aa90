/*
 * cuda_host_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets the reference's CUDA kernel headers (src/sorting.cuh,
 * src/contactsearch.cuh, src/contactmodels.cuh, src/cohesion.cuh,
 * src/integration.cuh) compile as host C++ so that ref_harness.cpp can run
 * the reference's own arithmetic on the CPU.  CUDA's vector types and
 * make_* helpers come from the toolkit's host headers; the execution-space
 * qualifiers become no-ops; __shared__ becomes thread_local storage, shared
 * by the emulated threads of one block (which all run on one OS thread);
 * thread and block indexes are thread_local variables set by the launcher.
 */
#ifndef SPHERE_REF_CUDA_HOST_SHIM_H_
#define SPHERE_REF_CUDA_HOST_SHIM_H_

#include <cuda_runtime.h>
#include <vector_functions.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#undef __global__
#undef __device__
#undef __host__
#undef __constant__
#undef __shared__
#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ thread_local

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

/* Block barrier: a no-op in sequential launches, a fiber switch in
 * launches that need barrier semantics (see ref_harness.cpp). */
void __syncthreads(void);

#endif
