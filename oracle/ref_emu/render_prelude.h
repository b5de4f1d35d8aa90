/*
 * render_prelude.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Force-included ahead of the reference's ray-tracer kernels and
 * DEM::cameraInit (src/raytracer.cuh up to DEM::rt_allocateGlobalDeviceMemory,
 * streamed from the reference sources by oracle/Makefile) so that they
 * compile as host C++ for sphere_render_ref.  It supplies:
 *  - the execution-space shim (cuda_host_shim.h) and the reference's
 *    constant-memory symbols (src/constants.cuh) as plain globals;
 *  - the DEM class (src/sphere.h), of which cameraInit is a member;
 *  - cudaMemcpyToSymbol as a host copy into those globals;
 *  - the float3 operations the ray tracer takes from the CUDA samples'
 *    helper_math.h (not part of the reference sources), written here from
 *    their definitions: componentwise + - * /, scaling by a float, dot,
 *    cross, length = sqrtf(dot(v, v)), normalize = v * (1 / sqrtf(dot(v, v))),
 *    make_float4(float3, float).
 */
#ifndef SPHERE_REF_RENDER_PRELUDE_H_
#define SPHERE_REF_RENDER_PRELUDE_H_

#include "cuda_host_shim.h"

#include <iostream>

#include "constants.cuh"
#include "sphere.h"

#define cudaMemcpyToSymbol(sym, src, n) std::memcpy(&(sym), (src), (n))

inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(float3 v) { return sqrtf(dot(v, v)); }
inline float3 normalize(float3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

#endif
