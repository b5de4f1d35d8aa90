// render_main.cpp -- TEST INFRASTRUCTURE ONLY.
//
// `sphere --render` on the CPU: the reference's own ray-tracer kernels
// (src/raytracer.cuh:14-288: imageInit, rayInitPerspective,
// rayIntersectSpheres, rayIntersectSpheresColormap) and its camera set-up
// (DEM::cameraInit, :291-338), compiled for the host by oracle/Makefile,
// driven in the order of DEM::render (:379-560) on a DEM object read from a
// .bin file as src/porosity.cpp:72 constructs it.  Each launch runs its
// threads one after the other (the kernels share nothing between threads;
// their barriers are no-ops here).  The host part of DEM::render (image and
// ray buffers, the linear array of the colour methods) is restated below.
// Writes width * height * 3 bytes (the PPM body, src/file_io.cpp:751-752).
//   sphere_render_ref <file.bin> <method> <maxval> <lower_cutoff> <width> <height> <out.rgb>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <string>
#include <vector>

#include "cuda_host_shim.h"
#define private public
#include "sphere.h"
#undef private

// the reference's kernels and constant symbols (src/raytracer.cuh,
// src/constants.cuh), compiled from the reference sources
void imageInit(unsigned char *dev_img, const unsigned int pixels);
void rayInitPerspective(float4 *dev_ray_origo, float4 *dev_ray_direction, const float4 eye,
                        const unsigned int width, const unsigned int height);
void rayIntersectSpheres(const float4 *dev_ray_origo, const float4 *dev_ray_direction,
                         const Float4 *dev_x, unsigned char *dev_img);
void rayIntersectSpheresColormap(const float4 *dev_ray_origo, const float4 *dev_ray_direction,
                                 const Float4 *dev_x, const Float4 *dev_vel,
                                 const Float *dev_linarr, const float max_val,
                                 const float lower_cutoff, unsigned char *dev_img);
extern unsigned int devC_np;

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
void __syncthreads(void) {}

static void launch(unsigned int blocks, unsigned int threads, const std::function<void()> &body)
{
    gridDim = dim3(blocks);
    blockDim = dim3(threads);
    for (unsigned int b = 0; b < blocks; ++b)
        for (unsigned int t = 0; t < threads; ++t) {
            blockIdx = make_uint3(b, 0, 0);
            threadIdx = make_uint3(t, 0, 0);
            body();
        }
}

int main(int argc, char **argv)
{
    if (argc < 8) {
        std::cerr << "usage: " << argv[0]
                  << " <file.bin> <method> <maxval> <lower_cutoff> <width> <height> <out.rgb>\n";
        return 2;
    }
    DEM dem(argv[1], 0, 0, 0, 0, 0);
    const int method = std::atoi(argv[2]);
    const float maxval = (float)std::atof(argv[3]);
    const float lower_cutoff = (float)std::atof(argv[4]);
    dem.width = (unsigned int)std::atoi(argv[5]);
    dem.height = (unsigned int)std::atoi(argv[6]);
    if (method < 0 || method > 5 || dem.width == 0 || dem.height == 0) return 2;
    const unsigned int np = dem.np;
    const unsigned int pixels = dem.width * dem.height;
    const unsigned int threadsPerBlock = 256;
    const unsigned int blocksPerGrid = (pixels + threadsPerBlock - 1) / threadsPerBlock;
    // the kernels' guards (`mempos > pixels`) let thread `pixels` through:
    // one more element than the image in every buffer
    std::vector<unsigned char> img(4 * ((size_t)pixels + 1), 0);
    std::vector<float4> origo((size_t)pixels + 1), direction((size_t)pixels + 1);
    launch(blocksPerGrid, threadsPerBlock, [&] { imageInit(img.data(), pixels); });

    const float imgw = dem.grid.L[0] * 1.35f;
    const Float3 maxpos = dem.maxPos();
    const float3 lookat = make_float3((float)maxpos.x / 2.0f, (float)maxpos.y / 2.0f,
                                      (float)maxpos.z / 2.0f);
    const float3 eye = make_float3(dem.grid.L[0] * 2.3f, dem.grid.L[1] * -5.0f,
                                   dem.grid.L[2] * 1.3f);
    dem.cameraInit(eye, lookat, imgw, 1.0f);
    devC_np = np;
    launch(blocksPerGrid, threadsPerBlock, [&] {
        rayInitPerspective(origo.data(), direction.data(), make_float4(eye.x, eye.y, eye.z, 0.0f),
                           dem.width, dem.height);
    });
    if (method == 0) {
        launch(blocksPerGrid, threadsPerBlock, [&] {
            rayIntersectSpheres(origo.data(), direction.data(), dem.k.x, img.data());
        });
    } else {
        std::vector<Float> linarr(np ? np : 1);
        for (unsigned int i = 0; i < np; ++i) {
            const Float4 *v = nullptr;
            switch (method) {
            case 1: linarr[i] = dem.e.p[i]; continue;
            case 2: v = dem.k.vel + i; break;
            case 3: v = dem.k.angvel + i; break;
            case 4: linarr[i] = dem.k.xyzsum[i].x; continue;
            default: v = dem.k.angpos + i; break;
            }
            linarr[i] = sqrt(v->x * v->x + v->y * v->y + v->z * v->z);
        }
        launch(blocksPerGrid, threadsPerBlock, [&] {
            rayIntersectSpheresColormap(origo.data(), direction.data(), dem.k.x, dem.k.vel,
                                        linarr.data(), maxval, lower_cutoff, img.data());
        });
    }
    FILE *f = std::fopen(argv[7], "wb");
    if (!f) return 1;
    for (unsigned int i = 0; i < pixels; ++i) std::fwrite(&img[4 * (size_t)i], 1, 3, f);
    std::fclose(f);
    return 0;
}
