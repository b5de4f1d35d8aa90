// sph_render.cu -- the reference's ray tracer (src/raytracer.cuh), headless:
// perspective rays from the camera the reference's render() sets up, the
// closest sphere along each ray, Lambertian shading with a uniform colour
// or a colour map, into an RGB image in device memory.
//
// The reference tests every sphere for every pixel.  Here the spheres are
// first binned into 16 x 16-pixel tiles by the projection of a bounding
// cube (the sphere widened by a margin that covers the rounding of the
// intersection test, plus two pixels), and each pixel tests only its tile's
// spheres.  The reference keeps the hit with the smallest |t| met first in
// index order, i.e. the lexicographic minimum of (|t|, index), which does
// not depend on the order the candidates are visited in; the intersection
// and shading arithmetic is the reference's, in FP32 with IEEE division and
// square root and without FMA contraction (this file is compiled with
// -fmad=false), so the image is the reference's arithmetic pixel for pixel.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "sph_internal.h"
#include "sphere_b200.h"

namespace sph {

namespace {

constexpr int TILE = 16;

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float3 divf(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3 neg(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dotf(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 crossf(float3 a, float3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float lengthf(float3 a) { return sqrtf(dotf(a, a)); }
// unit vector: the vector times 1 / sqrt(|v|^2)
__device__ __forceinline__ float3 normalizef(float3 v) { return mul(1.0f / sqrtf(dotf(v, v)), v); }

// blue - white - red colour map of src/colorbar.h:7-20
__device__ __forceinline__ float cm_red(float r)
{
    return fminf(1.0f, 0.209f * r * r * r - 2.49f * r * r + 3.0f * r + 0.0109f);
}
__device__ __forceinline__ float cm_green(float r) { return fminf(1.0f, -2.44f * r * r + 2.15f * r + 0.369f); }
__device__ __forceinline__ float cm_blue(float r) { return fminf(1.0f, -2.21f * r * r + 1.61f * r + 0.573f); }

struct Camera {
    float3 u, v, w, eye, light;
    float4 imgplane;   // l, r, b, t
    float d;
};

struct RtArgs {
    const double4 *x, *vel, *angvel, *angpos, *xyzsum;
    const double *p;
    const double *L;                     // the box's grid.L
    uint32_t p0, np;
    uint32_t width, height;
    uint32_t tx, ty;                     // tiles across and down, in (i, j)
    int method;
    float maxval, lower_cutoff;
    unsigned long long *maxbits;         // maxPos(), as bits of non-negative doubles
    Camera *cam;
    float4 *xf;                          // (float) centre and radius
    uint32_t *tcount, *toff, *tfill, *tlist;
    uint8_t *img;
};

// src/sphere.cpp:641-670 (maxPos): the componentwise maximum of the
// positions and zero.  Only positive values can raise it, and for those the
// order of the bit patterns is the order of the values.
__global__ void k_rt_maxpos(RtArgs R)
{
    unsigned long long m[3] = {0ull, 0ull, 0ull};
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < R.np; k += gridDim.x * blockDim.x) {
        const double4 x = R.x[R.p0 + k];
        const double c[3] = {x.x, x.y, x.z};
        for (int a = 0; a < 3; ++a)
            if (c[a] > 0.0) m[a] = max(m[a], (unsigned long long)__double_as_longlong(c[a]));
    }
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) m[a] = max(m[a], __shfl_xor_sync(0xffffffffu, m[a], o));
        if ((threadIdx.x & 31) == 0 && m[a]) atomicMax(R.maxbits + a, m[a]);
    }
}

// src/raytracer.cuh:379-400 (render) and :291-333 (cameraInit); one thread
__global__ void k_rt_camera(RtArgs R)
{
    const double *L = R.L;
    const float3 maxpos = f3((float)__longlong_as_double((long long)R.maxbits[0]),
                             (float)__longlong_as_double((long long)R.maxbits[1]),
                             (float)__longlong_as_double((long long)R.maxbits[2]));
    const float imgw = (float)(L[0] * 1.35f);
    const float3 lookat = divf(maxpos, 2.0f);
    const float3 eye = f3((float)(L[0] * 2.3f), (float)(L[1] * -5.0f), (float)(L[2] * 1.3f));
    const float hw_ratio = (float)(R.height / R.width);   // integer division, as there
    Camera c;
    c.imgplane = make_float4(-0.5f * imgw, 0.5f * imgw, -0.5f * imgw * hw_ratio, 0.5f * imgw * hw_ratio);
    const float3 view = sub(eye, lookat);
    const float3 up = f3(0.0f, 0.0f, 1.0f);
    c.w = divf(neg(view), lengthf(view));
    c.u = divf(crossf(up, c.w), lengthf(crossf(up, c.w)));
    c.v = crossf(c.w, c.u);
    c.d = lengthf(view) * 0.8f;
    const float3 le = mul(-1.0f, eye);
    c.light = normalizef(f3(le.x * 1.0f, le.y * 0.2f, le.z * 0.6f));
    c.eye = eye;
    *R.cam = c;
}

// value coloured by the colour-map methods (src/raytracer.cuh:452-499)
__device__ __forceinline__ double colour_value(const RtArgs &R, uint32_t g)
{
    switch (R.method) {
    case 1: return R.p[g];
    case 2: { const double4 v = R.vel[g]; return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
    case 3: { const double4 v = R.angvel[g]; return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
    case 4: return R.xyzsum[g].x;
    default: { const double4 v = R.angpos[g]; return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
    }
}

// Tile rectangle holding the central projection (through the eye, of the
// whole line: the reference takes |t|) of the cube of half-size rho around
// a sphere; false when the cube reaches the plane through the eye normal to
// the view (then: every tile).  rho = r + 2e-3 |c - eye| covers the rays
// that the FP32 discriminant counts as hits although they pass outside the
// sphere: its rounding error is below 16 eps |d|^2 |e - c|^2, so such rays
// pass within r + 1e-3 |e - c| of the centre.  Two more pixels cover the
// rounding of the ray directions.  (With the grid origin at or above zero,
// which the reference requires, the eye at (2.3 L0, -5 L1, 1.3 L2) sees
// every sphere on one side of that plane; the every-tile answer is the safe
// one for anything else.)
__device__ bool sphere_tiles(const RtArgs &R, const Camera &c, const double4 x, int &t0x, int &t1x,
                             int &t0y, int &t1y)
{
    const float3 cc = f3((float)x.x, (float)x.y, (float)x.z);
    const float rho = (float)x.w + 2e-3f * lengthf(sub(cc, c.eye));
    float imin = 1e30f, imax = -1e30f, jmin = 1e30f, jmax = -1e30f;
    int side = 0;
    const bool flat = !(c.imgplane.w - c.imgplane.z > 0.0f);   // hw_ratio = 0: all rows alike
    for (int q = 0; q < 8; ++q) {
        const float3 P = add(cc, f3((q & 1) ? rho : -rho, (q & 2) ? rho : -rho, (q & 4) ? rho : -rho));
        const float3 D = sub(P, c.eye);
        const float dw = -dotf(D, c.w);
        const float lim = 1e-4f * lengthf(D);
        const int s = dw > lim ? 1 : (dw < -lim ? -1 : 0);
        if (s == 0 || (side != 0 && s != side)) return false;
        side = s;
        const float pu = c.d * dotf(D, c.u) / dw, pv = c.d * dotf(D, c.v) / dw;
        const float fi = (pu - c.imgplane.x) / (c.imgplane.y - c.imgplane.x) * (float)R.width - 0.5f;
        imin = fminf(imin, fi);
        imax = fmaxf(imax, fi);
        if (!flat) {
            const float fj = (pv - c.imgplane.z) / (c.imgplane.w - c.imgplane.z) * (float)R.height - 0.5f;
            jmin = fminf(jmin, fj);
            jmax = fmaxf(jmax, fj);
        }
    }
    if (!(imin == imin && imax == imax && jmin == jmin && jmax == jmax)) return false;
    const float wlast = (float)R.width - 1.0f;   // j = row % width < width, like i
    if (imax < -3.0f || imin > wlast + 3.0f || (!flat && (jmax < -3.0f || jmin > wlast + 3.0f))) {
        t0x = 1;   // off the image
        t1x = 0;
        return true;
    }
    t0x = (int)fmaxf(floorf(imin) - 2.0f, 0.0f) / TILE;
    t1x = (int)fminf(ceilf(imax) + 2.0f, wlast) / TILE;
    if (flat) {
        t0y = 0;
        t1y = (int)R.ty - 1;
    } else {
        t0y = (int)fmaxf(floorf(jmin) - 2.0f, 0.0f) / TILE;
        t1y = (int)fminf(ceilf(jmax) + 2.0f, wlast) / TILE;
    }
    return true;
}

// Count (FILL = false) or list (FILL = true) each sphere in the tiles its
// bounding cube projects onto.  Spheres the cutoff excludes are left out,
// as the reference never takes them (src/raytracer.cuh:190-214).
template <bool FILL>
__global__ void __launch_bounds__(256) k_rt_bin(RtArgs R)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R.np) return;
    const uint32_t g = R.p0 + k;
    const double4 x = R.x[g];
    if (FILL) R.xf[k] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    if (R.method != 0 && R.lower_cutoff > 0.0f) {
        const float val = (float)colour_value(R, g);
        const float fixvel = (float)R.vel[g].w;
        if (!(val > R.lower_cutoff && fixvel == 0.f)) return;
    }
    const Camera c = *R.cam;
    int t0x, t1x, t0y, t1y;
    if (!sphere_tiles(R, c, x, t0x, t1x, t0y, t1y)) {
        t0x = 0;
        t1x = (int)R.tx - 1;
        t0y = 0;
        t1y = (int)R.ty - 1;
    }
    for (int ty = t0y; ty <= t1y; ++ty)
        for (int tx = t0x; tx <= t1x; ++tx) {
            const uint32_t t = (uint32_t)ty * R.tx + (uint32_t)tx;
            if (FILL) R.tlist[R.toff[t] + atomicAdd(&R.tfill[t], 1u)] = k;
            else atomicAdd(&R.tcount[t], 1u);
        }
}

// exclusive scan of the tile counts in one block; off[n] = total
__global__ void k_rt_scan(const uint32_t *count, uint32_t n, uint32_t *off)
{
    __shared__ uint32_t part[1024];
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = min(n, threadIdx.x * per), e = min(n, b + per);
    uint32_t s = 0;
    for (uint32_t q = b; q < e; ++q) s += count[q];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t q = 0; q < blockDim.x; ++q) {
            const uint32_t v = part[q];
            part[q] = run;
            run += v;
        }
        off[n] = run;
    }
    __syncthreads();
    uint32_t run = part[threadIdx.x];
    for (uint32_t q = b; q < e; ++q) {
        off[q] = run;
        run += count[q];
    }
}

// the nearer root of the ray-sphere quadratic (src/raytracer.cuh:104-107)
__device__ __forceinline__ float t_minus_of(float3 d, float3 ec, float r)
{
    return (dotf(neg(d), ec) - sqrtf(dotf(d, ec) * dotf(d, ec) - dotf(d, d) * (dotf(ec, ec) - r * r))) /
           dotf(d, d);
}

// One 16 x 16 block of pixels per thread block: src/raytracer.cuh:29-56
// (rayInitPerspective), :14-27 (imageInit), :59-144 (rayIntersectSpheres)
// and :146-288 (rayIntersectSpheresColormap).
__global__ void __launch_bounds__(TILE * TILE) k_rt_trace(RtArgs R)
{
    const uint32_t i = blockIdx.x * TILE + threadIdx.x;
    const uint32_t row = blockIdx.y * TILE + threadIdx.y;
    if (i >= R.width || row >= R.height) return;
    const uint32_t mempos = row * R.width + i;
    const Camera c = *R.cam;
    const uint32_t j = (uint32_t)((int)floorf((float)mempos / R.width)) % R.width;
    const float p_u = c.imgplane.x + (c.imgplane.y - c.imgplane.x) * (i + 0.5f) / R.width;
    const float p_v = c.imgplane.z + (c.imgplane.w - c.imgplane.z) * (j + 0.5f) / R.height;
    const float3 e = c.eye;
    const float3 d = add(add(mul(-c.d, c.w), mul(p_u, c.u)), mul(p_v, c.v));
    float tdist = 1e10f;
    uint32_t hit = 0xffffffffu;
    const uint32_t t = (j / TILE) * R.tx + i / TILE;
    const uint32_t q1 = R.toff[t + 1];
    for (uint32_t q = R.toff[t]; q < q1; ++q) {
        const uint32_t k = R.tlist[q];
        const float4 s = R.xf[k];
        const float3 ec = sub(e, f3(s.x, s.y, s.z));
        const float Delta =
            (2.0f * dotf(d, ec)) * (2.0f * dotf(d, ec)) - 4.0f * dotf(d, d) * (dotf(ec, ec) - s.w * s.w);
        if (!(Delta > 0.0f)) continue;
        const float at = fabsf(t_minus_of(d, ec, s.w));
        if (at < tdist || (at == tdist && k < hit)) {
            tdist = at;
            hit = k;
        }
    }
    uint8_t *px = R.img + 3 * (size_t)mempos;
    if (!(tdist < 1e10f)) {
        px[0] = px[1] = px[2] = 255;   // background
        return;
    }
    const float4 s = R.xf[hit];
    const float3 cc = f3(s.x, s.y, s.z);
    const float3 ec = sub(e, cc);
    const float3 p = add(e, mul(t_minus_of(d, ec, s.w), d));
    const float3 n = normalizef(mul(2.0f, sub(p, cc)));
    const float dotprod = fmaxf(0.0f, dotf(n, c.light));
    const float I_d = 40.0f, k_d = 5.0f, k_a = 10.0f, I_a = 5.0f;
    const float shade = k_d * I_d * dotprod + k_a * I_a;
    if (R.method == 0) {
        px[0] = (uint8_t)(shade * 0.48f);
        px[1] = (uint8_t)(shade * 0.41f);
        px[2] = (uint8_t)(shade * 0.27f);
        return;
    }
    const uint32_t g = R.p0 + hit;
    const float fixvel = (float)R.vel[g].w;
    float ratio = (float)(colour_value(R, g) / (double)R.maxval);
    if (ratio < 0.01f) ratio = 0.01f;
    if (ratio > 0.99f) ratio = 0.99f;
    float redv = cm_red(ratio), greenv = cm_green(ratio), bluev = cm_blue(ratio);
    if (fixvel > 0.f) redv = greenv = bluev = 0.5f;
    px[0] = (uint8_t)(shade * redv);
    px[1] = (uint8_t)(shade * greenv);
    px[2] = (uint8_t)(shade * bluev);
}

}  // namespace

int render_image(const StepArgs &A, uint32_t p0, uint32_t np, const double *d_L, int method,
                 float maxval, float lower_cutoff, uint32_t width, uint32_t height, uint8_t *d_img,
                 cudaStream_t st, RenderStats *stats)
{
    RtArgs R{};
    R.x = A.x;
    R.vel = A.vel;
    R.angvel = A.angvel;
    R.angpos = A.angpos;
    R.xyzsum = A.xyzsum;
    R.p = A.p;
    R.L = d_L;
    R.p0 = p0;
    R.np = np;
    R.width = width;
    R.height = height;
    R.tx = (width + TILE - 1) / TILE;
    R.ty = R.tx;   // j = row % width < width
    R.method = method;
    R.maxval = maxval;
    R.lower_cutoff = lower_cutoff;
    R.img = d_img;
    const uint32_t ntiles = R.tx * R.ty;
    // scratch: maxbits[3] | camera | xf[np] | tcount, tfill, toff[ntiles + 1]
    static_assert(sizeof(Camera) <= 224, "camera slot");
    const size_t off_cam = 32, off_xf = 256;
    const size_t off_t = off_xf + sizeof(float4) * (size_t)np;
    const size_t bytes = off_t + sizeof(uint32_t) * (3 * (size_t)ntiles + 1);
    char *buf = nullptr;
    if (cudaMalloc((void **)&buf, bytes) != cudaSuccess) return SPH_ERR_NOMEM;
    R.maxbits = (unsigned long long *)buf;
    R.cam = (Camera *)(buf + off_cam);
    R.xf = (float4 *)(buf + off_xf);
    R.tcount = (uint32_t *)(buf + off_t);
    R.tfill = R.tcount + ntiles;
    R.toff = R.tfill + ntiles;
    cudaMemsetAsync(buf, 0, 32, st);
    cudaMemsetAsync(R.tcount, 0, sizeof(uint32_t) * 2 * (size_t)ntiles, st);
    const unsigned gb = (np + 255) / 256;
    const unsigned gm = gb == 0 ? 1u : (gb < 1184u ? gb : 1184u);
    int launches = 0;
    k_rt_maxpos<<<gm, 256, 0, st>>>(R);
    k_rt_camera<<<1, 1, 0, st>>>(R);
    launches += 2;
    if (np) {
        k_rt_bin<false><<<gb, 256, 0, st>>>(R);
        ++launches;
    }
    k_rt_scan<<<1, 1024, 0, st>>>(R.tcount, ntiles, R.toff);
    ++launches;
    uint32_t total = 0;
    cudaMemcpyAsync(&total, R.toff + ntiles, sizeof total, cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(buf);
        return SPH_ERR_CUDA;
    }
    uint32_t *list = nullptr;
    if (cudaMalloc((void **)&list, sizeof(uint32_t) * (total ? total : 1)) != cudaSuccess) {
        cudaFree(buf);
        return SPH_ERR_NOMEM;
    }
    R.tlist = list;
    if (np) {
        k_rt_bin<true><<<gb, 256, 0, st>>>(R);
        ++launches;
    }
    const dim3 grid(R.tx, (height + TILE - 1) / TILE);
    k_rt_trace<<<grid, dim3(TILE, TILE), 0, st>>>(R);
    ++launches;
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFree(list);
    cudaFree(buf);
    if (stats) {
        stats->tiles = ntiles;
        stats->entries = total;
        stats->launches = launches;
    }
    return e == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

}  // namespace sph
