// sph_darcy.cu -- the Darcy flow coupling of the FP64 step (fluid == 1,
// cfd_solver == 1): src/darcy.cuh and the Darcy part of the step loop,
// src/device.cu:1891-2419.
//
// The fluid grid is the box's cell grid.  Every step with spheres adds the
// fluid's pressure force (the pressure gradient interpolated to the sphere
// times its volume, plus buoyancy) to the sphere forces between interact
// and integrate.  Every ndem steps the fluid is updated: porosities from
// the sorted spheres (a trilinear hat per cell, now and after an Euler step
// of the positions), Kozeny-Carman permeabilities, and the pressure from a
// relaxed Jacobi iteration of the diffusion equation with the porosity
// change as forcing, then the Darcy velocities.
//
// Design for the GPU: the reference runs the Jacobi loop from the host,
// four launches and a device synchronisation per iteration and a copy of
// the whole residual field to the host every tenth; here the whole loop is
// one cooperative launch (k_darcy_jacobi): each iteration is the update,
// a grid barrier, the copy of the new pressure with the flux ghosts and the
// next iteration's ghost layer (each cell writes its value and the ghost
// cells that copy it), and a barrier; every tenth iteration each block
// reduces the largest |residual| of its cells (the bits of a non-negative
// double, which order as the values do) and every block takes the same
// stop decision from all blocks' values.  The barriers are bounded
// (SPH_ERR_TIMEOUT).  A step with its fluid solve is one graph launch with
// no host round trip.  Which steps update the fluid
// (iter % ndem) and the top wall's cell (wall0_iz, from the reference's
// host copy of the wall, refreshed at outputs) are decided on the device,
// which keeps the reference's host file clock, so the results do not
// depend on how the steps are split into calls.  The modulated top
// pressure is computed on the host with the C library's sin, as the
// reference computes it, into a ring read by step index.
//
// Arithmetic: the kernels keep the reference's expressions and operand
// order and the file is compiled without FMA contraction, so the results
// equal the reference's bit for bit.  pow(r, 3) and pow(1 - phi, 2) are the
// correctly rounded cube and square (FMA-exact products), which the C
// library's pow returns.  Two writes of the reference depend on its launch
// grid and are reproduced: setDarcyTopPressure's condition reads
// (x < nx && y < ny && z == nz - 1) || z == wall0_iz, so at z == wall0_iz
// every thread of its 8 x 8 x 8 blocks writes, also those past nx or ny
// (their index lands on other cells of the padded array; writes past the
// array are dropped); and the Dirichlet test of the +y side compares y
// with nx - 1.
#include <cstdint>
#include <cstdio>

#include "sph_device.cuh"
#include "sph_internal.h"
#include "sph_sync.cuh"

namespace sph {

namespace {

constexpr int DARCY_THREADS = 256;
constexpr int JACOBI_THREADS = 512;   // the Jacobi loop: one block per SM
constexpr double DARCY_PI = 3.14159265358979323846;   // M_PI, which src/darcy.cuh uses

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// darcy.cuh:146-157 d_idx
__device__ __forceinline__ uint32_t d_idx(const DarcyArgs &D, int x, int y, int z)
{
    return (uint32_t)(x + 1) + (uint32_t)(D.nx + 2) * (uint32_t)(y + 1) +
           (uint32_t)(D.nx + 2) * (uint32_t)(D.ny + 2) * (uint32_t)(z + 1);
}

// Cell c of the interior (x fastest) as coordinates.
__device__ __forceinline__ bool cell_of(const DarcyArgs &D, uint32_t c, int &x, int &y, int &z)
{
    const uint32_t nxy = (uint32_t)D.nx * (uint32_t)D.ny;
    if (c >= nxy * (uint32_t)D.nz) return false;
    z = (int)(c / nxy);
    const uint32_t r = c - (uint32_t)z * nxy;
    y = (int)(r / (uint32_t)D.nx);
    x = (int)(r - (uint32_t)y * (uint32_t)D.nx);
    return true;
}

// The correctly rounded r^3 and r^2: the rounding error of each product is
// kept exactly by an FMA and added before the last rounding.
__device__ __forceinline__ double cube_rn(double r)
{
    const double p = __dmul_rn(r, r);
    const double e = __fma_rn(r, r, -p);
    const double hi = __dmul_rn(p, r);
    const double lo = __fma_rn(p, r, -hi);
    return __dadd_rn(hi, __fma_rn(e, r, lo));
}

// darcy.cuh:346-349 sphereVolume
__device__ __forceinline__ double sphere_volume(double r)
{
    const double c = 4.0 / 3.0 * DARCY_PI;
    return c * cube_rn(r);
}

// darcy.cuh:356-385 weight / weightDist, of the vector between the points
__device__ __forceinline__ double weight_dist(d3 x, double dx, double dy, double dz)
{
    const d3 dist = mk(fabs(x.x), fabs(x.y), fabs(x.z));
    if (dist.x < dx && dist.y < dy && dist.z < dz)
        return (1.0 - dist.x / dx) * (1.0 - dist.y / dy) * (1.0 - dist.z / dz);
    return 0.0;
}

__device__ __forceinline__ d3 ld3(const double *p) { return mk(p[0], p[1], p[2]); }
__device__ __forceinline__ void st3(double *p, d3 v)
{
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

// darcy.cuh:212-285 setDarcyGhostNodes: which ghost cells copy cell
// (x, y, z), one bit per condition of the reference, six per axis: along an
// axis of n cells with codes lo (at 0) and hi (at n - 1), bit 0: c == 0 and
// lo == 0 (ghost -1), 1: c == 1 and lo == 1 (-1), 2: c == 0 and lo == 2
// (n), 3: c == n - 1 and hi == 0 (n), 4: c == n - 2 and hi == 1 (n), 5:
// c == n - 1 and hi == 2 (-1).  Bits 0-5 are x, 6-11 y, 12-17 z.
__device__ __forceinline__ uint32_t ghost_axis(int c, int n, int lo, int hi)
{
    return (uint32_t)(c == 0 && lo == 0) | (uint32_t)(c == 1 && lo == 1) << 1 |
           (uint32_t)(c == 0 && lo == 2) << 2 | (uint32_t)(c == n - 1 && hi == 0) << 3 |
           (uint32_t)(c == n - 2 && hi == 1) << 4 | (uint32_t)(c == n - 1 && hi == 2) << 5;
}
__device__ __forceinline__ uint32_t ghost_bits(const DarcyArgs &D, int x, int y, int z)
{
    const SphDarcy &P = D.prm;
    return ghost_axis(x, D.nx, P.bc_xn, P.bc_xp) | ghost_axis(y, D.ny, P.bc_yn, P.bc_yp) << 6 |
           ghost_axis(z, D.nz, P.bc_bot, P.bc_top) << 12;
}

// The cell's value (M doubles) into the ghost cells of its bits (every
// ghost gets the same value, so their order does not matter).
template <int M>
__device__ __forceinline__ void put_ghost_bits(const DarcyArgs &D, double *f, int x, int y, int z,
                                               uint32_t bits, const double *val)
{
    while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1u;
        const int axis = b / 6, k = b - 6 * axis;
        const int n = axis == 0 ? D.nx : axis == 1 ? D.ny : D.nz;
        const int t = (k == 2 || k == 3 || k == 4) ? n : -1;
        double *o = f + (size_t)M * d_idx(D, axis == 0 ? t : x, axis == 1 ? t : y, axis == 2 ? t : z);
#pragma unroll
        for (int m = 0; m < M; ++m) o[m] = val[m];
    }
}

template <int M>
__device__ __forceinline__ void put_ghosts(const DarcyArgs &D, double *f, int x, int y, int z,
                                           const double *val)
{
    put_ghost_bits<M>(D, f, x, y, z, ghost_bits(D, x, y, z), val);
}

// Whether this step updates the fluid (set by k_darcy_begin).
__device__ __forceinline__ bool fluid_step(const DarcyArgs &D) { return D.st->active != 0u; }

// ------------------------------------------------------------ every step

// device.cu:1901-1904 (wall0_iz from the host copy of wall 0) and the
// choice of the fluid-update steps (iter % ndem == 0)
__global__ void k_darcy_begin(StepArgs A, DarcyArgs D)
{
    const DevBox &B = A.boxes[0];
    DarcyState *s = D.st;
    if (B.nw > 0 && (B.wmode[0] == 1 || B.wmode[0] == 3))
        s->wall0_iz = (uint32_t)(s->wall_w_host / (B.L[2] / B.num[2]));
    s->active = (B.iter % D.prm.ndem) == 0 ? 1u : 0u;
}

// setDarcyGhostNodes for M-double fields: one thread per interior cell
template <int M>
__global__ void k_darcy_ghost(DarcyArgs D, double *f, int gated)
{
    if (gated && !fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    double val[M];
    const double *src = f + (size_t)M * d_idx(D, x, y, z);
#pragma unroll
    for (int m = 0; m < M; ++m) val[m] = src[m];
    put_ghosts<M>(D, f, x, y, z, val);
}

// darcy.cuh:1101-1157 findDarcyPressureGradient (and :1535-1593
// findDarcyPermeabilityGradients): central differences
__global__ void k_darcy_grad(DarcyArgs D, const double *f, double *g, int gated)
{
    if (gated && !fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const double xn = f[d_idx(D, x - 1, y, z)], xp = f[d_idx(D, x + 1, y, z)];
    const double yn = f[d_idx(D, x, y - 1, z)], yp = f[d_idx(D, x, y + 1, z)];
    const double zn = f[d_idx(D, x, y, z - 1)], zp = f[d_idx(D, x, y, z + 1)];
    st3(g + 3 * (size_t)d_idx(D, x, y, z),
        mk((xp - xn) / (D.dx + D.dx), (yp - yn) / (D.dy + D.dy), (zp - zn) / (D.dz + D.dz)));
}

// darcy.cuh:1160-1318 findDarcyPressureForceLinear, per sphere: the index
// sums are unsigned as the reference's (a sphere in the bottom layer
// compares 0xffffffff with wall0_iz - 1)
__global__ void k_darcy_force(StepArgs A, DarcyArgs D)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const DevBox &B = A.boxes[0];
    const SphDarcy &P = D.prm;
    const uint32_t wall0_iz = D.st->wall0_iz;
    const double4 x = A.x[i];
    const d3 x3 = mk(x.x, x.y, x.z);
    const uint32_t i_x = (uint32_t)floor((x.x - B.origo[0]) / (B.L[0] / B.num[0]));
    const uint32_t i_y = (uint32_t)floor((x.y - B.origo[1]) / (B.L[1] / B.num[1]));
    const uint32_t i_z = (uint32_t)floor((x.z - B.origo[2]) / (B.L[2] / B.num[2]));
    const uint32_t nx = B.num[0], ny = B.num[1], nz = B.num[2];
    if (!(x.x >= B.origo[0] && x.y >= B.origo[1] && x.z >= B.origo[2]) || i_x >= nx ||
        i_y >= ny || i_z >= nz) {
        // a sphere outside the grid (the reference reads past its arrays):
        // no pressure force
        raise_flag(A.err, SPH_ERR_OUT_OF_GRID);
        D.f_p[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        return;
    }
    const double dx = B.L[0] / nx, dy = B.L[1] / ny, dz = B.L[2] / nz;
    const d3 X = mk(i_x * dx + 0.5 * dx, i_y * dy + 0.5 * dy, i_z * dz + 0.5 * dz);
    d3 grad_p = mk(0., 0., 0.);
    for (int d_iz = -1; d_iz < 2; d_iz++)
        for (int d_iy = -1; d_iy < 2; d_iy++)
            for (int d_ix = -1; d_ix < 2; d_ix++) {
                const int ix_n = (int)(i_x + (uint32_t)d_ix);
                const int iy_n = (int)(i_y + (uint32_t)d_iy);
                const int iz_n = (int)(i_z + (uint32_t)d_iz);
                d3 gpi = ld3(D.grad_p + 3 * (size_t)d_idx(D, ix_n, iy_n, iz_n));
                if ((ix_n == -1 && iy_n == -1) || (ix_n == -1 && iz_n == -1) ||
                    (iy_n == -1 && iz_n == -1) || (ix_n == (int)nx && iy_n == (int)ny) ||
                    (ix_n == (int)nx && iz_n == (int)nz) || (iy_n == (int)ny && iz_n == (int)nz) ||
                    (ix_n == (int)nx && iy_n == -1) || (ix_n == (int)nx && iz_n == -1) ||
                    (iy_n == (int)ny && ix_n == -1) || (iy_n == (int)ny && iz_n == -1) ||
                    (iz_n == (int)nz && ix_n == -1) || (iz_n == (int)nz && iy_n == -1))
                    gpi = mk(0., 0., 0.);
                if (P.bc_top == 0 && i_z + (uint32_t)d_iz >= wall0_iz - 1u) gpi.z = 0.0;
                const d3 n = mk(dx * d_ix, dy * d_iy, dz * d_iz);
                const double w = weight_dist(vsub(x3, vadd(X, n)), dx, dy, dz);
                grad_p = vadd(grad_p, smul(w, gpi));
            }
    const double v = sphere_volume(x.w);
    d3 f_p = vsub(muls(smul(-1.0, grad_p), v), smul(P.rho_f * v, mk(B.P.g[0], B.P.g[1], B.P.g[2])));
    if (P.bc_top == 0 && i_z >= wall0_iz) f_p.z = 0.0;
    const double4 F = A.force[i];
    A.force[i] = make_double4(F.x + f_p.x, F.y + f_p.y, F.z + f_p.z, F.w + 0.0);
    D.f_p[i] = make_double4(f_p.x, f_p.y, f_p.z, 0.0);
}

// ------------------------------------------------- the fluid update steps

// darcy.cuh:392-730 findDarcyPorositiesLinear: per cell, the solid volume
// of the spheres of the 27 cells around it under the trilinear hat centred
// on the cell, now and after an Euler step of the positions; the
// volume-weighted mean sphere velocity.  Spheres in sorted order.
__global__ void k_darcy_porosity(StepArgs A, DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const DevBox &B = A.boxes[0];
    const uint32_t cellidx = d_idx(D, x, y, z);
    if (A.ntot == 0) {
        D.phi[cellidx] = 0.9;
        D.dphi[cellidx] = 0.0;
        return;
    }
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const double dt = B.dt;
    double solid_volume = 0.0, solid_volume_new = 0.0;
    const d3 X = mk(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
    d3 vp_avg_num = mk(0.0, 0.0, 0.0);
    double vp_avg_denum = 0.0;
    const double phi_0 = D.phi[cellidx];
    for (int z_dim = -1; z_dim < 2; ++z_dim)
        for (int y_dim = -1; y_dim < 2; ++y_dim)
            for (int x_dim = -1; x_dim < 2; ++x_dim) {
                int tx = x + x_dim, ty = y + y_dim, tz = z + z_dim;
                if (tz == -1) tz = 1;
                if (B.periodic == 2) {
                    if (ty == -1) ty = 1;
                    if (ty == (int)B.num[1]) ty = (int)B.num[1] - 2;
                }
                int sx, sy;
                if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                const d3 distmod = shift_vec(B, sx, sy);
                const uint32_t cell = B.cell_base + (uint32_t)tx + (uint32_t)ty * B.num[0] +
                                      (B.num[0] * B.num[1]) * (uint32_t)tz;
                const uint32_t start = A.cell_off[cell], end = start + A.cell_count[cell];
                for (uint32_t a = start; a < end; ++a) {
                    double4 xr = A.xs[a];
                    const double4 vv = A.vs[a];
                    d3 dist = vadd(mk(X.x - xr.x, X.y - xr.y, X.z - xr.z), distmod);
                    const double sw = weight_dist(dist, dx, dy, dz);
                    const double vol_p = sphere_volume(xr.w);
                    solid_volume += sw * vol_p;
                    vp_avg_num = vadd(vp_avg_num, smul(sw * vol_p, mk(vv.x, vv.y, vv.z)));
                    vp_avg_denum += sw * vol_p;
                    xr.x += vv.x * dt;
                    xr.y += vv.y * dt;
                    xr.z += vv.z * dt;
                    dist = vadd(mk(X.x - xr.x, X.y - xr.y, X.z - xr.z), distmod);
                    solid_volume_new += weight_dist(dist, dx, dy, dz) * vol_p;
                }
            }
    double cell_volume = dx * dy * dz;
    if (z == D.nz - 1) cell_volume *= 0.875;
    const double phi = fmin(0.9, fmax(0.1, 1.0 - solid_volume / cell_volume));
    const double phi_new = fmin(0.9, fmax(0.1, 1.0 - solid_volume_new / cell_volume));
    double dphi;
    d3 vp_avg;
    if (B.iter == 0) {
        dphi = 0.0;
        vp_avg = mk(0.0, 0.0, 0.0);
    } else {
        dphi = 0.5 * (phi_new - phi_0);
        vp_avg = divs(vp_avg_num, fmax(1.0e-16, vp_avg_denum));
    }
    D.phi[cellidx] = phi * D.prm.c_phi;
    D.dphi[cellidx] = dphi * D.prm.c_phi;
    st3(D.vp_avg + 3 * (size_t)cellidx, vp_avg);
}

// darcy.cuh:733-807 copyDarcyPorositiesToEdges, then ...ToBottom
// (periodic == 2): phi, dphi, div_v_p, vp_avg of the y edge layers from
// the layer inside each, then of the bottom layer from the layer above
__device__ __forceinline__ void copy_cell(const DarcyArgs &D, uint32_t w, uint32_t r)
{
    D.phi[w] = D.phi[r];
    D.dphi[w] = D.dphi[r];
    D.div_v_p[w] = D.div_v_p[r];
    st3(D.vp_avg + 3 * (size_t)w, ld3(D.vp_avg + 3 * (size_t)r));
}

__global__ void k_darcy_edges(DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    if (!(y == 0 || y == D.ny - 1)) return;
    int y_read = 0;
    if (y == 0) y_read = 1;
    if (y == D.ny - 1) y_read = D.ny - 2;
    copy_cell(D, d_idx(D, x, y, z), d_idx(D, x, y_read, z));
}

__global__ void k_darcy_bottom(DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    if (z != 0) return;
    copy_cell(D, d_idx(D, x, y, 0), d_idx(D, x, y, 1));
}

// darcy.cuh:1414-1459 setDarcyTopPressure then setDarcyTopWallPressure:
// one thread per thread of the reference's launch grid (blocks of
// 8 x 8 x 8 covering the cells)
__global__ void k_darcy_top_pressure(DarcyArgs D, int gx, int gy, int gz, int wall_pass)
{
    if (!fluid_step(D)) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint32_t)gx * (uint32_t)gy * (uint32_t)gz) return;
    const int z = (int)(t / ((uint32_t)gx * (uint32_t)gy));
    const uint32_t r = t - (uint32_t)z * (uint32_t)gx * (uint32_t)gy;
    const int y = (int)(r / (uint32_t)gx), x = (int)(r - (uint32_t)y * (uint32_t)gx);
    const DarcyState *s = D.st;
    const double new_pressure = D.pmod[s->qstep % DARCY_RING];
    const uint32_t wall0_iz = s->wall0_iz;
    if (!wall_pass) {
        if ((x < D.nx && y < D.ny && z == D.nz - 1) || (uint32_t)z == wall0_iz) {
            const uint32_t k = d_idx(D, x, y, z);
            if (k < D.ncell) D.p[k] = new_pressure;
        }
    } else if (x < D.nx && y < D.ny && (uint32_t)z == wall0_iz) {
        D.p[d_idx(D, x, y, z)] = new_pressure;
    }
}

// darcy.cuh:1485-1532 findDarcyPermeabilities (Kozeny-Carman, capped)
__global__ void k_darcy_perm(DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const uint32_t ci = d_idx(D, x, y, z);
    double phi = D.phi[ci];
    if (phi > 0.9999) phi = 0.9999;
    const double q = 1.0 - phi;
    double k = D.prm.k_c * cube_rn(phi) / __dmul_rn(q, q);
    k = fmin(2.7e-10, k);
    D.k[ci] = k;
}

// darcy.cuh:288-329 setDarcyGhostNodesFlux (bc 4 at the bottom or top)
__global__ void k_darcy_flux(StepArgs A, DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const SphDarcy &P = D.prm;
    const double p = D.p[d_idx(D, x, y, z)];
    const double k = D.k[d_idx(D, x, y, z)];
    const double dz = A.boxes[0].L[2] / D.nz;
    double q_z = 0.;
    if (z == 0) q_z = P.bc_bot_flux;
    else if (z == D.nz - 1) q_z = P.bc_top_flux;
    const double p_ghost = -P.mu / k * q_z * dz + p;
    if (z == 0 && P.bc_bot == 4) D.p[d_idx(D, x, y, -1)] = p_ghost;
    if (z == D.nz - 1 && P.bc_top == 4) D.p[d_idx(D, x, y, D.nz)] = p_ghost;
}

// Before the Jacobi loop (device.cu:2193-2254): p_old = p (copyValues)
// and the ghost layer of p
__global__ void k_darcy_pre(DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const uint32_t ci = d_idx(D, x, y, z);
    const double val = D.p[ci];
    D.p_old[ci] = val;
    put_ghosts<1>(D, D.p, x, y, z, &val);
}

// darcy.cuh:1644-1923 firstDarcySolution and :1926-2226
// updateDarcySolution: the pressure change
//   ndt/(beta_f phi mu) div(k grad p) - ndt/(beta_f phi (1 - phi))
//                                       (dphi/ndt + vp_avg . grad phi),
// div(k grad p) with the harmonic means of k across the faces, zero at
// Dirichlet boundaries, at and above the wall with a Dirichlet top, and in
// cells of constant pressure (the +y test compares y with nx - 1, as
// written).  Everything but the pressures stays fixed during a solve, so
// k_darcy_first computes it once per fluid step with the reference's
// subexpressions (the same roundings): for each face the harmonic mean
// 2 k_n k / (k_n + k), the factor ndt/(beta_f phi mu), the forcing term,
// and whether the change is zero; dp_of then gives the change of any
// pressure field with the reference's remaining operations and order.
struct DpCoef {
    double a[6];   // faces xp, xn, yp, yn, zp, zn
    double c1, f, zero;
};

__device__ __forceinline__ DpCoef load_coef(const DarcyArgs &D, uint32_t c, uint32_t ncells)
{
    DpCoef q;
#pragma unroll
    for (int k = 0; k < 6; ++k) q.a[k] = D.coef[(size_t)k * ncells + c];
    q.c1 = D.coef[(size_t)6 * ncells + c];
    q.f = D.coef[(size_t)7 * ncells + c];
    q.zero = D.coef[(size_t)8 * ncells + c];
    return q;
}

// a / b correctly rounded for a divisor b that stays fixed (the cell
// sizes), from rb = RN(1 / b), by Markstein's correction (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(a rb) lies within one
// ulp of a / b, the remainder r = a - b q0 is exact (one FMA), and
// RN(q0 + r rb) is the correctly rounded quotient while q0 is a normal
// number away from the ends of the range.  A zero a gives q0 = +-0, the
// quotient with its sign (rb has the sign of b); tiny, huge, infinite and
// NaN q0 take the division itself.  One multiply and two FMAs instead of a
// division sequence -- and no division at all for the zero differences of
// a pressure field at rest, which are most of them in a layered pack.
struct CellInv {
    double rx, ry, rz;
};
__device__ __forceinline__ CellInv cell_inv(const DarcyArgs &D)
{
    return CellInv{1.0 / D.dx, 1.0 / D.dy, 1.0 / D.dz};
}
__device__ __forceinline__ double div_fixed(double a, double b, double rb)
{
    const double q0 = __dmul_rn(a, rb);
    const double aq = fabs(q0);
    if (aq > 0x1p-900 && aq < 0x1p+1000) return __fma_rn(__fma_rn(-q0, b, a), rb, q0);
    if (a == 0.0) return q0;
    return a / b;
}

// The pressure change from the pressures of the cell and its six
// neighbours (no-flow faces already replaced by the cell's own), with the
// divisions by the cell sizes as div_fixed (the same quotients).  It is
// evaluated also for a cell whose change is zero (the value is then
// dropped), so that the stencil's loads need not wait for the flag.
__device__ __forceinline__ double dp_stencil(const DarcyArgs &D, const DpCoef &q, const CellInv &iv,
                                             double p, double p_xn, double p_xp, double p_yn,
                                             double p_yp, double p_zn, double p_zp)
{
    // (a0 (p_xp - p) / dx - a1 (p - p_xn) / dx) / dx + ... (y, z alike)
    auto axis = [&](double a_p, double a_n, double pp, double pn_, double h, double rh) {
        const double t1 = div_fixed(a_p * (pp - p), h, rh);
        const double t2 = div_fixed(a_n * (p - pn_), h, rh);
        return div_fixed(t1 - t2, h, rh);
    };
    const double div_k_grad_p = axis(q.a[0], q.a[1], p_xp, p_xn, D.dx, iv.rx) +
                                axis(q.a[2], q.a[3], p_yp, p_yn, D.dy, iv.ry) +
                                axis(q.a[4], q.a[5], p_zp, p_zn, D.dz, iv.rz);
    const double dp = q.c1 * div_k_grad_p - q.f;
    return q.zero != 0.0 ? 0.0 : dp;
}

// The pressure change of cell (x, y, z) for the pressure field pf.
__device__ __forceinline__ double dp_of(const DarcyArgs &D, const DpCoef &q, const double *pf, int x,
                                        int y, int z, const CellInv &iv)
{
    const SphDarcy &P = D.prm;
    double p_xn = pf[d_idx(D, x - 1, y, z)];
    const double p = pf[d_idx(D, x, y, z)];
    double p_xp = pf[d_idx(D, x + 1, y, z)];
    double p_yn = pf[d_idx(D, x, y - 1, z)], p_yp = pf[d_idx(D, x, y + 1, z)];
    double p_zn = pf[d_idx(D, x, y, z - 1)], p_zp = pf[d_idx(D, x, y, z + 1)];
    if (x == 0 && P.bc_xn == 1) p_xn = p;
    if (x == D.nx - 1 && P.bc_xp == 1) p_xp = p;
    if (y == 0 && P.bc_yn == 1) p_yn = p;
    if (y == D.ny - 1 && P.bc_yp == 1) p_yp = p;
    if (z == 0 && P.bc_bot == 1) p_zn = p;
    if (z == D.nz - 1 && P.bc_top == 1) p_zp = p;
    return dp_stencil(D, q, iv, p, p_xn, p_xp, p_yn, p_yp, p_zn, p_zp);
}

// The fixed parts of the pressure change of each cell (above), and the
// explicit change dp_expl from the pressure at the start of the solve.
__global__ void k_darcy_first(StepArgs A, DarcyArgs D)
{
    if (!fluid_step(D)) return;
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (!cell_of(D, c, x, y, z)) return;
    const uint32_t ncells = (uint32_t)D.nx * (uint32_t)D.ny * (uint32_t)D.nz;
    const SphDarcy &P = D.prm;
    const int nx = D.nx, nz = D.nz;
    const double dx = D.dx, dy = D.dy, dz = D.dz;
    const uint32_t ci = d_idx(D, x, y, z);
    const double phi_xn = D.phi[d_idx(D, x - 1, y, z)], phi = D.phi[ci];
    const double phi_xp = D.phi[d_idx(D, x + 1, y, z)];
    const double phi_yn = D.phi[d_idx(D, x, y - 1, z)], phi_yp = D.phi[d_idx(D, x, y + 1, z)];
    const double phi_zn = D.phi[d_idx(D, x, y, z - 1)], phi_zp = D.phi[d_idx(D, x, y, z + 1)];
    const double dphi = D.dphi[ci];
    const d3 vp_avg = ld3(D.vp_avg + 3 * (size_t)ci);
    const int p_constant = D.p_constant[ci];
    const double k_xn = D.k[d_idx(D, x - 1, y, z)], k = D.k[ci];
    const double k_xp = D.k[d_idx(D, x + 1, y, z)];
    const double k_yn = D.k[d_idx(D, x, y - 1, z)], k_yp = D.k[d_idx(D, x, y + 1, z)];
    const double k_zn = D.k[d_idx(D, x, y, z - 1)], k_zp = D.k[d_idx(D, x, y, z + 1)];
    const d3 grad_phi = mk((phi_xp - phi_xn) / (dx + dx), (phi_yp - phi_yn) / (dy + dy),
                           (phi_zp - phi_zn) / (dz + dz));
    const double ndt = P.ndem * A.boxes[0].dt;
    DpCoef q;
    q.a[0] = 2. * k_xp * k / (k_xp + k);
    q.a[1] = 2. * k_xn * k / (k_xn + k);
    q.a[2] = 2. * k_yp * k / (k_yp + k);
    q.a[3] = 2. * k_yn * k / (k_yn + k);
    q.a[4] = 2. * k_zp * k / (k_zp + k);
    q.a[5] = 2. * k_zn * k / (k_zn + k);
    q.c1 = ndt / (P.beta_f * phi * P.mu);
    q.f = (ndt / (P.beta_f * phi * (1.0 - phi))) * (dphi / ndt + dot(vp_avg, grad_phi));
    q.zero = ((P.bc_bot == 0 && z == 0) || (P.bc_top == 0 && z == nz - 1) ||
              ((uint32_t)z >= D.st->wall0_iz && P.bc_top == 0) || (P.bc_xn == 0 && x == 0) ||
              (P.bc_xp == 0 && x == nx - 1) || (P.bc_yn == 0 && y == 0) ||
              (P.bc_yp == 0 && y == nx - 1) || p_constant == 1)
                 ? 1.0
                 : 0.0;
#pragma unroll
    for (int m = 0; m < 6; ++m) D.coef[(size_t)m * ncells + c] = q.a[m];
    D.coef[(size_t)6 * ncells + c] = q.c1;
    D.coef[(size_t)7 * ncells + c] = q.f;
    D.coef[(size_t)8 * ncells + c] = q.zero;
    D.dp_expl[ci] = dp_of(D, q, D.p, x, y, z, cell_inv(D));
}

// A cell of the Jacobi loop with what stays fixed for it during a solve:
// its coordinates and padded index, the coefficients of its pressure
// change, the part of the new pressure that does not depend on the iterate
// (p_old + (1 - epsilon) dp_expl, the reference's first two terms), the
// term of the flux ghost (-mu / k q_z dz, bc 4), and flags: bits 0-17 the
// ghost cells that copy it (ghost_bits), 18-23 the neighbours (xn, xp, yn,
// yp, zn, zp) a no-flow face (bc 1) replaces by the cell itself, 24 and 25
// the flux ghost below and above.
struct JCell {
    int x, y, z;
    uint32_t ci, bits;
    DpCoef q;
    double base, flux_t;
};

constexpr double JACOBI_EPSILON = 0.5;   // darcy.cuh updateDarcySolution
constexpr double JACOBI_THETA = 0.05;

__device__ __forceinline__ JCell jcell_init(const DarcyArgs &D, uint32_t c, uint32_t ncells, double dzf)
{
    const SphDarcy &P = D.prm;
    JCell j;
    cell_of(D, c, j.x, j.y, j.z);
    const int x = j.x, y = j.y, z = j.z;
    j.ci = d_idx(D, x, y, z);
    j.q = load_coef(D, c, ncells);
    j.base = D.p_old[j.ci] + (1.0 - JACOBI_EPSILON) * D.dp_expl[j.ci];
    uint32_t b = ghost_bits(D, x, y, z);
    b |= (uint32_t)(x == 0 && P.bc_xn == 1) << 18 | (uint32_t)(x == D.nx - 1 && P.bc_xp == 1) << 19 |
         (uint32_t)(y == 0 && P.bc_yn == 1) << 20 | (uint32_t)(y == D.ny - 1 && P.bc_yp == 1) << 21 |
         (uint32_t)(z == 0 && P.bc_bot == 1) << 22 | (uint32_t)(z == D.nz - 1 && P.bc_top == 1) << 23;
    j.flux_t = 0.0;
    if (P.bc_bot == 4 || P.bc_top == 4) {
        // darcy.cuh setDarcyGhostNodesFlux: p_ghost = -mu / k q_z dz + p
        double q_z = 0.;
        if (z == 0) q_z = P.bc_bot_flux;
        else if (z == D.nz - 1) q_z = P.bc_top_flux;
        j.flux_t = -P.mu / D.k[j.ci] * q_z * dzf;
        b |= (uint32_t)(z == 0 && P.bc_bot == 4) << 24 | (uint32_t)(z == D.nz - 1 && P.bc_top == 4) << 25;
    }
    j.bits = b;
    return j;
}

// One Jacobi update of the cell (reads pc, writes pn), and on a checked
// iteration its normalised residual into the running maximum.
__device__ __forceinline__ void jcell_update(const DarcyArgs &D, const JCell &j, const double *pc,
                                             double *pn, const CellInv &iv, bool check,
                                             unsigned long long &bmax, uint32_t &bnan)
{
    const uint32_t sy = (uint32_t)D.nx + 2u, sz = sy * ((uint32_t)D.ny + 2u);
    const uint32_t ci = j.ci;
    const double p = __ldcg(pc + ci);
    double p_xn = __ldcg(pc + ci - 1u), p_xp = __ldcg(pc + ci + 1u);
    double p_yn = __ldcg(pc + ci - sy), p_yp = __ldcg(pc + ci + sy);
    double p_zn = __ldcg(pc + ci - sz), p_zp = __ldcg(pc + ci + sz);
    const uint32_t b = j.bits;
    if (b & (1u << 18)) p_xn = p;
    if (b & (1u << 19)) p_xp = p;
    if (b & (1u << 20)) p_yn = p;
    if (b & (1u << 21)) p_yp = p;
    if (b & (1u << 22)) p_zn = p;
    if (b & (1u << 23)) p_zp = p;
    const double dp_impl = dp_stencil(D, j.q, iv, p, p_xn, p_xp, p_yn, p_yp, p_zn, p_zp);
    double p_new = j.base + JACOBI_EPSILON * dp_impl;
    p_new = p * (1.0 - JACOBI_THETA) + p_new * JACOBI_THETA;
    if (b & (1u << 24)) __stcg(pn + ci - sz, j.flux_t + p);
    if (b & (1u << 25)) __stcg(pn + ci + sz, j.flux_t + p);
    __stcg(pn + ci, p_new);
    if (b & 0x3ffffu) put_ghost_bits<1>(D, pn, j.x, j.y, j.z, b & 0x3ffffu, &p_new);
    if (check) {
        // the normalised residual; a zero change skips the division (its
        // quotient is +-0 unless the divisor is zero or NaN)
        const double num = p_new - p, den = p + 1.0e-16;
        const double r = (num == 0.0 && den == den && den != 0.0) ? 0.0 : fabs(num / den);
        if (r != r) {
            bnan = 1u;
        } else {
            const unsigned long long v = (unsigned long long)__double_as_longlong(r);
            bmax = v > bmax ? v : bmax;
        }
    }
}

// The Jacobi loop of one fluid step (device.cu:2218-2376) as one
// cooperative launch, the blocks taking the cells in turn, the pressure in
// two arrays that alternate (D.p and D.p_new): iteration n reads array
// n % 2 and writes the other.  Per iteration, per cell:
//  - updateDarcySolution: the new pressure and its normalised residual;
//  - setDarcyGhostNodesFlux (bc 4) from the cell's pressure before the
//    update, into the other array's ghost layer;
//  - copyValues(p_new -> p) and the ghost layer of the new pressure (the
//    reference's setDarcyGhostNodes at the start of the next iteration, or
//    after the loop): the new value into the other array with the ghost
//    cells that copy it;
// then a grid barrier.  With bc_top == 1, setDarcyTopWallFixedFlow (p at
// z = wall0_iz + 1 from z = wall0_iz - 1 in the array just read) runs
// between two barriers.  Every tenth iteration (src/debug.h:16 nijacnorm)
// each block's largest |residual| (the bits of a non-negative double,
// which order as the values do) and whether one was NaN go to the block's
// slot as it arrives at the barrier; after the barrier each warp reads all
// slots and takes the same decision as every other warp: stop when the
// largest residual is within the tolerance, or one was NaN (SPH_ERR_NAN);
// stop after maxiter iterations.  The final pressure ends up in D.p.  The
// barrier counts arrivals on a counter that only grows (D.bar, zeroed
// before the launch) and is bounded (SPH_ERR_TIMEOUT); the pressures other
// blocks write are read past L1.  Block 0 logs the solve.
// ONE: every thread has at most one cell, whose fixed state (JCell) it
// keeps in registers for the whole solve; otherwise each thread takes its
// cells in turn and gathers their state at every iteration.
template <bool ONE>
__global__ void __launch_bounds__(JACOBI_THREADS, 1) k_darcy_jacobi(StepArgs A, DarcyArgs D)
{
    __shared__ unsigned long long s_max[JACOBI_THREADS / 32];
    __shared__ uint32_t s_nan[JACOBI_THREADS / 32];
    DarcyState *st = D.st;
    const SphDarcy &P = D.prm;
    if (!(st->active && P.maxiter > 0)) return;   // the same in every block
    const uint32_t ncells = (uint32_t)D.nx * (uint32_t)D.ny * (uint32_t)D.nz;
    const uint32_t nxy = (uint32_t)D.nx * (uint32_t)D.ny;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const int gz = (D.nz + 7) / 8 * 8;
    const uint32_t wall0_iz = st->wall0_iz;
    const double dzf = A.boxes[0].L[2] / D.nz;
    double *const buf[2] = {D.p, D.p_new};
    const CellInv iv = cell_inv(D);
    const bool mine = first < ncells;
    JCell own;
    if (ONE && mine) own = jcell_init(D, first, ncells, dzf);
    unsigned long long target = 0ull;   // arrivals the next barrier waits for
    auto no_arrival_work = [] {};
    uint32_t nijac = 0;
    int ok = 0, bad = 0;
    for (;;) {
        double *pc = buf[nijac & 1u];
        double *pn = buf[(nijac & 1u) ^ 1u];
        const bool check = (nijac % 10u) == 0u;
        unsigned long long bmax = 0ull;
        uint32_t bnan = 0u;
        if (ONE) {
            if (mine) jcell_update(D, own, pc, pn, iv, check, bmax, bnan);
        } else {
            for (uint32_t c = first; c < ncells; c += stride)
                jcell_update(D, jcell_init(D, c, ncells, dzf), pc, pn, iv, check, bmax, bnan);
        }
        if (check) {
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long b = __shfl_xor_sync(0xffffffffu, bmax, o);
                bmax = b > bmax ? b : bmax;
            }
            const uint32_t anynan = __any_sync(0xffffffffu, bnan != 0u) ? 1u : 0u;
            if (lane == 0) {
                s_max[warp] = bmax;
                s_nan[warp] = anynan;
            }
        }
        if (P.bc_top == 1) {
            // after every cell has read the array it writes; cells past the
            // padded array (a wall at or above the top of the grid) are
            // skipped
            target += gridDim.x;
            if (!grid_sync_count(D.bar, target, BARRIER_LIMIT_NS, A.err, no_arrival_work)) return;
            const uint32_t z = wall0_iz + 1u;
            if (z < (uint32_t)gz)
                for (uint32_t t = first; t < nxy; t += stride) {
                    const int y = (int)(t / (uint32_t)D.nx), x = (int)(t - (uint32_t)y * (uint32_t)D.nx);
                    const uint32_t w = d_idx(D, x, y, (int)z), r = d_idx(D, x, y, (int)z - 2);
                    if (w < D.ncell && r < D.ncell) __stcg(pc + w, __ldcg(pc + r));
                }
        }
        // the block's largest residual goes out with its arrival (thread 0,
        // after the block barrier that makes the warps' values visible)
        target += gridDim.x;
        const bool passed = grid_sync_count(D.bar, target, BARRIER_LIMIT_NS, A.err, [&] {
            if (!check) return;
            unsigned long long m = 0ull;
            uint32_t nn = 0u;
            for (int w = 0; w < JACOBI_THREADS / 32; ++w) {
                m = s_max[w] > m ? s_max[w] : m;
                nn |= s_nan[w];
            }
            __stcg(D.part_max + blockIdx.x, m);
            __stcg(D.part_nan + blockIdx.x, nn);
        });
        if (!passed) return;
        int stop = 0, good = 0, nanseen = 0;
        if (check) {
            // every warp reduces all blocks' slots itself: no block barrier
            unsigned long long m = 0ull;
            uint32_t nn = 0u;
            for (uint32_t b = lane; b < gridDim.x; b += 32u) {
                const unsigned long long v = __ldcg(D.part_max + b);
                m = v > m ? v : m;
                nn |= __ldcg(D.part_nan + b);
            }
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
                m = v > m ? v : m;
            }
            if (__any_sync(0xffffffffu, nn != 0u)) {
                stop = 1;
                nanseen = 1;
            } else if (__longlong_as_double((long long)m) <= P.tolerance) {
                stop = 1;
                good = 1;
            }
        }
        if (!stop && nijac == P.maxiter - 1u) stop = 1;
        if (stop) {
            ok = good;
            bad = nanseen;
            if (pn != D.p)   // the result in D.p (every cell: the ghost layer too)
                for (uint32_t c = first; c < D.ncell; c += stride) __stcg(D.p + c, __ldcg(pn + c));
            break;
        }
        ++nijac;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (bad) raise_flag(A.err, SPH_ERR_NAN);
        const unsigned long long h = st->log_head;
        const uint32_t slot = (uint32_t)(h % SPH_DARCY_LOG);
        D.log_step[slot] = A.boxes[0].iter + 1;
        D.log_iters[slot] = nijac;
        D.log_ok[slot] = (uint32_t)ok;
        st->log_head = h + 1;
        st->nijac = nijac;
    }
}

// After the loop: dphi zeroed unless an output follows this step
// (device.cu:2379-2386, the host file clock), then findDarcyVelocities
// (darcy.cuh:2267-2325) from the pressure whose ghost layer the loop's
// last copy wrote
__global__ void k_darcy_post(StepArgs A, DarcyArgs D)
{
    if (!fluid_step(D)) return;
    int x, y, z;
    if (!cell_of(D, blockIdx.x * blockDim.x + threadIdx.x, x, y, z)) return;
    const uint32_t ci = d_idx(D, x, y, z);
    if (D.st->filetimeclock + A.boxes[0].dt < D.prm.file_dt) D.dphi[ci] = 0.0;
    const double *p = D.p;
    const double xn = p[d_idx(D, x - 1, y, z)], xp = p[d_idx(D, x + 1, y, z)];
    const double yn = p[d_idx(D, x, y - 1, z)], yp = p[d_idx(D, x, y + 1, z)];
    const double zn = p[d_idx(D, x, y, z - 1)], zp = p[d_idx(D, x, y, z + 1)];
    const double k = D.k[ci], phi = D.phi[ci];
    const d3 grad_p = mk((xp - xn) / (D.dx + D.dx), (yp - yn) / (D.dy + D.dy), (zp - zn) / (D.dz + D.dz));
    st3(D.v + 3 * (size_t)ci, divs(smul(-k / D.prm.mu, grad_p), phi));
}

// After the step's wall stage (device.cu:2537, 2569, 2672, 805): the file
// clock; at an output the host copy of wall 0 is refreshed; the step count
__global__ void k_darcy_tick(StepArgs A, DarcyArgs D)
{
    const DevBox &B = A.boxes[0];
    DarcyState *s = D.st;
    s->filetimeclock += B.dt;
    if (s->filetimeclock >= D.prm.file_dt) {
        s->filetimeclock = 0.0;
        if (B.nw > 0) s->wall_w_host = B.wnx[0][3];
    }
    s->qstep += 1;
}

static inline void record(cudaEvent_t ev, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    else cudaEventRecord(ev, st);
}

static inline void mark(Prof *prof, cudaStream_t st, const char *name)
{
    if (!prof || prof->n >= Prof::MAX) return;
    prof->name[prof->n] = name;
    record(prof->ev[prof->n + 1], st);
    prof->n++;
}

}  // namespace

int launch_darcy(const StepArgs &A, const DarcyArgs &D, const StepConfig &cfg, cudaStream_t st,
                 uint64_t *launches, Prof *prof)
{
    uint64_t nl = 0;
    const SphDarcy &P = D.prm;
    const uint32_t ncells = (uint32_t)D.nx * D.ny * D.nz;
    const unsigned gc = blocks_for(ncells, DARCY_THREADS);
    k_darcy_begin<<<1, 1, 0, st>>>(A, D);
    nl += 1;
    if (A.ntot > 0) {
        k_darcy_ghost<1><<<gc, DARCY_THREADS, 0, st>>>(D, D.p, 0);
        k_darcy_grad<<<gc, DARCY_THREADS, 0, st>>>(D, D.p, D.grad_p, 0);
        k_darcy_ghost<3><<<gc, DARCY_THREADS, 0, st>>>(D, D.grad_p, 0);
        k_darcy_force<<<blocks_for(A.ntot, DARCY_THREADS), DARCY_THREADS, 0, st>>>(A, D);
        mark(prof, st, "k_darcy_force");
        nl += 4;
    }
    // the fluid update: every kernel returns at once unless iter % ndem == 0
    k_darcy_porosity<<<gc, DARCY_THREADS, 0, st>>>(A, D);
    nl += 1;
    if (D.periodic == 2) {
        k_darcy_edges<<<gc, DARCY_THREADS, 0, st>>>(D);
        k_darcy_bottom<<<gc, DARCY_THREADS, 0, st>>>(D);
        nl += 2;
    }
    if (D.pmod) {
        const int gx = (D.nx + 7) / 8 * 8, gy = (D.ny + 7) / 8 * 8, gz = (D.nz + 7) / 8 * 8;
        const unsigned gt = blocks_for((uint64_t)gx * gy * gz, DARCY_THREADS);
        k_darcy_top_pressure<<<gt, DARCY_THREADS, 0, st>>>(D, gx, gy, gz, 0);
        k_darcy_top_pressure<<<gt, DARCY_THREADS, 0, st>>>(D, gx, gy, gz, 1);
        nl += 2;
    }
    k_darcy_perm<<<gc, DARCY_THREADS, 0, st>>>(D);
    k_darcy_ghost<1><<<gc, DARCY_THREADS, 0, st>>>(D, D.phi, 1);
    k_darcy_ghost<1><<<gc, DARCY_THREADS, 0, st>>>(D, D.k, 1);
    k_darcy_grad<<<gc, DARCY_THREADS, 0, st>>>(D, D.k, D.grad_k, 1);
    nl += 4;
    if (P.bc_bot == 4 || P.bc_top == 4) {
        k_darcy_flux<<<gc, DARCY_THREADS, 0, st>>>(A, D);
        nl += 1;
    }
    k_darcy_pre<<<gc, DARCY_THREADS, 0, st>>>(D);
    k_darcy_first<<<gc, DARCY_THREADS, 0, st>>>(A, D);
    nl += 2;
    mark(prof, st, "k_darcy_fluid");
    // the Jacobi loop: one cooperative launch, as many blocks as can be
    // resident at once (at most one per JACOBI_THREADS cells); the launch
    // fails rather than run blocks that could not all be resident
    {
        static int per_sm = -1, sms = 0;
        if (per_sm < 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            int a = 0, b = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_darcy_jacobi<true>, JACOBI_THREADS, 0);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_darcy_jacobi<false>, JACOBI_THREADS, 0);
            per_sm = a < b ? a : b;
        }
        unsigned cap = (unsigned)(per_sm > 0 ? per_sm : 1) * (unsigned)sms;
        const unsigned need = blocks_for(ncells, JACOBI_THREADS);
        if (cap > DARCY_PARTS) cap = DARCY_PARTS;
        cudaMemsetAsync(D.bar, 0, sizeof(unsigned long long), st);
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(need < cap ? need : cap);
        c.blockDim = dim3(JACOBI_THREADS);
        c.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        c.attrs = at;
        c.numAttrs = 1;
        const bool one = (uint64_t)c.gridDim.x * JACOBI_THREADS >= ncells;
        const cudaError_t le = one ? cudaLaunchKernelEx(&c, k_darcy_jacobi<true>, A, D)
                                   : cudaLaunchKernelEx(&c, k_darcy_jacobi<false>, A, D);
        if (le != cudaSuccess) return SPH_ERR_CUDA;
        nl += 2;
    }
    mark(prof, st, "k_darcy_jacobi");
    k_darcy_post<<<gc, DARCY_THREADS, 0, st>>>(A, D);
    nl += 1;
    mark(prof, st, "k_darcy_post");
    if (launches) *launches += nl;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "sphere_b200: Darcy launch failed: %s\n", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

void launch_darcy_tick(const StepArgs &A, const DarcyArgs &D, cudaStream_t st)
{
    k_darcy_tick<<<1, 1, 0, st>>>(A, D);
}

}  // namespace sph
