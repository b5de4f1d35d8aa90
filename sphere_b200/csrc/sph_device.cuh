// sph_device.cuh -- device-side data model and FP64 contact laws of the
// B200 DEM step.
//
// Every expression keeps the operand order of the reference's device code
// (src/contactmodels.cuh, src/cohesion.cuh, src/vector_arithmetic.h), and the
// FP64 kernels are compiled without FMA contraction, so the FP64 form
// reproduces the reference's arithmetic bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sphere_b200.h"

namespace sph {

// Wait for the kernel before this one in the stream when launched as a
// programmatic dependent launch (launch_k); returns at once otherwise.
__device__ __forceinline__ void grid_dependency_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

constexpr int NC = SPH_NC;
constexpr uint32_t EMPTY = 0xffffffffu;     // free contact slot
constexpr uint32_t ID_MASK = 0x0fffffffu;   // partner index bits of a slot word
constexpr int CODE_SHIFT = 28;              // periodic image code bits 28..31
constexpr double PI = 3.14159265358979;     // src/constants.h:15

// Error bits (1 << SphStatus) accumulated in device memory.
__device__ __forceinline__ void raise_flag(uint32_t *err, int status)
{
    atomicOr(err, 1u << status);
}

// One independent simulation box.  Time-dependent members (walls, time,
// L[2] of an adaptive grid, velocity-step state) are advanced on the device
// by k_box_step so that a step needs no host round trip.
struct DevBox {
    SphParams P;
    double origo[3], L[3];
    uint32_t num[3];
    int32_t periodic, adaptive;
    uint32_t np, p_base;       // particles [p_base, p_base + np)
    uint32_t cell_base;        // global id of the box's first cell
    uint32_t nb0, b_base;      // bonds [b_base, b_base + nb0)
    uint32_t part_base;        // first per-256-particle partial sum
    uint32_t nblocks;          // ceil(np / 256)
    uint32_t nw;
    int32_t wmode[SPH_MAXWALLS];
    double wnx[SPH_MAXWALLS][4];
    double wmvfd[SPH_MAXWALLS][4];
    double wacc[SPH_MAXWALLS];
    double tau_x;
    double tau_eff_x;          // sum of shear-stress partials (wmode 3)
    double dt, t_current;
    double L2_out;             // grid.L[2] of the last step (what an output file holds)
    float pre_margin;          // FP32 candidate prefilter margin (see k_interact)
    // neighbour lists (k_vlist_build): pairs closer than ra + rb + vskin
    // at the last build; rebuilt once a sphere has moved more than
    // sqrt(vdisp2) (< vskin / 2) since; candidates searched over
    // +-vrange cells
    float vskin;
    float vdisp2;
    int32_t vrange;
    uint64_t iter;
    int32_t velocity_state;
    int32_t change_velocity_state;
};

struct d3 {
    double x, y, z;
};

__device__ __forceinline__ d3 mk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 vadd(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ d3 vsub(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ d3 vadds(d3 a, double b) { return mk(a.x + b, a.y + b, a.z + b); }
__device__ __forceinline__ d3 smul(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ d3 muls(d3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ d3 divs(d3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ d3 vneg(d3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ d3 xyz(double4 v) { return mk(v.x, v.y, v.z); }

// Vector length.  LM == SPH_LEN_REFERENCE: sqrtf of the FP64 dot product
// (src/vector_arithmetic.h:317-320), i.e. rounded to FP32.
template <int LM>
__device__ __forceinline__ double vlen(d3 v)
{
    const double d = dot(v, v);
    if (LM == SPH_LEN_FP64) return sqrt(d);
    return (double)__fsqrt_rn(__double2float_rn(d));
}
__device__ __forceinline__ double fsqrtf_d(double d)
{
    return (double)__fsqrt_rn(__double2float_rn(d));
}

// Per-sphere sums of a step; the contact laws add to them through these
// members, in a fixed order per field.
struct Acc {
    d3 F, T;
    double es_dot, ev_dot, p;
    __device__ __forceinline__ void addF(d3 v) { F = vadd(F, v); }
    __device__ __forceinline__ void addT(d3 v) { T = vadd(T, v); }
    __device__ __forceinline__ void addEs(double v) { es_dot += v; }
    __device__ __forceinline__ void addEv(double v) { ev_dot += v; }
    __device__ __forceinline__ void addP(double v) { p += v; }
};

// The additions one contact law call makes, recorded instead of applied
// (contact laws add F, T and p once, es_dot at most once and ev_dot at
// most twice), so that another thread can replay them into the sphere's
// sums in slot order with the same rounding.  nev < 0 marks a slot whose
// contact ended this step (nothing to add).
struct ContactRec {
    d3 F, T;
    double ev0, ev1, es, p;
    int32_t nev, nes;
    __device__ __forceinline__ void addF(d3 v) { F = v; }
    __device__ __forceinline__ void addT(d3 v) { T = v; }
    __device__ __forceinline__ void addEs(double v) { es = v; nes = 1; }
    __device__ __forceinline__ void addEv(double v)
    {
        if (nev == 0) ev0 = v;
        else ev1 = v;
        ++nev;
    }
    __device__ __forceinline__ void addP(double v) { p = v; }
};

__device__ __forceinline__ void replay(Acc &a, const ContactRec &r)
{
    a.addF(r.F);
    a.addT(r.T);
    if (r.nev > 0) a.addEv(r.ev0);
    if (r.nev > 1) a.addEv(r.ev1);
    if (r.nes) a.addEs(r.es);
    a.addP(r.p);
}

// Periodic image of a neighbour cell: src/contactsearch.cuh:12-83
// (findDistMod).  Returns false when the cell lies outside the grid; sx, sy
// receive the image shift in units of L[0], L[1].
__device__ __forceinline__ bool image_cell(const DevBox &B, int &tx, int &ty, int tz, int &sx,
                                           int &sy)
{
    sx = 0;
    sy = 0;
    const int nx = (int)B.num[0], ny = (int)B.num[1], nz = (int)B.num[2];
    if (B.periodic == 1) {
        if (tx < 0) { tx += nx; sx = 1; }
        if (tx >= nx) { tx -= nx; sx = -1; }
        if (ty < 0) { ty += ny; sy = 1; }
        if (ty >= ny) { ty -= ny; sy = -1; }
    } else if (B.periodic == 2) {
        if (tx < 0) { tx += nx; sx = 1; }
        if (tx >= nx) { tx -= nx; sx = -1; }
        if (ty < 0 || ty >= ny) return false;
    } else {
        if (tx < 0 || tx >= nx) return false;
        if (ty < 0 || ty >= ny) return false;
    }
    if (tz < 0 || tz >= nz) return false;
    // A particle far outside the grid (already flagged SPH_ERR_OUT_OF_GRID by
    // k_hash) can still be outside after one periodic wrap; never index
    // outside the box's cells.
    if (tx < 0 || tx >= nx || ty < 0 || ty >= ny) return false;
    return true;
}

// Cell coordinates packed 21 bits each (k_hash writes them per sphere).
__device__ __forceinline__ uint64_t pack_cell(uint32_t x, uint32_t y, uint32_t z)
{
    return (uint64_t)x | ((uint64_t)y << 21) | ((uint64_t)z << 42);
}
__device__ __forceinline__ void unpack_cell(uint64_t c, int &x, int &y, int &z)
{
    x = (int)(c & 0x1fffffu);
    y = (int)((c >> 21) & 0x1fffffu);
    z = (int)((c >> 42) & 0x1fffffu);
}

// The neighbour-cell offset (dx, dy, dz in -1..1) and image shift (sx, sy)
// under which the cell search around cell g visits a sphere in cell b,
// i.e. the inverse of image_cell; false when the search never visits b's
// cell.  Needs num >= 3 along periodic axes (checked at sph_create), which
// makes the offset unique.
__device__ __forceinline__ bool relative_cell(const DevBox &B, const int g[3], int bx, int by,
                                              int bz, int &dx, int &dy, int &dz, int &sx, int &sy)
{
    dz = bz - g[2];
    if (dz < -1 || dz > 1) return false;
    const int nx = (int)B.num[0], ny = (int)B.num[1];
    sx = 0;
    sy = 0;
    dx = bx - g[0];
    if (dx < -1 || dx > 1) {
        if (B.periodic != 1 && B.periodic != 2) return false;
        if (dx == nx - 1 && g[0] == 0) { dx = -1; sx = 1; }
        else if (dx == 1 - nx && g[0] == nx - 1) { dx = 1; sx = -1; }
        else return false;
    }
    dy = by - g[1];
    if (dy < -1 || dy > 1) {
        if (B.periodic != 1) return false;
        if (dy == ny - 1 && g[1] == 0) { dy = -1; sy = 1; }
        else if (dy == 1 - ny && g[1] == ny - 1) { dy = 1; sy = -1; }
        else return false;
    }
    return true;
}

// Image shift vector exactly as findDistMod accumulates it from zero.
__device__ __forceinline__ d3 shift_vec(const DevBox &B, int sx, int sy)
{
    const double dx = sx == 0 ? 0.0 : (sx > 0 ? B.L[0] : -B.L[0]);
    const double dy = sy == 0 ? 0.0 : (sy > 0 ? B.L[1] : -B.L[1]);
    return mk(dx, dy, 0.0);
}

__device__ __forceinline__ uint32_t shift_code(int sx, int sy)
{
    return (uint32_t)(sx & 3) | ((uint32_t)(sy & 3) << 2);
}
__device__ __forceinline__ void decode_shift(uint32_t code, int &sx, int &sy)
{
    sx = (int)(code & 3u);
    sy = (int)((code >> 2) & 3u);
    if (sx == 3) sx = -1;
    if (sy == 3) sy = -1;
}

// contactmodels.cuh:10-117 contactLinear_wall
template <int LM, class AccT>
__device__ __forceinline__ double contact_linear_wall(const SphParams &P, double dt, AccT &a,
                                                      d3 vel_linear, d3 angvel, double radius_a,
                                                      d3 n, double delta, double wvel)
{
    d3 vel = vadds(vadd(vel_linear, smul(radius_a + delta / 2.0, cross(n, angvel))), wvel);
    double vel_n = dot(vel_linear, n);
    d3 vel_t = vsub(vel, muls(n, dot(n, vel)));
    double vel_t_length = vlen<LM>(vel_t);
    double k_n = P.k_n;
    if (P.E > .001) k_n = 3.141592654 / 2.0 * P.E * radius_a;
    d3 f_n = smul(fmax(0.0, -k_n * delta - P.gamma_wn * vel_n), n);
    double f_n_length = vlen<LM>(f_n);
    a.addEv(P.gamma_wn * vel_n * vel_n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0 && P.gamma_wt > 0.0) {
        d3 f_t_visc = smul(P.gamma_wt, vel_t);
        double f_t_visc_length = vlen<LM>(f_t_visc);
        double f_t_limit;
        if (vel_t_length > 0.0) f_t_limit = P.mu_wd * f_n_length;
        else f_t_limit = P.mu_ws * f_n_length;
        if (f_t_visc_length < f_t_limit) {
            f_t = smul(-1.0, f_t_visc);
        } else {
            f_t = divs(smul(-f_t_limit, vel_t), vel_t_length);
            a.addEs(vlen<LM>(muls(smul(vlen<LM>(f_t), vel_t), dt)) / dt);
        }
    }
    a.addF(vadd(f_n, f_t));
    a.addT(cross(smul(-(radius_a + delta * 0.5), n), f_t));
    a.addP(f_n_length / (4.0 * PI * radius_a * radius_a));
    return dot(f_n, n);
}

// contactmodels.cuh:122-240 contactLinearViscous (contact model 1)
template <int LM, class AccT>
__device__ __forceinline__ void contact_linear_viscous(const SphParams &P, AccT &a, d3 vel_a,
                                                       d3 vel_b, d3 angvel_a, d3 angvel_b,
                                                       double radius_a, double radius_b,
                                                       d3 x_ab, double x_ab_length,
                                                       double delta_ab, double kappa)
{
    d3 n_ab = divs(x_ab, x_ab_length);
    d3 vel_ab_linear = vsub(vel_a, vel_b);
    d3 vel_ab = vadd(vadd(vel_ab_linear, smul(radius_a + delta_ab / 2.0, cross(n_ab, angvel_a))),
                     smul(radius_b + delta_ab / 2.0, cross(n_ab, angvel_b)));
    double vel_n_ab = dot(vel_ab_linear, n_ab);
    d3 vel_t_ab = vsub(vel_ab, muls(n_ab, dot(vel_ab, n_ab)));
    double vel_t_ab_length = vlen<LM>(vel_t_ab);
    double k_n = P.k_n;
    if (P.E > .001) k_n = 3.141592654 / 2.0 * P.E * (radius_a + radius_b) / 2.;
    d3 f_n = smul(fmax(0.0, -k_n * delta_ab - P.gamma_n * vel_n_ab), n_ab);
    if (dot(f_n, n_ab) < 0.0) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen<LM>(f_n);
    d3 f_c = smul(-kappa * fsqrtf_d(radius_a * radius_b), n_ab);
    d3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_ab_length > 0.0) {
        double f_t_visc = P.gamma_t * vel_t_ab_length;
        double f_t_limit;
        if (vel_t_ab_length > (double)0.001f) f_t_limit = P.mu_d * vlen<LM>(vsub(f_n, f_c));
        else f_t_limit = P.mu_s * vlen<LM>(vsub(f_n, f_c));
        if (f_t_visc < f_t_limit) f_t = divs(smul(-f_t_visc, vel_t_ab), vel_t_ab_length);
        else f_t = divs(smul(-f_t_limit, vel_t_ab), vel_t_ab_length);
    }
    a.addF(vadd(vadd(f_n, f_t), f_c));
    a.addT(smul(-(radius_a + delta_ab / 2.0), cross(n_ab, f_t)));
    a.addP(f_n_length / (4.0 * PI * radius_a * radius_a));
}

// contactmodels.cuh:244-411 contactLinear (contact model 2); returns the new
// tangential displacement.  Where the reference leaves it uninitialised
// (both lengths zero) it is zero.
template <int LM, class AccT>
__device__ __forceinline__ d3 contact_linear(const SphParams &P, double dt, AccT &a, d3 vel_a,
                                             d3 vel_b, d3 angvel_a, d3 angvel_b, double radius_a,
                                             double radius_b, d3 x, double x_length,
                                             double delta, d3 delta_t0_uncor)
{
    d3 n = divs(x, x_length);
    d3 vel_linear = vsub(vel_a, vel_b);
    d3 vel = vadd(vadd(vel_linear, smul(radius_a + delta / 2.0, cross(n, angvel_a))),
                  smul(radius_b + delta / 2.0, cross(n, angvel_b)));
    double vel_n = -dot(vel_linear, n);
    d3 vel_t = vsub(vel, muls(n, dot(n, vel)));
    double vel_t_length = vlen<LM>(vel_t);
    d3 delta_t0 = vsub(delta_t0_uncor, muls(n, dot(n, delta_t0_uncor)));
    double delta_t0_length = vlen<LM>(delta_t0);
    d3 delta_t = mk(0.0, 0.0, 0.0);
    double k_n = P.k_n, k_t = P.k_t;
    if (P.E > .001) {
        k_n = 3.141592654 / 2.0 * P.E * (radius_a + radius_b) / 2.;
        k_t = k_n;
    }
    d3 f_n = smul(fmax(0.0, -k_n * delta + P.gamma_n * vel_n), n);
    double f_n_length = vlen<LM>(f_n);
    a.addEv(0.5 * P.gamma_n * vel_n * vel_n);
    d3 f_c = smul(-P.kappa * fsqrtf_d(radius_a * radius_b), n);
    d3 f_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = vadd(delta_t0, muls(vel_t, dt));
        d3 f_t_elast = smul(-k_t, delta_t);
        d3 f_t_visc = smul(-P.gamma_t, vel_t);
        f_t = vadd(f_t_elast, f_t_visc);
        double f_t_length = vlen<LM>(f_t);
        double f_t_limit = P.mu_s * vlen<LM>(vsub(f_n, f_c));
        a.addEv(0.5 * P.gamma_t * vel_t_length * vel_t_length);
        if (f_t_length > f_t_limit) {
            d3 t = divs(f_t, vlen<LM>(f_t));
            f_t = smul(f_t_limit, t);
            delta_t = smul(-1.0 / k_t, vadd(smul(P.mu_d * vlen<LM>(vsub(f_n, f_c)), t),
                                            smul(P.gamma_t, vel_t)));
            a.addEs(0.5 * vlen<LM>(muls(smul(vlen<LM>(f_t), vel_t), dt)) / dt);
        }
    }
    a.addF(vadd(vadd(f_n, f_t), f_c));
    a.addT(cross(smul(-(radius_a + delta * 0.5), n), f_t));
    a.addP(f_n_length / (4.0 * PI * radius_a * radius_a));
    return delta_t;
}

// contactmodels.cuh:417-600 contactHertz (contact model 3).  The reference
// raises the negative overlap to fractional powers (NaN); here
// delta^(3/2) = delta*sqrt(|delta|) and delta^(1/4), delta^(1/2) act on
// |delta|.
template <int LM, class AccT>
__device__ __forceinline__ d3 contact_hertz(const SphParams &P, double dt, AccT &a, d3 vel_a,
                                            d3 vel_b, d3 angvel_a, d3 angvel_b, double radius_a,
                                            double radius_b, d3 x_ab, double x_ab_length,
                                            double delta_ab, d3 delta_t0_uncor)
{
    const double ad = fabs(delta_ab);
    const double d12 = sqrt(ad);
    const double d14 = sqrt(d12);
    const double d32 = delta_ab * d12;
    d3 n_ab = divs(x_ab, x_ab_length);
    d3 vel_ab_linear = vsub(vel_a, vel_b);
    d3 vel_ab = vadd(vadd(vel_ab_linear, smul(radius_a + delta_ab / 2.0, cross(n_ab, angvel_a))),
                     smul(radius_b + delta_ab / 2.0, cross(n_ab, angvel_b)));
    d3 angvel_ab = vsub(angvel_a, angvel_b);
    double angvel_ab_length = vlen<LM>(angvel_ab);
    double vel_n_ab = dot(vel_ab_linear, n_ab);
    d3 vel_t_ab = vsub(vel_ab, muls(n_ab, dot(vel_ab, n_ab)));
    double vel_t_ab_length = vlen<LM>(vel_t_ab);
    d3 delta_t0 = vsub(delta_t0_uncor, muls(n_ab, dot(delta_t0_uncor, n_ab)));
    double delta_t0_length = vlen<LM>(delta_t0);
    d3 delta_t = mk(0.0, 0.0, 0.0);
    double k_n = P.k_n, k_t = P.k_t;
    if (P.E > .001) {
        k_n = 3.141592654 / 2.0 * P.E * (radius_a + radius_b) / 2.;
        k_t = k_n;
    }
    d3 f_n = smul(-k_n * d32 - P.gamma_n * d14 * vel_n_ab, n_ab);
    a.addEv(P.gamma_n * vel_n_ab * vel_n_ab);
    if (dot(f_n, n_ab) < 0.0) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen<LM>(f_n);
    d3 f_c = smul(-P.kappa * fsqrtf_d(radius_a * radius_b), n_ab);
    d3 f_t = mk(0.0, 0.0, 0.0);
    d3 T_res = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_ab_length > 0.0) {
        d3 f_t_elast = smul(-k_t * d12, delta_t0);
        d3 f_t_visc = smul(-P.gamma_t * d14, vel_t_ab);
        double f_t_limit;
        if (vel_t_ab_length > (double)0.001f) f_t_limit = P.mu_d * vlen<LM>(vsub(f_n, f_c));
        else f_t_limit = P.mu_s * vlen<LM>(vsub(f_n, f_c));
        f_t = vadd(f_t_elast, f_t_visc);
        double f_t_length = vlen<LM>(f_t);
        if (f_t_length > f_t_limit) {
            f_t = muls(f_t, f_t_limit / f_t_length);
            delta_t = divs(vadd(f_t, smul(P.gamma_t * d14, vel_t_ab)), -k_t * d12);
            a.addEs(vlen<LM>(vsub(delta_t0, delta_t)) * k_t / dt);
        } else {
            delta_t = vadd(delta_t0, muls(vel_t_ab, dt));
        }
    }
    if (angvel_ab_length > 0.0) {
        T_res = divs(smul(-1.0 * fmin(P.gamma_r * radius_a * angvel_ab_length,
                                      P.mu_r * radius_a * f_n_length),
                          angvel_ab),
                     angvel_ab_length);
    }
    a.addF(vadd(vadd(f_n, f_t), f_c));
    a.addT(vadd(smul(-(radius_a + delta_ab / 2.0), cross(n_ab, f_t)), T_res));
    a.addP(f_n_length / (4.0 * PI * radius_a * radius_a));
    return delta_t;
}

// cohesion.cuh:237-277 capillaryCohesion_exp
__device__ __forceinline__ void capillary_cohesion_exp(const SphParams &P, Acc &a,
                                                       double radius_a, double radius_b,
                                                       double delta_ab, d3 x_ab,
                                                       double x_ab_length, double kappa)
{
    d3 n_ab = divs(x_ab, x_ab_length);
    double r;
    if ((radius_a / radius_b) > (radius_b / radius_a)) r = radius_a / radius_b;
    else r = radius_b / radius_a;
    double h = -fsqrtf_d(r);
    double R_har = (2.0 * radius_a * radius_b) / (radius_a + radius_b);
    double R_geo = fsqrtf_d(radius_a * radius_b);
    double lambda = (double)0.9f * h * fsqrtf_d(P.V_b / R_har);
    d3 f_c = smul(-kappa * R_geo * (double)expf(__double2float_rn(-delta_ab / lambda)), n_ab);
    a.addF(f_c);
}

}  // namespace sph
