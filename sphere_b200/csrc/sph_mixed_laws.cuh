// sph_mixed_laws.cuh -- contact laws of the FP32-mixed step (SPH_PREC_MIXED).
//
// Split of precisions (per contact):
//  - FP64: the centre line x_ab and the overlap delta (FP32 cannot resolve
//    overlaps of ~1e-9 m on ~1 m coordinates), the tangential-displacement
//    history (projection and accumulation), and the per-sphere sums of
//    force, torque and energy rates (Acc);
//  - FP32: everything else of the law -- normal, relative velocities,
//    stiffness and damping terms, Coulomb limit, torque arm.
// Same formulas and branches as the FP64 laws in sph_device.cuh
// (src/contactmodels.cuh:122-600).
#pragma once

#include "sph_device.cuh"

namespace sph {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 fk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 fadd(f3 a, f3 b) { return fk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 fsub(f3 a, f3 b) { return fk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 fmul(float s, f3 a) { return fk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float fdot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 fcross(f3 a, f3 b)
{
    return fk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// FP32 square root and reciprocal of the laws: the GPU's approximate
// special-function instructions (sqrt.approx.ftz.f32, rcp.approx.ftz.f32;
// relative error of a few 2^-23), written as PTX.  Each is one defined
// instruction, so every kernel that inlines the laws gets the same bits
// from it whatever its register budget (a correctly rounded division or an
// approximate one left to the compiler is a sequence the code generator may
// lay out differently per kernel), at one special-function operation each.
__device__ __forceinline__ float fsqrt_a(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float frcp_a(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float flen(f3 v) { return fsqrt_a(fdot(v, v)); }
__device__ __forceinline__ f3 tof(d3 v) { return fk((float)v.x, (float)v.y, (float)v.z); }
__device__ __forceinline__ d3 tod(f3 v) { return mk((double)v.x, (double)v.y, (double)v.z); }
__device__ __forceinline__ f3 xyzf(double4 v) { return fk((float)v.x, (float)v.y, (float)v.z); }

struct MixedPair {
    f3 n;           // unit normal, FP32
    f3 vel_linear;  // vel_a - vel_b, subtracted in FP64
    f3 angvel_a, angvel_b;
    float ra, rb, delta;
};

__device__ __forceinline__ MixedPair mixed_pair(d3 x_ab, double x_length, double delta, d3 vel_a,
                                                d3 vel_b, f3 angvel_a, f3 angvel_b, double ra,
                                                double rb)
{
    MixedPair q;
    const float inv = frcp_a((float)x_length);
    q.n = fmul(inv, tof(x_ab));
    q.vel_linear = tof(vsub(vel_a, vel_b));
    q.angvel_a = angvel_a;
    q.angvel_b = angvel_b;
    q.ra = (float)ra;
    q.rb = (float)rb;
    q.delta = (float)delta;
    return q;
}

__device__ __forceinline__ void mixed_stiffness(const SphParams &P, float ra, float rb, float &k_n,
                                                float &k_t)
{
    k_n = (float)P.k_n;
    k_t = (float)P.k_t;
    if (P.E > .001) {
        k_n = 3.141592654f / 2.0f * (float)P.E * (ra + rb) / 2.f;
        k_t = k_n;
    }
}

// contactLinear (contact model 2), contactmodels.cuh:244-411
template <class AccT>
__device__ __forceinline__ d3 contact_linear_mixed(const SphParams &P, double dt, AccT &a,
                                                   const MixedPair &q, d3 delta_t0_uncor)
{
    const f3 n = q.n;
    const float delta = q.delta;
    const f3 vel = fadd(fadd(q.vel_linear, fmul(q.ra + delta * 0.5f, fcross(n, q.angvel_a))),
                        fmul(q.rb + delta * 0.5f, fcross(n, q.angvel_b)));
    const float vel_n = -fdot(q.vel_linear, n);
    const f3 vel_t = fsub(vel, fmul(fdot(n, vel), n));
    const float vel_t_length = flen(vel_t);
    const d3 nd = tod(n);
    const d3 delta_t0 = vsub(delta_t0_uncor, muls(nd, dot(nd, delta_t0_uncor)));
    // the law reads the length of delta_t0 only as "> 0" (the FP64 law's
    // length(delta_t0) > 0.0): its square says the same without a square root
    const bool delta_t0_nonzero = dot(delta_t0, delta_t0) > 0.0;
    float k_n, k_t;
    mixed_stiffness(P, q.ra, q.rb, k_n, k_t);
    const float gn = (float)P.gamma_n, gt = (float)P.gamma_t;
    const float fnm = fmaxf(0.0f, -k_n * delta + gn * vel_n);
    const f3 f_n = fmul(fnm, n);
    const float f_n_length = fabsf(fnm);
    a.addEv((double)(0.5f * gn * vel_n * vel_n));
    const f3 f_c = fmul(-(float)P.kappa * fsqrt_a(q.ra * q.rb), n);
    f3 f_t = fk(0.f, 0.f, 0.f);
    d3 delta_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_nonzero || vel_t_length > 0.0f) {
        delta_t = vadd(delta_t0, muls(tod(vel_t), dt));
        f_t = fsub(fmul(-k_t, tof(delta_t)), fmul(gt, vel_t));
        const float f_t_length = flen(f_t);
        const float fnc = flen(fsub(f_n, f_c));
        const float f_t_limit = (float)P.mu_s * fnc;
        a.addEv((double)(0.5f * gt * vel_t_length * vel_t_length));
        if (f_t_length > f_t_limit) {
            const f3 t = fmul(frcp_a(f_t_length), f_t);
            f_t = fmul(f_t_limit, t);
            delta_t = tod(fmul(-frcp_a(k_t), fadd(fmul((float)P.mu_d * fnc, t), fmul(gt, vel_t))));
            a.addEs((double)(0.5f * flen(fmul((float)dt * f_t_limit, vel_t)) * frcp_a((float)dt)));
        }
    }
    a.addF(tod(fadd(fadd(f_n, f_t), f_c)));
    a.addT(tod(fcross(fmul(-(q.ra + delta * 0.5f), n), f_t)));
    a.addP((double)(f_n_length * frcp_a(4.0f * 3.14159265358979f * q.ra * q.ra)));
    return delta_t;
}

// contactHertz (contact model 3) with the overlap-magnitude powers of the
// FP64 form, contactmodels.cuh:417-600
template <class AccT>
__device__ __forceinline__ d3 contact_hertz_mixed(const SphParams &P, double dt, AccT &a,
                                                  const MixedPair &q, d3 delta_t0_uncor)
{
    const f3 n = q.n;
    const float delta = q.delta;
    const float d12 = fsqrt_a(fabsf(delta)), d14 = fsqrt_a(d12), d32 = delta * d12;
    const f3 vel_ab = fadd(fadd(q.vel_linear, fmul(q.ra + delta * 0.5f, fcross(n, q.angvel_a))),
                           fmul(q.rb + delta * 0.5f, fcross(n, q.angvel_b)));
    const f3 angvel_ab = fsub(q.angvel_a, q.angvel_b);
    const float angvel_ab_length = flen(angvel_ab);
    const float vel_n_ab = fdot(q.vel_linear, n);
    const f3 vel_t_ab = fsub(vel_ab, fmul(fdot(vel_ab, n), n));
    const float vel_t_ab_length = flen(vel_t_ab);
    const d3 nd = tod(n);
    const d3 delta_t0 = vsub(delta_t0_uncor, muls(nd, dot(delta_t0_uncor, nd)));
    const bool delta_t0_nonzero = dot(delta_t0, delta_t0) > 0.0;   // length > 0
    float k_n, k_t;
    mixed_stiffness(P, q.ra, q.rb, k_n, k_t);
    const float gn = (float)P.gamma_n, gt = (float)P.gamma_t;
    f3 f_n = fmul(-k_n * d32 - gn * d14 * vel_n_ab, n);
    a.addEv((double)(gn * vel_n_ab * vel_n_ab));
    if (fdot(f_n, n) < 0.0f) f_n = fk(0.f, 0.f, 0.f);
    const float f_n_length = flen(f_n);
    const f3 f_c = fmul(-(float)P.kappa * fsqrt_a(q.ra * q.rb), n);
    f3 f_t = fk(0.f, 0.f, 0.f);
    f3 T_res = fk(0.f, 0.f, 0.f);
    d3 delta_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_nonzero || vel_t_ab_length > 0.0f) {
        const f3 f_t_elast = fmul(-k_t * d12, tof(delta_t0));
        const f3 f_t_visc = fmul(-gt * d14, vel_t_ab);
        const float fnc = flen(fsub(f_n, f_c));
        const float f_t_limit = vel_t_ab_length > 0.001f ? (float)P.mu_d * fnc : (float)P.mu_s * fnc;
        f_t = fadd(f_t_elast, f_t_visc);
        const float f_t_length = flen(f_t);
        if (f_t_length > f_t_limit) {
            f_t = fmul(f_t_limit * frcp_a(f_t_length), f_t);
            delta_t = tod(fmul(frcp_a(-k_t * d12), fadd(f_t, fmul(gt * d14, vel_t_ab))));
            a.addEs(sqrt(dot(vsub(delta_t0, delta_t), vsub(delta_t0, delta_t))) * (double)k_t / dt);
        } else {
            delta_t = vadd(delta_t0, muls(tod(vel_t_ab), dt));
        }
    }
    if (angvel_ab_length > 0.0f)
        T_res = fmul(-fminf((float)P.gamma_r * q.ra * angvel_ab_length,
                            (float)P.mu_r * q.ra * f_n_length) * frcp_a(angvel_ab_length),
                     angvel_ab);
    a.addF(tod(fadd(fadd(f_n, f_t), f_c)));
    a.addT(tod(fadd(fmul(-(q.ra + delta * 0.5f), fcross(n, f_t)), T_res)));
    a.addP((double)(f_n_length * frcp_a(4.0f * 3.14159265358979f * q.ra * q.ra)));
    return delta_t;
}

// contactLinearViscous (contact model 1), contactmodels.cuh:122-240
template <class AccT>
__device__ __forceinline__ void contact_linear_viscous_mixed(const SphParams &P, AccT &a,
                                                             const MixedPair &q, float kappa)
{
    const f3 n = q.n;
    const float delta = q.delta;
    const f3 vel_ab = fadd(fadd(q.vel_linear, fmul(q.ra + delta * 0.5f, fcross(n, q.angvel_a))),
                           fmul(q.rb + delta * 0.5f, fcross(n, q.angvel_b)));
    const float vel_n_ab = fdot(q.vel_linear, n);
    const f3 vel_t_ab = fsub(vel_ab, fmul(fdot(vel_ab, n), n));
    const float vel_t_ab_length = flen(vel_t_ab);
    float k_n, k_t;
    mixed_stiffness(P, q.ra, q.rb, k_n, k_t);
    f3 f_n = fmul(fmaxf(0.0f, -k_n * delta - (float)P.gamma_n * vel_n_ab), n);
    if (fdot(f_n, n) < 0.0f) f_n = fk(0.f, 0.f, 0.f);
    const float f_n_length = flen(f_n);
    const f3 f_c = fmul(-kappa * fsqrt_a(q.ra * q.rb), n);
    f3 f_t = fk(0.f, 0.f, 0.f);
    if (vel_t_ab_length > 0.0f) {
        const float f_t_visc = (float)P.gamma_t * vel_t_ab_length;
        const float fnc = flen(fsub(f_n, f_c));
        const float f_t_limit = vel_t_ab_length > 0.001f ? (float)P.mu_d * fnc : (float)P.mu_s * fnc;
        const float mag = f_t_visc < f_t_limit ? f_t_visc : f_t_limit;
        f_t = fmul(-mag * frcp_a(vel_t_ab_length), vel_t_ab);
    }
    a.addF(tod(fadd(fadd(f_n, f_t), f_c)));
    a.addT(tod(fmul(-(q.ra + delta * 0.5f), fcross(n, f_t))));
    a.addP((double)(f_n_length * frcp_a(4.0f * 3.14159265358979f * q.ra * q.ra)));
}

}  // namespace sph
