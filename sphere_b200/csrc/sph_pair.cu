// sph_pair.cu -- the list step of the FP32-mixed form (launch variant 4).
//
// The FP64 form reproduces the reference's NC-slot contact rows
// (contactsearch.cuh:194-322): a new contact takes a free slot in the order
// the 27-cell search meets it, and each sphere's sums run in slot order,
// which is what makes its forces equal the reference's bit for bit.  The
// FP32-mixed form is held to a stated error instead (per-step force
// relative L2 <= 1e-5 against the FP64 form), so it keeps the contact
// history where the neighbour list already has a place for it:
//
//  * contact set: the same exact FP64 overlap test on the same centre line
//    as the FP64 form ((xa - xb) + image shift, FP64 length as the length
//    mode says, no contraction), over every entry of the sphere's
//    neighbour list (all spheres within ra + rb + skin at the list build),
//    so the touching pairs are the FP64 form's;
//  * history: the tangential displacement of a touching pair is kept with
//    its list entry (three FP64), with a bit per entry that says whether the
//    pair touched at the last step; a rebuild of the lists carries every
//    history over to the entry of the same partner in the new list;
//  * order: a sphere's contacts are summed in list order (ascending
//    partner index) instead of slot order;
//  * one kernel per step does the contact laws, the walls, the sums and the
//    integration (k_pair_step): partners are read from the state of the
//    step's start and the new state is written to the other half of a
//    ping-pong pair, so no second pass is needed; the wall stage sums the
//    wall force in fixed-order chunks (deterministic, FP64) and advances
//    the walls and time (k_pair_chunks, k_pair_box);
//  * storage: FP64 where the precision contract keeps FP64 (positions,
//    velocities, the history, xyzsum, es/ev, the wall force), FP32 for the
//    rest (angular velocity, angpos, acc, angacc, force, torque, energy
//    rates) -- the per-sphere bytes of the mixed budget.
//
// The lists are rebuilt inside the step graph only when a sphere has moved
// more than half the skin since the last build: a conditional graph node
// whose body is the cell sort, the list build and the history carry-over
// (launch_step_pair), set by k_pair_cond from the flag the integration
// raises.  Every launch shape gives the same bits: the code generator may
// fuse a multiply and an add, or lay out an approximate division,
// differently in one shape than in another (it decides under each shape's
// register budget), so the file is compiled without FMA contraction, the
// contact laws' FP32 square roots and reciprocals are single approximate
// instructions written as PTX (sph_mixed_laws.cuh), and any other FP32
// division or square root is correctly rounded.  The overlap test is
// written with explicitly rounded operations so that it matches the FP64
// form.
#include <cstdint>
#include <cstdio>

#include "sph_device.cuh"
#include "sph_internal.h"
#include "sph_mixed_laws.cuh"
#include "sph_step.cuh"
#include "sph_sync.cuh"

namespace sph {

namespace {

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }


// The centre line a - b of a touching pair under the image the cell search
// uses (the nearest one: along a periodic axis a difference over half the
// box is shifted by -+L), rounded as the FP64 form's (xa - xb) + shift;
// code: the image code of a slot word (shift_code).
__device__ __forceinline__ d3 centre_line(const DevBox &B, const double4 &xa, const double4 &xb,
                                          uint32_t *code)
{
    double dx = __dsub_rn(xa.x, xb.x), dy = __dsub_rn(xa.y, xb.y);
    const double dz = __dsub_rn(xa.z, xb.z);
    int sx = 0, sy = 0;
    if (B.periodic == 1 || B.periodic == 2) {
        if (dx > 0.5 * B.L[0]) { dx = __dadd_rn(dx, -B.L[0]); sx = -1; }
        else if (dx < -0.5 * B.L[0]) { dx = __dadd_rn(dx, B.L[0]); sx = 1; }
    }
    if (B.periodic == 1) {
        if (dy > 0.5 * B.L[1]) { dy = __dadd_rn(dy, -B.L[1]); sy = -1; }
        else if (dy < -0.5 * B.L[1]) { dy = __dadd_rn(dy, B.L[1]); sy = 1; }
    }
    if (code) *code = shift_code(sx, sy);
    return mk(dx, dy, dz);
}

// vlen<LM> with the dot product rounded operation by operation.
template <int LM>
__device__ __forceinline__ double len_rn(d3 v)
{
    const double d = __dadd_rn(__dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y)),
                               __dmul_rn(v.z, v.z));
    if (LM == SPH_LEN_FP64) return __dsqrt_rn(d);
    return (double)__fsqrt_rn(__double2float_rn(d));
}

// Sphere i's list and history in their entry-major layout (PairArgs):
// entry k's id at ids[k * nrow], history component c at
// hist[(3 k + c) * nrow], from the sphere's own column.
struct ListRow {
    const uint32_t *ids;
    double *hist;
    size_t nrow;
    __device__ __forceinline__ ListRow(const PairArgs &P, uint32_t sel, uint32_t i)
        : ids(P.ids[sel] + i), hist(P.hist[sel] + i), nrow(P.nrow)
    {
    }
    __device__ __forceinline__ uint32_t id(uint32_t k) const { return ids[(size_t)k * nrow]; }
    __device__ __forceinline__ double *h(uint32_t k, int c) const
    {
        return hist + (size_t)(3u * k + (uint32_t)c) * nrow;
    }
    __device__ __forceinline__ d3 hist3(uint32_t k) const { return mk(*h(k, 0), *h(k, 1), *h(k, 2)); }
    __device__ __forceinline__ void put3(uint32_t k, d3 v) const
    {
        *h(k, 0) = v.x;
        *h(k, 1) = v.y;
        *h(k, 2) = v.z;
    }
};

// A sphere's sums in the list step: force and torque in FP64 (they drive
// the FP64 integration, where the contacts' forces largely cancel), the
// energy rates and pressure in FP32 (stored in FP32; es and ev accumulate
// them in FP64).
struct MixedAcc {
    d3 F, T;
    float es_dot, ev_dot, p;
    __device__ __forceinline__ void addF(d3 v) { F = vadd(F, v); }
    __device__ __forceinline__ void addT(d3 v) { T = vadd(T, v); }
    __device__ __forceinline__ void addEs(double v) { es_dot += (float)v; }
    __device__ __forceinline__ void addEv(double v) { ev_dot += (float)v; }
    __device__ __forceinline__ void addP(double v) { p += (float)v; }
};

__device__ __forceinline__ MixedPair mixed_pair_f(d3 x_ab, double x_length, double delta, float4 va,
                                                  float4 vb, float4 wa, float4 wb, double ra,
                                                  double rb)
{
    MixedPair q;
    const float inv = frcp_a((float)x_length);
    q.n = fmul(inv, tof(x_ab));
    q.vel_linear = fk(va.x - vb.x, va.y - vb.y, va.z - vb.z);
    q.angvel_a = fk(wa.x, wa.y, wa.z);
    q.angvel_b = fk(wb.x, wb.y, wb.z);
    q.ra = (float)ra;
    q.rb = (float)rb;
    q.delta = (float)delta;
    return q;
}

// The plane walls of contactsearch.cuh:428-465 and :602-701 for one sphere
// of the list step: wall w is the box's wall w when w < nw, else the
// default plane (top at L[2], sides at 0 and L); the normal force on wall 0
// is returned.  Reads each wall from the box table where it is used.
template <int LM>
__device__ __forceinline__ double walls_pair(const DevBox &B, double4 xa, d3 vel_a, d3 angvel_a,
                                             MixedAcc &acc)
{
    const SphParams &Pm = B.P;
    const double dt = B.dt, r = xa.w;
    const uint32_t nw = B.nw;
    auto plane = [&](uint32_t w, double dx, double dy, double dz, double dpos, d3 &n, double &pos,
                     double &vel) {
        if (w < nw) {
            n = mk(B.wnx[w][0], B.wnx[w][1], B.wnx[w][2]);
            pos = B.wnx[w][3];
            vel = B.wmvfd[w][1];
        } else {
            n = mk(dx, dy, dz);
            pos = dpos;
            vel = 0.0;
        }
    };
    d3 n;
    double pos, wv, w0_force = 0.0;
    plane(0, 0.0, 0.0, -1.0, B.L[2], n, pos, wv);
    double delta_w = pos - (xa.z + r);
    if (delta_w < 0.0) w0_force = contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, n, delta_w, wv);
    delta_w = xa.z - r - B.origo[2];
    if (delta_w < 0.0)
        (void)contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, mk(0.0, 0.0, 1.0), delta_w, 0.0);
    if (B.periodic == 0) {
        plane(1, -1.0, 0.0, 0.0, B.L[0], n, pos, wv);
        delta_w = pos - (xa.x + r);
        if (delta_w < 0.0) (void)contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, n, delta_w, wv);
        plane(2, 1.0, 0.0, 0.0, 0.0, n, pos, wv);
        delta_w = xa.x - r - pos;
        if (delta_w < 0.0) (void)contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, n, delta_w, wv);
    }
    if (B.periodic == 0 || B.periodic == 2) {
        plane(3, 0.0, -1.0, 0.0, B.L[1], n, pos, wv);
        delta_w = pos - (xa.y + r);
        if (delta_w < 0.0) (void)contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, n, delta_w, wv);
        plane(4, 0.0, 1.0, 0.0, 0.0, n, pos, wv);
        delta_w = xa.y - r - pos;
        if (delta_w < 0.0) (void)contact_linear_wall<LM>(Pm, dt, acc, vel_a, angvel_a, r, n, delta_w, wv);
    }
    return w0_force;
}

// integration.cuh:14-305 (TY3) for one sphere of the list step: FP64
// arithmetic on the compact state; the new state goes to the [nxt] half of
// the ping-pong arrays and to the sphere's own arrays.
__device__ __forceinline__ void integrate_pair(const StepArgs &A, const PairArgs &P,
                                               const DevBox &B, uint32_t i, uint32_t nxt,
                                               double4 x, double4 vel, float4 wf, d3 F, d3 T)
{
    const SphParams &Pm = B.P;
    const double dt = B.dt;
    const float4 apf = P.angpos[i];
    double4 xyzsum = P.xyzsum[i];
    double a0[3] = {0.0, 0.0, 0.0}, w0[3] = {0.0, 0.0, 0.0};
    if (B.iter != 0) {
        const float4 q = P.acc[i], r = P.angacc[i];
        a0[0] = q.x; a0[1] = q.y; a0[2] = q.z;
        w0[0] = r.x; w0[1] = r.y; w0[2] = r.z;
    }
    const double radius = x.w;
    const double m = 4.0 / 3.0 * PI * radius * radius * radius * Pm.rho;
    // reciprocals once (FP64 divisions are long instruction sequences)
    const double inv_m = 1.0 / m, inv_dt = 1.0 / dt;
    const double inv_i = inv_m * (5.0 / 2.0) / (radius * radius);
    double acc[3], angacc[3];
    acc[0] = F.x * inv_m + Pm.g[0];
    acc[1] = F.y * inv_m + Pm.g[1];
    acc[2] = F.z * inv_m + Pm.g[2];
    angacc[0] = T.x * inv_i;
    angacc[1] = T.y * inv_i;
    angacc[2] = T.z * inv_i;
    if (vel.w > 0.0001 && vel.w < 10.0) {
        acc[0] = 0.0;
        acc[1] = 0.0;
        acc[2] -= Pm.g[2];
        angacc[0] = angacc[1] = angacc[2] = 0.0;
    }
    if (vel.w >= 10.0) {
        acc[1] = 0.0;
        angacc[0] = 0.0;
        angacc[2] = 0.0;
    }
    if (vel.w < -0.0001) {
        acc[0] = acc[1] = acc[2] = 0.0;
        angacc[0] = angacc[1] = angacc[2] = 0.0;
    }
    const double xv[3] = {x.x, x.y, x.z};
    const double vv[3] = {vel.x, vel.y, vel.z};
    const double pv[3] = {apf.x, apf.y, apf.z};
    const double wv[3] = {wf.x, wf.y, wf.z};
    double sv[3] = {xyzsum.x, xyzsum.y, xyzsum.z};
    double xn[3], vn[3], pn[3], wn[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double dacc = (acc[d] - a0[d]) * inv_dt;
        const double dangacc = (angacc[d] - w0[d]) * inv_dt;
        const double dx = vv[d] * dt + 0.5 * acc[d] * dt * dt + 1.0 / 6.0 * dacc * dt * dt * dt;
        xn[d] = xv[d] + dx;
        vn[d] = vv[d] + acc[d] * dt + 0.5 * dacc * dt * dt;
        pn[d] = pv[d] + wv[d] * dt + 0.5 * angacc[d] * dt * dt + 1.0 / 6.0 * dangacc * dt * dt * dt;
        wn[d] = wv[d] + angacc[d] * dt + 0.5 * dangacc * dt * dt;
        sv[d] += dx;
    }
    if (B.periodic == 1) {
        if (xn[0] < B.origo[0]) xn[0] += B.L[0];
        if (xn[0] > B.L[0]) xn[0] -= B.L[0];
        if (xn[1] < B.origo[1]) xn[1] += B.L[1];
        if (xn[1] > B.L[1]) xn[1] -= B.L[1];
    } else if (B.periodic == 2) {
        if (xn[0] < B.origo[0]) xn[0] += B.L[0];
        if (xn[0] > B.L[0]) xn[0] -= B.L[0];
    }
    {
        // neighbour-list validity: displacement since the list build
        // (nearest periodic image), FP32
        const float4 r = A.xref[i];
        float ex = (float)xn[0] - r.x, ey = (float)xn[1] - r.y;
        const float ez = (float)xn[2] - r.z;
        if (B.periodic == 1 || B.periodic == 2) {
            const float lx = (float)B.L[0];
            if (ex > 0.5f * lx) ex -= lx;
            else if (ex < -0.5f * lx) ex += lx;
        }
        if (B.periodic == 1) {
            const float ly = (float)B.L[1];
            if (ey > 0.5f * ly) ey -= ly;
            else if (ey < -0.5f * ly) ey += ly;
        }
        if (!(ex * ex + ey * ey + ez * ez <= B.vdisp2)) A.vflag[0] = 1u;
    }
    if (vel.w > 5.0 && vel.w < 10.0) {
        if (B.change_velocity_state == 1) vn[0] *= 10.0;
        else if (B.change_velocity_state == -1) vn[0] /= 10.0;
    }
    P.xyzsum[i] = make_double4(sv[0], sv[1], sv[2], 0.0);
    P.acc[i] = make_float4((float)acc[0], (float)acc[1], (float)acc[2], 0.f);
    P.angacc[i] = make_float4((float)angacc[0], (float)angacc[1], (float)angacc[2], 0.f);
    P.angpos[i] = make_float4((float)pn[0], (float)pn[1], (float)pn[2], apf.w);
    P.vel[i] = make_double4(vn[0], vn[1], vn[2], vel.w);
    P.xr[nxt][i] = make_double4(xn[0], xn[1], xn[2], x.w);
    P.vw[nxt][2 * i] = make_float4((float)vn[0], (float)vn[1], (float)vn[2], 0.f);
    P.vw[nxt][2 * i + 1] = make_float4((float)wn[0], (float)wn[1], (float)wn[2], 0.f);
}

// After a sphere's contacts: its touching bits, walls, sums and integration.
template <int LM>
__device__ __forceinline__ void finish_sphere(const StepArgs &A, const PairArgs &P,
                                              const DevBox &B, uint32_t i, uint32_t nxt,
                                              uint32_t ls, double4 xa, float4 wa, MixedAcc &acc,
                                              unsigned long long live_old,
                                              unsigned long long live_new)
{
    const double dt = B.dt;
    if (__popcll(live_new) > NC) raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
    if (live_new != live_old) P.live[ls][i] = live_new;
    const double4 vel = P.vel[i];
    const double w0_force = walls_pair<LM>(B, xa, xyz(vel), mk(wa.x, wa.y, wa.z), acc);
    P.force[i] = make_float4((float)acc.F.x, (float)acc.F.y, (float)acc.F.z, 0.f);
    P.torque[i] = make_float4((float)acc.T.x, (float)acc.T.y, (float)acc.T.z, 0.f);
    P.epp[i] = make_float4(acc.es_dot, acc.ev_dot, acc.p, 0.f);
    const double2 e0 = P.eacc[i];
    P.eacc[i] = make_double2(e0.x + (double)acc.es_dot * dt, e0.y + (double)acc.ev_dot * dt);
    if (B.nw > 0) A.wf_pp[i] = w0_force;
    integrate_pair(A, P, B, i, nxt, xa, vel, wa, acc.F, acc.T);
}

// One sphere of the list step (thread slot t of the ordering): its list
// entries in order, each tested with the exact FP64 overlap test and, for a
// touching pair, the contact law with the entry's history; then walls, sums
// and the integration of the sphere.  AHEAD: the loads of the next entry --
// partner state and, when its pair touched, its history -- are issued before
// the current entry is computed (more loads in flight per thread, about 20
// more registers); without it each entry is loaded at its turn and the
// latency is hidden by more resident warps.  Both give the same bits.
template <int LM, bool AHEAD = true>
__device__ __forceinline__ void pair_sphere(const StepArgs &A, const PairArgs &P, uint32_t t,
                                            uint32_t cur, uint32_t nxt, uint32_t ls)
{
    const uint32_t i = P.order[ls][t];
    const double4 *__restrict__ xr = P.xr[cur];
    const float4 *__restrict__ vw = P.vw[cur];
    const DevBox &B = A.boxes[box_index(A, i)];
    uint32_t n = P.cnt[ls][i];
    if (n > (uint32_t)VL_MAX) {   // the list overflowed at its build
        raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
        n = 0;
    }
    const unsigned long long live_old = P.live[ls][i];
    unsigned long long live_new = 0ull;
    const ListRow L(P, ls, i);
    const double4 xa = xr[i];
    const float4 va = vw[2 * i], wa = vw[2 * i + 1];
    const double dt = B.dt;

    MixedAcc acc;
    acc.F = mk(0.0, 0.0, 0.0);
    acc.T = mk(0.0, 0.0, 0.0);
    acc.es_dot = 0.f;
    acc.ev_dot = 0.f;
    acc.p = 0.f;
    if (!AHEAD) {
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t b = L.id(k);
            const double4 xb = xr[b];
            const float4 vb = vw[2 * b], wb = vw[2 * b + 1];
            d3 hb = mk(0.0, 0.0, 0.0);
            if ((live_old >> k) & 1ull) hb = L.hist3(k);
            const d3 x_ab = centre_line(B, xa, xb, nullptr);
            const double x_ab_length = len_rn<LM>(x_ab);
            const double delta_n = __dsub_rn(x_ab_length, __dadd_rn(xa.w, xb.w));
            if (delta_n < 0.0) {
                const MixedPair q = mixed_pair_f(x_ab, x_ab_length, delta_n, va, vb, wa, wb, xa.w, xb.w);
                const d3 nd = B.P.contactmodel == 2 ? contact_linear_mixed(B.P, dt, acc, q, hb)
                                                    : contact_hertz_mixed(B.P, dt, acc, q, hb);
                L.put3(k, nd);
                live_new |= 1ull << k;
            }
        }
        finish_sphere<LM>(A, P, B, i, nxt, ls, xa, wa, acc, live_old, live_new);
        return;
    }
    // entry k's partner state and history are loaded during entry k - 1,
    // entry k's partner id during entry k - 2 (the row holds VL_MAX >= 2
    // ids; those at or past n are not used)
    double4 xb = make_double4(0.0, 0.0, 0.0, 0.0);
    float4 vb = make_float4(0.f, 0.f, 0.f, 0.f), wb = vb;
    d3 hb = mk(0.0, 0.0, 0.0);
    uint32_t b_next = L.id(1);
    if (n) {
        const uint32_t b = L.id(0);
        xb = xr[b];
        vb = vw[2 * b];
        wb = vw[2 * b + 1];
        if (live_old & 1ull) hb = L.hist3(0);
    }
    for (uint32_t k = 0; k < n; ++k) {
        double4 xq = xb;
        float4 vq = vb, wq = wb;
        d3 hq = mk(0.0, 0.0, 0.0);
        if (k + 1 < n) {
            const uint32_t b = b_next;
            if (k + 2 < n) b_next = L.id(k + 2);
            xq = xr[b];
            vq = vw[2 * b];
            wq = vw[2 * b + 1];
            if ((live_old >> (k + 1)) & 1ull)
                hq = L.hist3(k + 1);
        }
        const d3 x_ab = centre_line(B, xa, xb, nullptr);
        const double x_ab_length = len_rn<LM>(x_ab);
        const double delta_n = __dsub_rn(x_ab_length, __dadd_rn(xa.w, xb.w));
        if (delta_n < 0.0) {
            const MixedPair q = mixed_pair_f(x_ab, x_ab_length, delta_n, va, vb, wa, wb, xa.w, xb.w);
            const d3 nd = B.P.contactmodel == 2 ? contact_linear_mixed(B.P, dt, acc, q, hb)
                                                : contact_hertz_mixed(B.P, dt, acc, q, hb);
            L.put3(k, nd);
            live_new |= 1ull << k;
        }
        xb = xq;
        vb = vq;
        wb = wq;
        hb = hq;
    }
    finish_sphere<LM>(A, P, B, i, nxt, ls, xa, wa, acc, live_old, live_new);
}

template <int LM, int NT, int MINB, bool AHEAD = true>
__global__ void __launch_bounds__(NT, MINB) k_pair_step(StepArgs A, PairArgs P)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.ntot) return;
    const uint32_t cur = *P.pp;
    pair_sphere<LM, AHEAD>(A, P, t, cur, cur ^ 1u, *P.lsel);
}

// cp.async (global -> shared, issued per thread, completion per thread by
// commit groups): the staging of partner data below.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Partner data of D list entries per thread in flight, staged in shared
// memory (field-major: slot, field, thread, so that a warp's accesses to
// one field are consecutive): position+radius, velocity, angular velocity
// and the entry's history.
template <int NT, int D>
struct PairStage {
    double4 x[D][NT];
    float4 v[D][NT];
    float4 w[D][NT];
    double h[D][3][NT];
};

// The list step with the partner data of entry k + D copied into shared
// memory (cp.async) while entry k is computed: D entries' loads in flight
// per thread without holding them in registers.  The same arithmetic as
// k_pair_step.
template <int LM, int NT, int MINB, int D>
__global__ void __launch_bounds__(NT, MINB) k_pair_step_async(StepArgs A, PairArgs P)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    PairStage<NT, D> &S = *reinterpret_cast<PairStage<NT, D> *>(s_raw);
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const int tx = (int)threadIdx.x;
    if (t >= A.ntot) return;
    const uint32_t cur = *P.pp, nxt = cur ^ 1u, ls = *P.lsel;
    const uint32_t i = P.order[ls][t];
    const double4 *__restrict__ xr = P.xr[cur];
    const float4 *__restrict__ vw = P.vw[cur];
    const DevBox &B = A.boxes[box_index(A, i)];
    uint32_t n = P.cnt[ls][i];
    if (n > (uint32_t)VL_MAX) {   // the list overflowed at its build
        raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
        n = 0;
    }
    const unsigned long long live_old = P.live[ls][i];
    unsigned long long live_new = 0ull;
    const ListRow L(P, ls, i);
    auto stage = [&](uint32_t k) {
        // entry k into slot k % D (an empty commit group past the list's end)
        if (k < n) {
            const int q = (int)(k % D);
            const uint32_t b = L.id(k);
            const double4 *gx = xr + b;
            cp_async16(&S.x[q][tx], gx);
            cp_async16(reinterpret_cast<char *>(&S.x[q][tx]) + 16, reinterpret_cast<const char *>(gx) + 16);
            cp_async16(&S.v[q][tx], vw + 2 * b);
            cp_async16(&S.w[q][tx], vw + 2 * b + 1);
            if ((live_old >> k) & 1ull) {
                cp_async8(&S.h[q][0][tx], L.h(k, 0));
                cp_async8(&S.h[q][1][tx], L.h(k, 1));
                cp_async8(&S.h[q][2][tx], L.h(k, 2));
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < D; ++k) stage((uint32_t)k);
    const double4 xa = xr[i];
    const float4 va = vw[2 * i], wa = vw[2 * i + 1];
    const double dt = B.dt;

    MixedAcc acc;
    acc.F = mk(0.0, 0.0, 0.0);
    acc.T = mk(0.0, 0.0, 0.0);
    acc.es_dot = 0.f;
    acc.ev_dot = 0.f;
    acc.p = 0.f;
    for (uint32_t k = 0; k < n; ++k) {
        cp_async_wait<D - 1>();
        const int q = (int)(k % D);
        const double4 xb = S.x[q][tx];
        const float4 vb = S.v[q][tx], wb = S.w[q][tx];
        d3 hb = mk(0.0, 0.0, 0.0);
        if ((live_old >> k) & 1ull) hb = mk(S.h[q][0][tx], S.h[q][1][tx], S.h[q][2][tx]);
        const d3 x_ab = centre_line(B, xa, xb, nullptr);
        const double x_ab_length = len_rn<LM>(x_ab);
        const double delta_n = __dsub_rn(x_ab_length, __dadd_rn(xa.w, xb.w));
        if (delta_n < 0.0) {
            const MixedPair mp = mixed_pair_f(x_ab, x_ab_length, delta_n, va, vb, wa, wb, xa.w, xb.w);
            const d3 nd = B.P.contactmodel == 2 ? contact_linear_mixed(B.P, dt, acc, mp, hb)
                                                : contact_hertz_mixed(B.P, dt, acc, mp, hb);
            L.put3(k, nd);
            live_new |= 1ull << k;
        }
        // slot k % D is refilled only after its values were used (the copy
        // cannot overtake the reads)
        stage(k + D);
    }
    cp_async_wait<0>();
    finish_sphere<LM>(A, P, B, i, nxt, ls, xa, wa, acc, live_old, live_new);
}

// Wall-force sum of one chunk of 2^chunk_log2 spheres of one box, and the
// sum of a box's chunks: FP64 sums in a fixed order, the same whatever the
// block that runs them (the chunk and box kernels, or the persistent
// kernel with its own block size).
constexpr int CHUNK_THREADS = 256;
constexpr int PBOX_THREADS = 128;

// The sum of get(0), ..., get(n - 1) in a fixed order for a given V: term k
// goes to virtual lane k mod V, each lane adds its terms in index order,
// each group of 32 lanes is reduced by the xor-shuffle tree, and the V / 32
// group sums are added in order.  The block's threads (blockDim.x, a
// multiple of 32 dividing V, at least V / 4) play lanes t, t + blockDim.x,
// ...: thread t of warp w holds lane t + j blockDim.x, whose group is
// w + j blockDim.x / 32, with the same lane in it.  Thread 0 returns the
// sum (the others 0).
template <int V, class G>
__device__ __forceinline__ double ordered_sum(uint32_t n, G get, double *s_w)
{
    constexpr int RMAX = 4;
    const uint32_t nt = blockDim.x, r = V / nt;
    double acc[RMAX];
#pragma unroll
    for (int j = 0; j < RMAX; ++j) {
        double s = 0.0;
        if ((uint32_t)j < r)
            for (uint32_t k = threadIdx.x + (uint32_t)j * nt; k < n; k += V) s += get(k);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        acc[j] = s;
    }
    __syncthreads();
    if ((threadIdx.x & 31u) == 0) {
#pragma unroll
        for (int j = 0; j < RMAX; ++j)
            if ((uint32_t)j < r) s_w[(threadIdx.x >> 5) + (uint32_t)j * (nt >> 5)] = acc[j];
    }
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < V / 32; ++w) t += s_w[w];
    return t;
}

// The wall-force sum of chunk c by the calling block.
__device__ __forceinline__ void chunk_sum(const StepArgs &A, const PairArgs &P, uint32_t c,
                                          double *s_w)
{
    const uint32_t bx = P.chunk_box[c];
    const DevBox &B = A.boxes[bx];
    const uint32_t start = (c - P.box_chunk0[bx]) << P.chunk_log2;
    const uint32_t end = min(B.np, start + (1u << P.chunk_log2));
    const double *wf = A.wf_pp + B.p_base + start;
    const double t = ordered_sum<CHUNK_THREADS>(B.nw > 0 ? end - start : 0u,
                                                [&](uint32_t k) { return wf[k]; }, s_w);
    if (threadIdx.x == 0) P.chunk_part[c] = t;
}

// Box bx by the calling block: its chunks' sums in a fixed order (FP64),
// then integrateWalls and the time bookkeeping (advance_box).
__device__ __forceinline__ void box_sum_advance(const StepArgs &A, const PairArgs &P, uint32_t bx,
                                                double *s_w)
{
    DevBox &B = A.boxes[bx];
    bool any = false;
    for (uint32_t w = 0; w < B.nw; ++w) any = any || B.wmode[w] != 0;
    uint32_t nch = 0;
    if (B.np > 0 && any) nch = (B.np + (1u << P.chunk_log2) - 1) >> P.chunk_log2;
    const double *part = P.chunk_part + P.box_chunk0[bx];
    const double fsum = ordered_sum<PBOX_THREADS>(nch, [&](uint32_t k) { return part[k]; }, s_w);
    if (threadIdx.x == 0) advance_box(B, fsum);
}

__global__ void __launch_bounds__(CHUNK_THREADS) k_pair_chunks(StepArgs A, PairArgs P)
{
    grid_dependency_wait();
    __shared__ double s_w[32];
    chunk_sum(A, P, blockIdx.x, s_w);
}

// Per box: the chunks' sums, integrateWalls, time; block 0 then hands the
// ping-pong state to the next step.

__global__ void __launch_bounds__(PBOX_THREADS) k_pair_box(StepArgs A, PairArgs P)
{
    grid_dependency_wait();
    __shared__ double s_w[32];
    box_sum_advance(A, P, blockIdx.x, s_w);
    if (blockIdx.x == 0 && threadIdx.x == 0) *P.pp ^= 1u;
}

// The list step as one persistent, cooperative launch: the blocks take the
// spheres in turn (slots t = block + k * grid), then, after a grid barrier,
// the chunks' wall-force sums, and after another the boxes (walls, time)
// and the hand-over of the ping-pong state.  The same arithmetic and order
// of sums as k_pair_step + k_pair_chunks + k_pair_box.
template <int LM, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_pair_persist(StepArgs A, PairArgs P, GridSync G)
{
    __shared__ double s_w[32];
    const uint32_t cur = *P.pp, nxt = cur ^ 1u, ls = *P.lsel;
    for (uint32_t base = blockIdx.x * NT; base < A.ntot; base += gridDim.x * NT) {
        const uint32_t t = base + threadIdx.x;
        if (t < A.ntot) pair_sphere<LM>(A, P, t, cur, nxt, ls);
    }
    if (!grid_barrier(G, gridDim.x, A.err)) return;
    for (uint32_t c = blockIdx.x; c < P.nchunks; c += gridDim.x) chunk_sum(A, P, c, s_w);
    if (!grid_barrier(G, gridDim.x, A.err)) return;
    for (uint32_t bx = blockIdx.x; bx < A.nboxes; bx += gridDim.x) box_sum_advance(A, P, bx, s_w);
    if (blockIdx.x == 0 && threadIdx.x == 0) *P.pp ^= 1u;
}

// Self-check of the barrier: `rounds` barriers among the launch's blocks,
// counting `expected` arrivals per barrier (fewer blocks than expected: no
// barrier opens and every block gives up after the limit).
__global__ void k_barrier_check(GridSync G, uint32_t expected, uint32_t rounds, uint32_t *err)
{
    for (uint32_t r = 0; r < rounds; ++r)
        if (!grid_barrier(G, expected, err)) return;
}

// Rebuild request -> the condition of the rebuild node.
__global__ void k_pair_cond(cudaGraphConditionalHandle hc, const uint32_t *vflag)
{
    cudaGraphSetConditional(hc, vflag[0] != 0u ? 1u : 0u);
}

// After a list build into the buffers not in use: each sphere's touching
// entries (and their histories) carried over to the new list -- from the
// old list, or, after pair_load, from the FP64 contact rows.
__global__ void k_pair_remap(StepArgs A, PairArgs P)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const uint32_t ls = *P.lsel, nw = ls ^ 1u;
    const ListRow NL(P, nw, i);
    uint32_t nn = P.cnt[nw][i];
    if (nn > (uint32_t)VL_MAX) nn = 0;   // overflowed: raised by the step kernel
    unsigned long long live = 0ull;
    auto find = [&](uint32_t b) -> int {
        int lo = 0, hi = (int)nn;   // first entry >= b
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (NL.id((uint32_t)mid) < b) lo = mid + 1;
            else hi = mid;
        }
        return lo < (int)nn && NL.id((uint32_t)lo) == b ? lo : -1;
    };
    if (*P.from_rows) {
        for (int s = 0; s < NC; ++s) {
            const uint32_t w = A.slots[(size_t)i * NC + s];
            if (w == EMPTY) continue;
            const int k = find(w & ID_MASK);
            if (k < 0) continue;
            const double4 h = A.hist[(size_t)i * NC + s];
            NL.put3((uint32_t)k, mk(h.x, h.y, h.z));
            live |= 1ull << k;
        }
    } else {
        const ListRow OL(P, ls, i);
        const uint32_t on = min(P.cnt[ls][i], (uint32_t)VL_MAX);
        for (unsigned long long m = P.live[ls][i]; m; m &= m - 1ull) {
            const int ko = __ffsll((long long)m) - 1;
            if ((uint32_t)ko >= on) break;
            const int k = find(OL.id((uint32_t)ko));
            if (k < 0) continue;
            NL.put3((uint32_t)k, OL.hist3((uint32_t)ko));
            live |= 1ull << k;
        }
    }
    P.live[nw][i] = live;
}

// The threads' order over the new lists (P.order[*lsel ^ 1]): within each
// group of PAIR_ORDER_GROUP spheres, ascending list length, ties by index
// (a stable rank), spheres past the end last.  One block per group.
__global__ void __launch_bounds__(PAIR_ORDER_GROUP) k_pair_order(StepArgs A, PairArgs P)
{
    __shared__ uint32_t s_key[PAIR_ORDER_GROUP];
    const uint32_t nw = *P.lsel ^ 1u;
    const uint32_t base = blockIdx.x * PAIR_ORDER_GROUP, t = threadIdx.x, i = base + t;
    uint32_t key = 0xffffffffu;
    if (i < A.ntot) key = min(P.cnt[nw][i], (uint32_t)VL_MAX + 1u);
    s_key[t] = key;
    __syncthreads();
    uint32_t rank = 0;
    for (uint32_t u = 0; u < PAIR_ORDER_GROUP; ++u) {
        const uint32_t k = s_key[u];
        rank += (k < key || (k == key && u < t)) ? 1u : 0u;
    }
    if (i < A.ntot) P.order[nw][base + rank] = i;
}

__global__ void k_pair_done(StepArgs A, PairArgs P)
{
    *P.lsel ^= 1u;
    *P.from_rows = 0u;
    A.vflag[0] = 0u;
    A.vflag[1] += 1u;
}

// The FP64 arrays -> the compact state (into the [*pp] half); the next step
// rebuilds the lists and takes the histories from the contact rows.
__global__ void k_pair_load(StepArgs A, PairArgs P)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t c = *P.pp;
    if (i == 0) {
        *P.from_rows = 1u;
        A.vflag[0] = 1u;
    }
    if (i >= A.ntot) return;
    const double4 v = A.vel[i], w = A.angvel[i], ap = A.angpos[i];
    const double4 ac = A.acc[i], aa = A.angacc[i], f = A.force[i], t = A.torque[i];
    P.xr[c][i] = A.x[i];
    P.vel[i] = v;
    P.vw[c][2 * i] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
    P.vw[c][2 * i + 1] = make_float4((float)w.x, (float)w.y, (float)w.z, 0.f);
    P.angpos[i] = make_float4((float)ap.x, (float)ap.y, (float)ap.z, (float)ap.w);
    P.xyzsum[i] = A.xyzsum[i];
    P.acc[i] = make_float4((float)ac.x, (float)ac.y, (float)ac.z, 0.f);
    P.angacc[i] = make_float4((float)aa.x, (float)aa.y, (float)aa.z, (float)aa.w);
    P.force[i] = make_float4((float)f.x, (float)f.y, (float)f.z, 0.f);
    P.torque[i] = make_float4((float)t.x, (float)t.y, (float)t.z, 0.f);
    P.epp[i] = make_float4((float)A.es_dot[i], (float)A.ev_dot[i], (float)A.p[i], 0.f);
    P.eacc[i] = make_double2(A.es[i], A.ev[i]);
}

// The compact state -> the FP64 arrays, and the touching entries of each
// list -> the sphere's contact row (in list order, slots 0, 1, ...) with
// their histories and image codes.
__global__ void k_pair_flush(StepArgs A, PairArgs P)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const uint32_t c = *P.pp, ls = *P.lsel;
    const double4 xa = P.xr[c][i];
    const float4 w = P.vw[c][2 * i + 1], ap = P.angpos[i], ac = P.acc[i], aa = P.angacc[i];
    const float4 f = P.force[i], t = P.torque[i], e = P.epp[i];
    const double2 ea = P.eacc[i];
    A.x[i] = xa;
    A.vel[i] = P.vel[i];
    A.angvel[i] = make_double4(w.x, w.y, w.z, 0.0);
    A.angpos[i] = make_double4(ap.x, ap.y, ap.z, ap.w);
    A.xyzsum[i] = P.xyzsum[i];
    A.acc[i] = make_double4(ac.x, ac.y, ac.z, 0.0);
    A.angacc[i] = make_double4(aa.x, aa.y, aa.z, aa.w);
    A.force[i] = make_double4(f.x, f.y, f.z, 0.0);
    A.torque[i] = make_double4(t.x, t.y, t.z, 0.0);
    A.es_dot[i] = e.x;
    A.ev_dot[i] = e.y;
    A.p[i] = e.z;
    A.es[i] = ea.x;
    A.ev[i] = ea.y;
    const DevBox &B = A.boxes[box_index(A, i)];
    const ListRow L(P, ls, i);
    const uint32_t nn = min(P.cnt[ls][i], (uint32_t)VL_MAX);
    int s = 0;
    for (unsigned long long m = P.live[ls][i]; m && s < NC; m &= m - 1ull) {
        const int k = __ffsll((long long)m) - 1;
        if ((uint32_t)k >= nn) break;
        const uint32_t b = L.id((uint32_t)k);
        uint32_t code = 0;
        (void)centre_line(B, xa, P.xr[c][b], &code);
        A.slots[(size_t)i * NC + s] = b | (code << CODE_SHIFT);
        const d3 hk = L.hist3((uint32_t)k);
        A.hist[(size_t)i * NC + s] = make_double4(hk.x, hk.y, hk.z, 0.0);
        ++s;
    }
    for (; s < NC; ++s) {
        A.slots[(size_t)i * NC + s] = EMPTY;
        A.hist[(size_t)i * NC + s] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

__global__ void k_pair_count(StepArgs A, PairArgs P, unsigned long long *count)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ls = *P.lsel;
    const unsigned long long v = i < A.ntot ? (unsigned long long)__popcll(P.live[ls][i]) : 0ull;
    unsigned long long s = v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31u) == 0 && s) atomicAdd(count, s);
}

inline void record(cudaEvent_t ev, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    else cudaEventRecord(ev, st);
}

inline void mark(Prof *prof, cudaStream_t st, const char *name)
{
    if (!prof || prof->n >= Prof::MAX) return;
    prof->name[prof->n] = name;
    record(prof->ev[prof->n + 1], st);
    prof->n++;
}

// The list-step kernel at one of its launch shapes (cfg.pair_shape, chosen
// by sph_autotune): threads per block x resident blocks per SM (the
// register budget per thread) and, for the staged kernel, the entries in
// flight per thread --
//   0: 128 x 4 (128 registers)       3: 64 x 8 (128)       4: 256 x 2 (128)
//   1: 128 x 5 (102)                 2: 128 x 6 (85)
//   5: staged, 64 x 8, 4 entries     6: staged, 64 x 8, 6 entries
//   7: staged, 128 x 4, 4 entries    8: staged, 64 x 10, 3 entries
// Fewer registers give more warps to hide the partner gathers, at the cost
// of spilled values; staging keeps more gathers in flight per thread; the
// arithmetic is the same in every shape.
template <int LM, int NT, int MINB, int D>
void launch_staged(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    const size_t sm = sizeof(PairStage<NT, D>);
    static bool attr = false;   // per instantiation: allow more than 48 KB of shared memory
    if (!attr) {
        cudaFuncSetAttribute(k_pair_step_async<LM, NT, MINB, D>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        attr = true;
    }
    k_pair_step_async<LM, NT, MINB, D><<<blocks_for(A.ntot, NT), NT, sm, st>>>(A, P);
}

// The persistent kernel: as many blocks as can be resident at once (at
// most one per NT spheres), launched cooperatively (the launch fails rather
// than run blocks that could not all be resident); the barrier's count is
// cleared before each launch.
template <int LM, int NT, int MINB>
void launch_persistent(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    static int per_sm = -1, sms = 0;
    if (per_sm < 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_persist<LM, NT, MINB>, NT, 0);
    }
    const unsigned need = blocks_for(A.ntot, NT);
    const unsigned cap = (unsigned)(per_sm > 0 ? per_sm : 1) * (unsigned)sms;
    GridSync G;
    G.count = P.bar;
    G.gen = P.bar + 1;
    G.limit_ns = BARRIER_LIMIT_NS;
    cudaMemsetAsync(P.bar, 0, sizeof(uint32_t), st);
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(need < cap ? need : cap);
    c.blockDim = dim3(NT);
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    c.attrs = at;
    c.numAttrs = 1;
    cudaLaunchKernelEx(&c, k_pair_persist<LM, NT, MINB>, A, P, G);
}

template <int LM>
void launch_pair_lm(const StepArgs &A, const PairArgs &P, int shape, cudaStream_t st)
{
    switch (shape) {
    case 1: k_pair_step<LM, 128, 5><<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, P); break;
    case 2: k_pair_step<LM, 128, 6><<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, P); break;
    case 3: k_pair_step<LM, 64, 8><<<blocks_for(A.ntot, 64), 64, 0, st>>>(A, P); break;
    case 4: k_pair_step<LM, 256, 2><<<blocks_for(A.ntot, 256), 256, 0, st>>>(A, P); break;
    case 5: launch_staged<LM, 64, 8, 4>(A, P, st); break;
    case 6: launch_staged<LM, 64, 8, 6>(A, P, st); break;
    case 7: launch_staged<LM, 128, 4, 4>(A, P, st); break;
    case 8: launch_staged<LM, 64, 10, 3>(A, P, st); break;
    case 9: launch_persistent<LM, 64, 8>(A, P, st); break;
    case 10: launch_persistent<LM, 128, 4>(A, P, st); break;
    case 11: k_pair_step<LM, 64, 10, false><<<blocks_for(A.ntot, 64), 64, 0, st>>>(A, P); break;
    case 12: k_pair_step<LM, 64, 12, false><<<blocks_for(A.ntot, 64), 64, 0, st>>>(A, P); break;
    default: k_pair_step<LM, 128, 4><<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, P); break;
    }
}

void launch_pair_kernel(const StepArgs &A, const PairArgs &P, const StepConfig &cfg,
                        cudaStream_t st)
{
    if (cfg.lenmode == SPH_LEN_FP64) launch_pair_lm<SPH_LEN_FP64>(A, P, cfg.pair_shape, st);
    else launch_pair_lm<SPH_LEN_REFERENCE>(A, P, cfg.pair_shape, st);
}

void launch_rebuild_body(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    launch_pair_sort_build(A, P, st);
    k_pair_remap<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A, P);
    k_pair_order<<<blocks_for(A.ntot, PAIR_ORDER_GROUP), PAIR_ORDER_GROUP, 0, st>>>(A, P);
    k_pair_done<<<1, 1, 0, st>>>(A, P);
}

}  // namespace

// One step of the list form on st.  Under stream capture the list rebuild
// is a conditional node (run when the integration of the step before asked
// for it); outside a capture the request is read on the host.  cfg.side:
// a second stream, on which the conditional node's body is captured.
int launch_step_pair(const StepArgs &A, const PairArgs &P, const StepConfig &cfg, cudaStream_t st,
                     uint64_t *launches, Prof *prof)
{
    uint64_t nl = 0;
    if (prof) {
        prof->n = 0;
        record(prof->ev[0], st);
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return SPH_ERR_CUDA;
    if (cs == cudaStreamCaptureStatusActive) {
        if (!cfg.side) return SPH_ERR_CUDA;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd) != cudaSuccess)
            return SPH_ERR_CUDA;
        cudaGraphConditionalHandle hc;
        if (cudaGraphConditionalHandleCreate(&hc, g, 0u, cudaGraphCondAssignDefault) != cudaSuccess)
            return SPH_ERR_CUDA;
        k_pair_cond<<<1, 1, 0, st>>>(hc, A.vflag);
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd) != cudaSuccess)
            return SPH_ERR_CUDA;
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = hc;
        np.conditional.type = cudaGraphCondTypeIf;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g, deps, nd, &np) != cudaSuccess) return SPH_ERR_CUDA;
        if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) !=
            cudaSuccess)
            return SPH_ERR_CUDA;
        cudaGraph_t body = np.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(cfg.side, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return SPH_ERR_CUDA;
        launch_rebuild_body(A, P, cfg.side);
        cudaGraph_t done = nullptr;
        if (cudaStreamEndCapture(cfg.side, &done) != cudaSuccess) return SPH_ERR_CUDA;
        nl += 1;
    } else {
        uint32_t flag = 0;
        if (cudaMemcpyAsync(&flag, A.vflag, sizeof flag, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return SPH_ERR_CUDA;
        if (flag) launch_rebuild_body(A, P, st);
    }
    mark(prof, st, "k_pair_cond");
    launch_pair_kernel(A, P, cfg, st);
    if (pair_shape_persistent(cfg.pair_shape)) {
        // the persistent shapes do the wall stage themselves
        mark(prof, st, "k_pair_persist");
        if (launches) *launches += nl + 1;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            fprintf(stderr, "sphere_b200: list-step launch failed: %s\n", cudaGetErrorString(e));
            return SPH_ERR_CUDA;
        }
        return SPH_OK;
    }
    mark(prof, st, "k_pair_step");
    const bool pdl = prof == nullptr;
    if (cfg.any_walls) {
        launch_k(pdl, k_pair_chunks, P.nchunks, CHUNK_THREADS, st, A, P);
        mark(prof, st, "k_pair_chunks");
        nl += 1;
    }
    launch_k(pdl && cfg.any_walls, k_pair_box, A.nboxes, PBOX_THREADS, st, A, P);
    mark(prof, st, "k_pair_box");
    nl += 2;
    if (launches) *launches += nl;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "sphere_b200: list-step launch failed: %s\n", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

int barrier_check(uint32_t blocks, uint32_t expected, uint32_t rounds,
                  unsigned long long limit_ns, uint32_t *d_words, uint32_t *d_err,
                  cudaStream_t st)
{
    if (cudaMemsetAsync(d_words, 0, 2 * sizeof(uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st) != cudaSuccess)
        return SPH_ERR_CUDA;
    GridSync G;
    G.count = d_words;
    G.gen = d_words + 1;
    G.limit_ns = limit_ns;
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(blocks);
    c.blockDim = dim3(32);
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    c.attrs = at;
    c.numAttrs = 1;
    if (cudaLaunchKernelEx(&c, k_barrier_check, G, expected, rounds, d_err) != cudaSuccess)
        return SPH_ERR_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

int pair_load(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    k_pair_load<<<blocks_for(A.ntot ? A.ntot : 1, 256), 256, 0, st>>>(A, P);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

int pair_flush(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    if (A.ntot) k_pair_flush<<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, P);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

int pair_count_live(const StepArgs &A, const PairArgs &P, cudaStream_t st,
                    unsigned long long *d_count)
{
    cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
    if (A.ntot) k_pair_count<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A, P, d_count);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

}  // namespace sph
