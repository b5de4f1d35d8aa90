// sph_step.cuh -- the fused per-sphere step kernel (topology, interact,
// walls, bond forces, TY3 integration) shared by the FP64 step
// (sph_kernels.cu, no FMA contraction) and the FP32-mixed step
// (sph_mixed.cu).
#pragma once

#include <cstdint>

#include "sph_device.cuh"
#include "sph_internal.h"
#include "sph_mixed_laws.cuh"

namespace sph {

// Conservative FP32 candidate test: false only when the pair certainly does
// not satisfy the exact FP64 test `length - (ra + rb) < extra` (extra = 0
// for contacts, db for capillary bonds).  B.pre_margin bounds the rounding
// of the FP32 copies, differences, periodic shifts and of the reference's
// FP32-rounded lengths (set per box by the host: 2^-19 (max L + 2 r_max)).
__device__ __forceinline__ bool maybe_touching(float4 xa, float4 xb, float sx, float sy,
                                               float margin_plus_extra)
{
    const float dx = (xa.x - xb.x) + sx, dy = (xa.y - xb.y) + sy, dz = xa.z - xb.z;
    const float rr = xa.w + xb.w + margin_plus_extra;
    return dx * dx + dy * dy + dz * dz < rr * rr;
}

// Box of sphere i; a single box needs no lookup (one dependent load fewer
// on the way to the box's parameters).
__device__ __forceinline__ uint32_t box_index(const StepArgs &A, uint32_t i)
{
    return A.nboxes == 1 ? 0u : A.box_of[i];
}

// ---------------------------------------------------------------- integrate

// integration.cuh:14-305 integrate (TY3) for one particle.
__device__ __forceinline__ void integrate_particle(const StepArgs &A, const DevBox &B,
                                                   uint32_t i, double4 x, double4 vel,
                                                   double4 angvel, d3 F, d3 T)
{
    const SphParams &P = B.P;
    const double dt = B.dt;
    const double4 angpos = A.angpos[i];
    double4 xyzsum = A.xyzsum[i];
    int wall0mode = 0;
    double wall0mass = 0.0;
    if (B.nw > 0) {
        wall0mode = B.wmode[0];
        wall0mass = B.wmvfd[0][0];
    }
    double4 acc0 = make_double4(0.0, 0.0, 0.0, 0.0), angacc0 = acc0;
    if (B.iter != 0) {
        acc0 = A.acc[i];
        angacc0 = A.angacc[i];
    }
    const double radius = x.w;
    const double m = 4.0 / 3.0 * PI * radius * radius * radius * P.rho;
    double acc[3], angacc[3];
    acc[0] = F.x / m + P.g[0];
    acc[1] = F.y / m + P.g[1];
    acc[2] = F.z / m + P.g[2];
    angacc[0] = T.x * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc[1] = T.y * 1.0 / (2.0 / 5.0 * m * radius * radius);
    angacc[2] = T.z * 1.0 / (2.0 / 5.0 * m * radius * radius);
    double angacc_w = 0.0;
    if (wall0mode == 3 && vel.w > 0.0001 && x.z > B.L[2] * 0.5) {
        const double f_tau_x = (B.tau_x + B.tau_eff_x) * B.L[0] * B.L[1];
        acc[0] = f_tau_x / wall0mass;
        acc[1] = 0.0;
        acc[2] -= P.g[2];
        angacc[0] = angacc[1] = angacc[2] = 0.0;
        angacc_w = 0.0;
    } else if (vel.w > 0.0001 && vel.w < 10.0) {
        acc[0] = 0.0;
        acc[1] = 0.0;
        acc[2] -= P.g[2];
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
    const double a0[3] = {acc0.x, acc0.y, acc0.z};
    const double w0[3] = {angacc0.x, angacc0.y, angacc0.z};
    const double xv[3] = {x.x, x.y, x.z};
    const double vv[3] = {vel.x, vel.y, vel.z};
    const double pv[3] = {angpos.x, angpos.y, angpos.z};
    const double wv[3] = {angvel.x, angvel.y, angvel.z};
    double sv[3] = {xyzsum.x, xyzsum.y, xyzsum.z};
    double xn[3], vn[3], pn[3], wn[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double dacc = (acc[d] - a0[d]) / dt;
        const double dangacc = (angacc[d] - w0[d]) / dt;
        xn[d] = xv[d] + vv[d] * dt + 0.5 * acc[d] * dt * dt + 1.0 / 6.0 * dacc * dt * dt * dt;
        vn[d] = vv[d] + acc[d] * dt + 0.5 * dacc * dt * dt;
        pn[d] = pv[d] + wv[d] * dt + 0.5 * angacc[d] * dt * dt + 1.0 / 6.0 * dangacc * dt * dt * dt;
        wn[d] = wv[d] + angacc[d] * dt + 0.5 * dangacc * dt * dt;
        sv[d] += vv[d] * dt + 0.5 * acc[d] * dt * dt + 1.0 / 6.0 * dacc * dt * dt * dt;
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
    if (A.xref) {
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
    xyzsum.x = sv[0];
    xyzsum.y = sv[1];
    xyzsum.z = sv[2];
    A.xyzsum[i] = xyzsum;
    A.acc[i] = make_double4(acc[0], acc[1], acc[2], 0.0);
    A.angacc[i] = make_double4(angacc[0], angacc[1], angacc[2], angacc_w);
    A.angvel[i] = make_double4(wn[0], wn[1], wn[2], angvel.w);
    A.vel[i] = make_double4(vn[0], vn[1], vn[2], vel.w);
    A.angpos[i] = make_double4(pn[0], pn[1], pn[2], angpos.w);
    A.x[i] = make_double4(xn[0], xn[1], xn[2], x.w);
}

// integration.cuh:344-450 integrateWalls with the wall-force total fsum,
// then the loop bookkeeping of device.cu:2536-2538, the adaptive grid of
// device.cu:1050 and the velocity-step state of device.cu:2455-2462 for
// the next step.  One thread per box.
__device__ __forceinline__ void advance_box(DevBox &B, double fsum)
{
    const double dt = B.dt;
    if (B.np > 0) {
        for (uint32_t w = 0; w < B.nw; ++w) {
            const int wmode = B.wmode[w];
            if (wmode == 0) continue;
            const double acc0 = B.iter == 0 ? 0.0 : B.wacc[w];
            B.wmvfd[w][2] = fsum;
            const double sigma_0 =
                B.wmvfd[w][3] + B.P.sigma0_A * sin(2.0 * PI * B.P.sigma0_f * B.t_current);
            const double N = -sigma_0 * B.L[0] * B.L[1];
            double acc = (B.wmvfd[w][2] + N) / B.wmvfd[w][0];
            if (wmode == 2) acc = 0.0;
            const double dacc_dt = (acc - acc0) / dt;
            B.wnx[w][3] += B.wmvfd[w][1] * dt + 0.5 * acc * dt * dt + 1.0 / 6.0 * dacc_dt * dt * dt * dt;
            B.wmvfd[w][1] += acc * dt + 0.5 * dacc_dt * dt * dt;
            B.wacc[w] = acc;
        }
    }
    B.t_current += dt;
    B.iter += 1;
    B.L2_out = B.L[2];
    if (B.adaptive == 1 && B.nw > 0) B.L[2] = B.wnx[0][3];
    int change = 0;
    if (B.t_current >= 10.0 && B.t_current < 15.0 && B.velocity_state == 1) {
        change = 1;
        B.velocity_state = 2;
    } else if (B.t_current >= 15.0 && B.velocity_state == 2) {
        change = -1;
        B.velocity_state = 1;
    }
    B.change_velocity_state = change;
}

// ------------------------------------------------------------------ interact

// Neighbour-list entry k of sphere a (partner id bo): the cell search visits
// the partner's cell at ordinal (dz, dy, dx) of the 27-cell loop under image
// (sx, sy), and the exact FP64 test says the pair touches.  Returns the
// insertion key (ordinal << 10 | image code << 6 | k), or NO_KEY.
constexpr uint16_t NO_KEY = 0xffffu;

template <int LM>
__device__ __forceinline__ uint16_t list_key(const StepArgs &A, const DevBox &B, double4 xa,
                                             const int g[3], uint32_t bo, uint32_t k)
{
    int bx, by, bz, dx, dy, dz, sx, sy;
    unpack_cell(A.cellc[bo], bx, by, bz);
    if (!relative_cell(B, g, bx, by, bz, dx, dy, dz, sx, sy)) return NO_KEY;
    const double4 xb = A.xs[A.rank[bo]];
    const d3 dm = shift_vec(B, sx, sy);
    d3 x_ab = mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
    x_ab = vadd(x_ab, dm);
    const double len = vlen<LM>(x_ab);
    if (!(len - (xa.w + xb.w) < 0.0)) return NO_KEY;
    const int ord = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
    return (uint16_t)((ord << 10) | (shift_code(sx, sy) << 6) | (int)k);
}

// list_key for entries k0 .. k0 + KB - 1 (those below vc), their loads
// issued together so that KB gathers are in flight at once.  For the split
// step only: the partner's position is read in original order (A.x), which
// holds the step's start positions until k_finish, one gather fewer than
// the sorted copy through rank.
constexpr int KB = 4;   // (the overflow path of k_search spells out KB entries)

// FILTER: entries whose partner already holds a slot of the row (srow[j] >=
// 0) are not tested: only their image code is brought up to date (in place,
// *dirty set when it changes); the caller uses this when the row cannot
// overflow, where such entries do not change where the new ones go.
template <int LM, bool FILTER>
__device__ __forceinline__ void list_keys_batch(const StepArgs &A, const DevBox &B, double4 xa,
                                                const int g[3], const uint32_t bo[KB], uint32_t k0,
                                                uint32_t vc, uint16_t out[KB], const int srow[KB],
                                                uint32_t *row, int RS, bool *dirty)
{
    uint64_t cc[KB];
    double4 xb[KB];
#pragma unroll
    for (int j = 0; j < KB; ++j) {
        const bool test = k0 + j < vc && (!FILTER || srow[j] < 0);
        cc[j] = k0 + j < vc ? A.cellc[bo[j]] : 0ull;
        xb[j] = test ? A.x[bo[j]] : make_double4(0.0, 0.0, 0.0, 0.0);
    }
#pragma unroll
    for (int j = 0; j < KB; ++j) {
        out[j] = NO_KEY;
        if (k0 + j >= vc) continue;
        int bx, by, bz, dx, dy, dz, sx, sy;
        unpack_cell(cc[j], bx, by, bz);
        if (!relative_cell(B, g, bx, by, bz, dx, dy, dz, sx, sy)) continue;
        if (FILTER && srow[j] >= 0) {
            const uint32_t v = bo[j] | (shift_code(sx, sy) << CODE_SHIFT);
            if (row[srow[j] * RS] != v) {
                row[srow[j] * RS] = v;
                *dirty = true;
            }
            continue;
        }
        const d3 dm = shift_vec(B, sx, sy);
        d3 x_ab = mk(xa.x - xb[j].x, xa.y - xb[j].y, xa.z - xb[j].z);
        x_ab = vadd(x_ab, dm);
        const double len = vlen<LM>(x_ab);
        if (!(len - (xa.w + xb[j].w) < 0.0)) continue;
        const int ord = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
        out[j] = (uint16_t)((ord << 10) | (shift_code(sx, sy) << 6) | (int)(k0 + j));
    }
}

// Insert the touching list entries, keys sorted ascending (keys[q * KS]),
// into the slot row with the reference's rule: an existing contact keeps
// its slot, a new one takes the last free slot (slot nc when none is free);
// more than NC contacts raise SPH_ERR_NC_OVERFLOW and skip the rest of that
// cell, as the cell search does.  occ: bit s set when slot s is in use
// (updated).  Returns whether the row changed.
__device__ __forceinline__ bool insert_keys(const StepArgs &A, const uint16_t *keys, int nk, int KS,
                                            const uint32_t *lst, uint32_t *row, int RS,
                                            uint32_t &occ)
{
    bool dirty = false;
    int nc = 0, cur_ord = -1;
    bool full = false;
    for (int q = 0; q < nk; ++q) {
        const uint32_t key = keys[q * KS];
        const int ord = (int)(key >> 10);
        if (ord != cur_ord) {
            cur_ord = ord;
            full = false;
        }
        if (full) continue;
        const uint32_t b_orig = lst[key & 63u];
        // the partner's slot if it is in the row, else the highest free slot
        int cpos = -1;
        for (uint32_t m = occ; m; m &= m - 1u) {
            const int s = __ffs(m) - 1;
            if ((row[s * RS] & ID_MASK) == b_orig) {
                cpos = s;
                break;
            }
        }
        if (cpos < 0) cpos = ~occ ? 31 - __clz(~occ) : nc;
        if (cpos < NC) {
            // the row goes back to memory only if an entry changed
            const uint32_t v = b_orig | (((key >> 6) & 15u) << CODE_SHIFT);
            if (row[cpos * RS] != v) {
                row[cpos * RS] = v;
                dirty = true;
            }
            occ |= 1u << cpos;
        } else {
            raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
        }
        ++nc;
        if (nc > NC) {
            raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
            full = true;
        }
    }
    return dirty;
}

__device__ __forceinline__ uint32_t occupancy(const uint32_t *row, int RS)
{
    uint32_t occ = 0;
#pragma unroll
    for (int s = 0; s < NC; ++s) occ |= (row[s * RS] != EMPTY ? 1u : 0u) << s;
    return occ;
}

// The 27-cell contact search (contactsearch.cuh:329-371 and :194-322) on
// the slot row, for spheres without a usable neighbour list.
template <int LM>
__device__ __forceinline__ bool search_cells(const StepArgs &A, const DevBox &B, uint32_t a,
                                             double4 xa, const int g[3], float4 xaf,
                                             uint32_t *row, int RS)
{
    const double radius_a = xa.w;
    const int nx = (int)B.num[0], ny = (int)B.num[1];
    const float Lf0 = (float)B.L[0], Lf1 = (float)B.L[1];
    const float margin = B.pre_margin;
    bool dirty = false;
    int nc = 0;
    for (int dz = -1; dz < 2; ++dz)
        for (int dy = -1; dy < 2; ++dy)
            for (int dx = -1; dx < 2; ++dx) {
                int tx = g[0] + dx, ty = g[1] + dy, sx, sy;
                const int tz = g[2] + dz;
                if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                const d3 dm = shift_vec(B, sx, sy);
                const float fsx = sx == 0 ? 0.f : (sx > 0 ? Lf0 : -Lf0);
                const float fsy = sy == 0 ? 0.f : (sy > 0 ? Lf1 : -Lf1);
                const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                const uint32_t start = A.cell_off[cell], end = A.cell_off[cell + 1];
                for (uint32_t b = start; b < end; ++b) {
                    if (b == a) continue;
                    if (!maybe_touching(xaf, A.xf[b], fsx, fsy, margin)) continue;
                    const double4 xb = A.xs[b];
                    d3 x_ab = mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
                    x_ab = vadd(x_ab, dm);
                    const double len = vlen<LM>(x_ab);
                    const double delta = len - (radius_a + xb.w);
                    if (delta < 0.0) {
                        const uint32_t b_orig = A.perm[b];
                        int cpos = nc;
                        for (int s = 0; s < NC; ++s) {
                            const uint32_t w = row[s * RS];
                            if (w == EMPTY) cpos = s;
                            else if ((w & ID_MASK) == b_orig) { cpos = s; break; }
                        }
                        if (cpos < NC) {
                            const uint32_t v = b_orig | (shift_code(sx, sy) << CODE_SHIFT);
                            if (row[cpos * RS] != v) {
                                row[cpos * RS] = v;
                                dirty = true;
                            }
                        } else {
                            raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
                        }
                        ++nc;
                        if (nc > NC) {
                            raise_flag(A.err, SPH_ERR_NC_OVERFLOW);
                            break;
                        }
                    }
                }
            }
    return dirty;
}

// The contact search of one sphere (contact models 2 and 3) on its slot row
// staged in shared memory (row[s * RS]), one thread: from the neighbour list
// when the sphere has one (the touching entries keyed and inserted in the
// order the cell search would find them), else the 27-cell search.  keys:
// shared scratch of VL_MAX entries at stride RS.  Returns whether the row
// changed.
template <int LM>
__device__ __forceinline__ bool search_contacts(const StepArgs &A, const DevBox &B, uint32_t a,
                                                uint32_t i, double4 xa, const int g[3],
                                                float4 xaf, uint32_t *row, uint16_t *keys,
                                                int RS)
{
    const uint32_t vc = A.vlist ? A.vcount[i] : (uint32_t)VL_MAX + 1u;
    if (vc > (uint32_t)VL_MAX) return search_cells<LM>(A, B, a, xa, g, xaf, row, RS);
    const uint32_t *lst = A.vlist + (size_t)i * VL_MAX;
    int nk = 0;
    for (uint32_t k = 0; k < vc; ++k) {
        const uint16_t key = list_key<LM>(A, B, xa, g, lst[k], k);
        if (key == NO_KEY) continue;
        int q = nk;
        while (q > 0 && keys[(q - 1) * RS] > key) {
            keys[q * RS] = keys[(q - 1) * RS];
            --q;
        }
        keys[q * RS] = key;
        ++nk;
    }
    uint32_t occ = occupancy(row, RS);
    return insert_keys(A, keys, nk, RS, lst, row, RS, occ);
}

// Static and dynamic walls (contactsearch.cuh:428-465 and :602-701) and the
// bond forces in ascending bond order (cohesion.cuh:220-226), added to acc
// after the contacts.  Returns the normal force on wall 0.
template <int LM>
__device__ __forceinline__ double walls_and_bonds(const StepArgs &A, const DevBox &B, uint32_t i,
                                                  double4 xa, d3 vel_a, d3 angvel_a, Acc &acc)
{
    const SphParams &P = B.P;
    const double dt = B.dt;
    const double radius_a = xa.w;
    double wnx[5][4] = {{0.0, 0.0, -1.0, B.L[2]}, {-1.0, 0.0, 0.0, B.L[0]}, {1.0, 0.0, 0.0, 0.0},
                        {0.0, -1.0, 0.0, B.L[1]}, {0.0, 1.0, 0.0, 0.0}};
    double wvel[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const uint32_t nw = B.nw;
    for (uint32_t w = 0; w < 5 && w < nw; ++w) {
        wnx[w][0] = B.wnx[w][0];
        wnx[w][1] = B.wnx[w][1];
        wnx[w][2] = B.wnx[w][2];
        wnx[w][3] = B.wnx[w][3];
        wvel[w] = B.wmvfd[w][1];
    }
    double w0_force = 0.0;
    {
        double delta_w = wnx[0][3] - (xa.z + radius_a);
        if (delta_w < 0.0)
            w0_force = contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a,
                                               mk(wnx[0][0], wnx[0][1], wnx[0][2]), delta_w, wvel[0]);
        delta_w = xa.z - radius_a - B.origo[2];
        if (delta_w < 0.0)
            (void)contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a, mk(0.0, 0.0, 1.0),
                                          delta_w, 0.0);
        if (B.periodic == 0) {
            delta_w = wnx[1][3] - (xa.x + radius_a);
            if (delta_w < 0.0)
                (void)contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a,
                                              mk(wnx[1][0], wnx[1][1], wnx[1][2]), delta_w, wvel[1]);
            delta_w = xa.x - radius_a - wnx[2][3];
            if (delta_w < 0.0)
                (void)contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a,
                                              mk(wnx[2][0], wnx[2][1], wnx[2][2]), delta_w, wvel[2]);
        }
        if (B.periodic == 0 || B.periodic == 2) {
            delta_w = wnx[3][3] - (xa.y + radius_a);
            if (delta_w < 0.0)
                (void)contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a,
                                              mk(wnx[3][0], wnx[3][1], wnx[3][2]), delta_w, wvel[3]);
            delta_w = xa.y - radius_a - wnx[4][3];
            if (delta_w < 0.0)
                (void)contact_linear_wall<LM>(P, dt, acc, vel_a, angvel_a, radius_a,
                                              mk(wnx[4][0], wnx[4][1], wnx[4][2]), delta_w, wvel[4]);
        }
    }

    // ---- bond forces in ascending bond order: cohesion.cuh:220-226
    if (A.nbonds) {
        const uint32_t e0 = A.bcsr_off[i], e1 = A.bcsr_off[i + 1];
        for (uint32_t e = e0; e < e1; ++e) {
            const uint32_t ent = A.bcsr_ent[e];
            const uint32_t k = ent >> 1;
            const double4 f = A.bf[k];
            if (f.w == 0.0) continue;
            const double4 t = A.bt[k];
            if ((ent & 1u) == 0) {
                acc.F = vadd(acc.F, xyz(f));
                acc.T = vsub(acc.T, xyz(t));
            } else {
                acc.F = vsub(acc.F, xyz(f));
                acc.T = vadd(acc.T, xyz(t));
            }
        }
    }

    return w0_force;
}

// The per-sphere sums of the step (contactsearch.cuh:707-724).
__device__ __forceinline__ void store_sums(const StepArgs &A, const DevBox &B, uint32_t i,
                                           const Acc &acc, double w0_force)
{
    const double dt = B.dt;
    A.force[i] = make_double4(acc.F.x, acc.F.y, acc.F.z, 0.0);
    A.torque[i] = make_double4(acc.T.x, acc.T.y, acc.T.z, 0.0);
    A.es_dot[i] = acc.es_dot;
    A.ev_dot[i] = acc.ev_dot;
    A.es[i] += acc.es_dot * dt;
    A.ev[i] += acc.ev_dot * dt;
    A.p[i] = acc.p;
    if (B.nw > 0) A.wf_pp[i] = w0_force;

}

constexpr int INTERACT_THREADS = 128;

// Fused topology + interact + walls + bond gather (+ integrate when FUSED)
// for the particle at sorted position a.  Neighbour data is read from the
// sorted copies only, so writing the particle's new state in place is safe.
// The particle's contact row is staged in shared memory (slot-major, one
// column per thread); only live slots are processed, empty slots keep a
// zero tangential history by construction.
template <int LM, bool FUSED, bool MIXED, int MINB>
__global__ void __launch_bounds__(INTERACT_THREADS, MINB) k_interact(StepArgs A)
{
    __shared__ uint32_t s_row[NC * INTERACT_THREADS];
    __shared__ uint16_t s_keys[VL_MAX * INTERACT_THREADS];
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ntot) return;
    uint32_t *row = s_row + threadIdx.x;
    const int RS = INTERACT_THREADS;
    const uint32_t i = A.perm[a];
    const DevBox &B = A.boxes[box_index(A, i)];
    const SphParams &P = B.P;
    const double dt = B.dt;
    const double4 xa = A.xs[a];
    const double radius_a = xa.w;
    const double4 va4 = A.vs[a];
    const double4 wa4 = A.ws[a];
    const d3 vel_a = xyz(va4);
    const d3 angvel_a = xyz(wa4);
    const uint32_t cm = P.contactmodel;

    const uint4 *grow = reinterpret_cast<const uint4 *>(A.slots + (size_t)i * NC);
#pragma unroll
    for (int q = 0; q < NC / 4; ++q) {
        const uint4 w = grow[q];
        row[(4 * q + 0) * RS] = w.x;
        row[(4 * q + 1) * RS] = w.y;
        row[(4 * q + 2) * RS] = w.z;
        row[(4 * q + 3) * RS] = w.w;
    }
    bool dirty = false;
    if (A.tape_rows_pre) {
        uint4 *t = reinterpret_cast<uint4 *>(A.tape_rows_pre + (size_t)i * NC);
#pragma unroll
        for (int q = 0; q < NC / 4; ++q) t[q] = grow[q];
    }

    Acc acc;
    acc.F = mk(0.0, 0.0, 0.0);
    acc.T = mk(0.0, 0.0, 0.0);
    acc.es_dot = 0.0;
    acc.ev_dot = 0.0;
    acc.p = 0.0;

    const int nx = (int)B.num[0], ny = (int)B.num[1];
    int g[3];
    if (cm != 0) {
        g[0] = (int)floor((xa.x - B.origo[0]) / (B.L[0] / B.num[0]));
        g[1] = (int)floor((xa.y - B.origo[1]) / (B.L[1] / B.num[1]));
        g[2] = (int)floor((xa.z - B.origo[2]) / (B.L[2] / B.num[2]));
    }

    const float4 xaf = A.xf[a];
    const float Lf0 = (float)B.L[0], Lf1 = (float)B.L[1];
    if (cm == 2 || cm == 3) {
        // ---- topology: contactsearch.cuh:329-371 and :194-322
        if (search_contacts<LM>(A, B, a, i, xa, g, xaf, row, s_keys + threadIdx.x, RS)) dirty = true;

        // ---- interact over the contact row: contactsearch.cuh:484-559
        double4 *hist = A.hist + (size_t)i * NC;
        if (A.tape_rows_post) {
            for (int s = 0; s < NC; ++s) {
                const uint32_t w = row[s * RS];
                A.tape_rows_post[(size_t)i * NC + s] = w;
                if (w != EMPTY) A.tape_hist[(size_t)i * NC + s] = hist[s];
            }
        }
        // live slots in ascending order, so that the threads of a warp work
        // on their q-th contact together (the forces still add up in slot
        // order)
        uint16_t *live = s_keys + threadIdx.x;
        int nlive = 0;
        for (int s = 0; s < NC; ++s)
            if (row[s * RS] != EMPTY) live[(nlive++) * RS] = (uint16_t)s;
        for (int q = 0; q < nlive; ++q) {
            const int s = live[q * RS];
            const uint32_t w = row[s * RS];
            const uint32_t b_orig = w & ID_MASK;
            int sx, sy;
            decode_shift(w >> CODE_SHIFT, sx, sy);
            const d3 dm = shift_vec(B, sx, sy);
            const uint32_t bs = A.rank[b_orig];
            const double4 xb = A.xs[bs];
            const d3 x_ab = mk(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            const double x_ab_length = vlen<LM>(x_ab);
            const double delta_n = x_ab_length - (radius_a + xb.w);
            if (delta_n < 0.0) {
                const d3 vel_b = xyz(A.vs[bs]);
                const d3 h0 = xyz(hist[s]);
                d3 nd;
                if (MIXED) {
                    const MixedPair q = mixed_pair(x_ab, x_ab_length, delta_n, vel_a, vel_b,
                                                   tof(angvel_a), xyzf(A.ws[bs]), radius_a, xb.w);
                    if (cm == 2) nd = contact_linear_mixed(P, dt, acc, q, h0);
                    else nd = contact_hertz_mixed(P, dt, acc, q, h0);
                } else {
                    const d3 angvel_b = xyz(A.ws[bs]);
                    if (cm == 2)
                        nd = contact_linear<LM>(P, dt, acc, vel_a, vel_b, angvel_a, angvel_b,
                                                radius_a, xb.w, x_ab, x_ab_length, delta_n, h0);
                    else
                        nd = contact_hertz<LM>(P, dt, acc, vel_a, vel_b, angvel_a, angvel_b,
                                               radius_a, xb.w, x_ab, x_ab_length, delta_n, h0);
                }
                hist[s] = make_double4(nd.x, nd.y, nd.z, 0.0);
            } else {
                row[s * RS] = EMPTY;
                dirty = true;
                hist[s] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
        }
    } else if (cm == 1) {
        // ---- contact model 1: contactsearch.cuh:564-598 and :91-186
        const float reach = B.pre_margin + (float)fmax(P.db, 0.0) * 1.0001f;
        for (int dz = -1; dz < 2; ++dz)
            for (int dy = -1; dy < 2; ++dy)
                for (int dx = -1; dx < 2; ++dx) {
                    int tx = g[0] + dx, ty = g[1] + dy, sx, sy;
                    const int tz = g[2] + dz;
                    if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                    const d3 dm = shift_vec(B, sx, sy);
                    const float fsx = sx == 0 ? 0.f : (sx > 0 ? Lf0 : -Lf0);
                    const float fsy = sy == 0 ? 0.f : (sy > 0 ? Lf1 : -Lf1);
                    const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                    const uint32_t start = A.cell_off[cell], end = A.cell_off[cell + 1];
                    for (uint32_t b = start; b < end; ++b) {
                        if (b == a) continue;
                        if (!maybe_touching(xaf, A.xf[b], fsx, fsy, reach)) continue;
                        const double4 xb = A.xs[b];
                        const double kappa = P.kappa;
                        d3 x_ab = mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
                        x_ab = vadd(x_ab, dm);
                        const double x_ab_length = vlen<LM>(x_ab);
                        const double delta_ab = x_ab_length - (radius_a + xb.w);
                        if (delta_ab < 0.0) {
                            if (MIXED)
                                contact_linear_viscous_mixed(
                                    P, acc,
                                    mixed_pair(x_ab, x_ab_length, delta_ab, vel_a, xyz(A.vs[b]),
                                               tof(angvel_a), xyzf(A.ws[b]), radius_a, xb.w),
                                    (float)kappa);
                            else
                                contact_linear_viscous<LM>(P, acc, vel_a, xyz(A.vs[b]), angvel_a,
                                                           xyz(A.ws[b]), radius_a, xb.w, x_ab,
                                                           x_ab_length, delta_ab, kappa);
                        } else if (delta_ab < P.db) {
                            capillary_cohesion_exp(P, acc, radius_a, xb.w, delta_ab, x_ab,
                                                   x_ab_length, kappa);
                        }
                    }
                }
    }

    const double w0_force = walls_and_bonds<LM>(A, B, i, xa, vel_a, angvel_a, acc);

    if (dirty) {
        uint4 *wrow = reinterpret_cast<uint4 *>(A.slots + (size_t)i * NC);
#pragma unroll
        for (int q = 0; q < NC / 4; ++q)
            wrow[q] = make_uint4(row[(4 * q) * RS], row[(4 * q + 1) * RS], row[(4 * q + 2) * RS],
                                 row[(4 * q + 3) * RS]);
    }

    store_sums(A, B, i, acc, w0_force);

    if (FUSED) integrate_particle(A, B, i, xa, va4, wa4, acc.F, acc.T);
}

// ------------------------------------------------------------ split step
//
// The step of k_interact for contact models 2 and 3 with fused integration,
// in three launches that keep more memory requests in flight:
//   k_search   one thread per sphere: contact search on the slot row (kept
//              with a bitmask of the slots in use), the list of live slots
//              (ascending);
//   k_contacts one warp per 32 spheres, the warp's live contacts dealt to
//              its lanes 32 at a time: the contact law with its additions
//              recorded (ContactRec), the new history written, ended
//              contacts removed from the row; the records go through shared
//              memory to the lane of their sphere, which adds them in slot
//              order and stores the sums;
//   k_finish   one thread per sphere, original order: walls, bonds, sums,
//              integration.
// Each contact's arithmetic and the order of every sum are those of
// k_interact, so the results are bit-identical.
constexpr int SEARCH_THREADS = 128;
constexpr int CONTACT_THREADS = 128;
constexpr int FINISH_THREADS = 128;

// Contact search of sphere i (original index: its row, list and state are
// read without a permutation lookup) on its slot row, staged in shared
// memory (row[s * RS]); returns the bitmask of occupied slots.
template <int LM>
__device__ __forceinline__ uint32_t search_sphere(const StepArgs &A, uint32_t i, uint32_t *row,
                                                  uint16_t *keys, int RS)
{
    const DevBox &B = A.boxes[box_index(A, i)];
    const double4 xa = A.x[i];
    const uint4 *grow = reinterpret_cast<const uint4 *>(A.slots + (size_t)i * NC);
    uint32_t occ = 0;
#pragma unroll
    for (int q = 0; q < NC / 4; ++q) {
        const uint4 w = grow[q];
        row[(4 * q + 0) * RS] = w.x;
        row[(4 * q + 1) * RS] = w.y;
        row[(4 * q + 2) * RS] = w.z;
        row[(4 * q + 3) * RS] = w.w;
        occ |= (w.x != EMPTY ? 1u : 0u) << (4 * q);
        occ |= (w.y != EMPTY ? 1u : 0u) << (4 * q + 1);
        occ |= (w.z != EMPTY ? 1u : 0u) << (4 * q + 2);
        occ |= (w.w != EMPTY ? 1u : 0u) << (4 * q + 3);
    }
    if (A.tape_rows_pre) {
        uint4 *tp = reinterpret_cast<uint4 *>(A.tape_rows_pre + (size_t)i * NC);
#pragma unroll
        for (int q = 0; q < NC / 4; ++q) tp[q] = grow[q];
    }
    int g[3];
    g[0] = (int)floor((xa.x - B.origo[0]) / (B.L[0] / B.num[0]));
    g[1] = (int)floor((xa.y - B.origo[1]) / (B.L[1] / B.num[1]));
    g[2] = (int)floor((xa.z - B.origo[2]) / (B.L[2] / B.num[2]));
    const uint32_t *lst = A.vlist ? A.vlist + (size_t)i * VL_MAX : nullptr;
    const uint32_t vc = lst ? A.vcount[i] : (uint32_t)VL_MAX + 1u;
    // the first entries are read together with the count (the list row
    // holds VL_MAX >= 2 KB entries; those at or past the count go unused)
    uint32_t nb[KB];
#pragma unroll
    for (int j = 0; j < KB; ++j) nb[j] = lst ? lst[j] : 0u;
    bool dirty = false;
    if (vc <= (uint32_t)VL_MAX) {
        // Partners already in the row keep their slots whatever the order,
        // so when the row cannot overflow only the other entries are
        // tested and inserted (in visit order, each into the highest free
        // slot); otherwise every entry goes through the reference's
        // counting of touching entries.
        const uint32_t occ0 = occ;
        int nk = 0;
        for (uint32_t k0 = 0; k0 < vc; k0 += KB) {
            uint32_t bo[KB];
            int srow[KB];
#pragma unroll
            for (int j = 0; j < KB; ++j) {
                bo[j] = nb[j];
                srow[j] = -1;
                if (k0 + j < vc)
                    for (uint32_t m = occ0; m; m &= m - 1u) {
                        const int sl = __ffs(m) - 1;
                        if ((row[sl * RS] & ID_MASK) == bo[j]) {
                            srow[j] = sl;
                            break;
                        }
                    }
            }
            if (k0 + KB < vc) {
#pragma unroll
                for (int j = 0; j < KB; ++j) nb[j] = lst[k0 + KB + j];
            }
            uint16_t kb[KB];
            list_keys_batch<LM, true>(A, B, xa, g, bo, k0, vc, kb, srow, row, RS, &dirty);
#pragma unroll
            for (int j = 0; j < KB; ++j) {
                const uint16_t key = kb[j];
                if (key == NO_KEY) continue;
                int q = nk;
                while (q > 0 && keys[(q - 1) * RS] > key) {
                    keys[q * RS] = keys[(q - 1) * RS];
                    --q;
                }
                keys[q * RS] = key;
                ++nk;
            }
        }
        if (__popc(occ0) + nk > NC) {
            // the row may overflow: all touching entries, counted in order
            nk = 0;
            const int none[KB] = {-1, -1, -1, -1};
            for (uint32_t k0 = 0; k0 < vc; k0 += KB) {
                uint32_t bo[KB];
#pragma unroll
                for (int j = 0; j < KB; ++j) bo[j] = k0 + j < vc ? lst[k0 + j] : 0u;
                uint16_t kb[KB];
                list_keys_batch<LM, false>(A, B, xa, g, bo, k0, vc, kb, none, row, RS, &dirty);
#pragma unroll
                for (int j = 0; j < KB; ++j) {
                    const uint16_t key = kb[j];
                    if (key == NO_KEY) continue;
                    int q = nk;
                    while (q > 0 && keys[(q - 1) * RS] > key) {
                        keys[q * RS] = keys[(q - 1) * RS];
                        --q;
                    }
                    keys[q * RS] = key;
                    ++nk;
                }
            }
        }
        if (insert_keys(A, keys, nk, RS, lst, row, RS, occ)) dirty = true;
    } else {
        const uint32_t a = A.rank[i];   // the cell search walks the sorted copies
        dirty = search_cells<LM>(A, B, a, xa, g, A.xf[a], row, RS);
        occ = occupancy(row, RS);
    }
    if (A.tape_rows_post) {
        const double4 *hist = A.hist + (size_t)i * NC;
        for (int s = 0; s < NC; ++s) {
            const uint32_t w = row[s * RS];
            A.tape_rows_post[(size_t)i * NC + s] = w;
            if (w != EMPTY) A.tape_hist[(size_t)i * NC + s] = hist[s];
        }
    }
    if (dirty) {
        uint4 *wrow = reinterpret_cast<uint4 *>(A.slots + (size_t)i * NC);
#pragma unroll
        for (int q = 0; q < NC / 4; ++q)
            wrow[q] = make_uint4(row[(4 * q) * RS], row[(4 * q + 1) * RS], row[(4 * q + 2) * RS],
                                 row[(4 * q + 3) * RS]);
    }
    return occ;
}

template <int LM>
__global__ void __launch_bounds__(SEARCH_THREADS) k_search(StepArgs A)
{
    __shared__ uint32_t s_row[NC * SEARCH_THREADS];
    __shared__ uint16_t s_keys[VL_MAX * SEARCH_THREADS];
    grid_dependency_wait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const int RS = SEARCH_THREADS;
    uint32_t *row = s_row + threadIdx.x;
    const uint32_t occ =
        i < A.ntot ? search_sphere<LM>(A, i, row, s_keys + threadIdx.x, RS) : 0u;
    // the warp's live contacts, sphere after sphere, each in slot order,
    // written contiguously from the start of the warp's region
    const uint32_t nl = __popc(occ);
    uint32_t incl = nl;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (i >= A.ntot) return;
    uint2 *ent = A.lent + (size_t)(i - lane) * NC + (incl - nl);
    uint32_t q = 0;
    for (uint32_t m = occ; m; m &= m - 1u) {
        const int sl = __ffs(m) - 1;
        // slot word (partner's original id | image code), i | slot << 27
        ent[q++] = make_uint2(row[sl * RS], i | ((uint32_t)sl << 27));
    }
    A.nlive[i] = nl;
}

// One warp-round of contact records in shared memory, field by field
// (consecutive lanes hit consecutive words).
struct RecSlab {
    double f[10][CONTACT_THREADS];   // F.x F.y F.z T.x T.y T.z ev0 ev1 es p
    int32_t n[CONTACT_THREADS];      // (nev + 1) | nes << 4
};

__device__ __forceinline__ void put_rec(RecSlab &S, int t, const ContactRec &r)
{
    S.f[0][t] = r.F.x;
    S.f[1][t] = r.F.y;
    S.f[2][t] = r.F.z;
    S.f[3][t] = r.T.x;
    S.f[4][t] = r.T.y;
    S.f[5][t] = r.T.z;
    S.f[6][t] = r.ev0;
    S.f[7][t] = r.ev1;
    S.f[8][t] = r.es;
    S.f[9][t] = r.p;
    S.n[t] = (r.nev + 1) | (r.nes << 4);
}

__device__ __forceinline__ ContactRec get_rec(const RecSlab &S, int t)
{
    ContactRec r;
    r.F = mk(S.f[0][t], S.f[1][t], S.f[2][t]);
    r.T = mk(S.f[3][t], S.f[4][t], S.f[5][t]);
    r.ev0 = S.f[6][t];
    r.ev1 = S.f[7][t];
    r.es = S.f[8][t];
    r.p = S.f[9][t];
    const int32_t n = S.n[t];
    r.nev = (n & 15) - 1;
    r.nes = n >> 4;
    return r;
}

// One warp per 32 consecutive spheres (original indexes), its lanes dealt
// the warp's live contacts in order: round r computes contacts 32r .. 32r +
// 31 of the warp's list (the spheres' live lists one after the other), so a
// lane is idle only in the last round.  Each lane then adds, in slot order,
// the round's records of its own sphere.
template <int LM, bool MIXED>
__global__ void __launch_bounds__(CONTACT_THREADS, 6) k_contacts(StepArgs A)
{
    __shared__ RecSlab S;
    grid_dependency_wait();
    const uint32_t lane = threadIdx.x & 31u;
    const int wbase = (int)(threadIdx.x & ~31u);
    const uint32_t i_own = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i0 = i_own - lane;
    const bool valid = i_own < A.ntot;
    const uint32_t nl_own = valid ? A.nlive[i_own] : 0u;
    // inclusive prefix sum of the live counts over the warp
    uint32_t incl = nl_own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    const uint32_t excl = incl - nl_own;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    Acc acc;
    acc.F = mk(0.0, 0.0, 0.0);
    acc.T = mk(0.0, 0.0, 0.0);
    acc.es_dot = 0.0;
    acc.ev_dot = 0.0;
    acc.p = 0.0;
    const uint2 *ent = A.lent + (size_t)i0 * NC;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t f = base + lane;
        ContactRec r;
        r.F = mk(0.0, 0.0, 0.0);
        r.T = mk(0.0, 0.0, 0.0);
        r.ev0 = r.ev1 = r.es = r.p = 0.0;
        r.nev = -1;   // nothing to add unless a live contact is computed
        r.nes = 0;
        if (f < total) {
            const uint2 e = ent[f];
            const uint32_t i = e.y & SPLIT_ID_MASK;
            const int s = (int)(e.y >> 27);
            const uint32_t w = e.x;
            const DevBox &B = A.boxes[box_index(A, i)];
            const SphParams &P = B.P;
            const double dt = B.dt;
            const uint32_t cm = P.contactmodel;
            // the sphere's own data in original order (the step's start
            // state until k_finish), like its partner's
            const double4 xa = A.x[i];
            const double radius_a = xa.w;
            const d3 vel_a = xyz(A.vel[i]);
            const d3 angvel_a = xyz(A.angvel[i]);
            uint32_t *slots = A.slots + (size_t)i * NC;
            double4 *hist = A.hist + (size_t)i * NC;
            const uint32_t bo = w & ID_MASK;   // partner's original id
            int sx, sy;
            decode_shift(w >> CODE_SHIFT, sx, sy);
            const d3 dm = shift_vec(B, sx, sy);
            // the partner's data (original order: A.x, A.vel, A.angvel hold
            // the step's start state until k_finish) and the history are
            // loaded together
            const double4 xb = A.x[bo];
            const double4 vb4 = A.vel[bo];
            const double4 wb4 = A.angvel[bo];
            const double4 h4 = hist[s];
            const d3 x_ab = mk(xa.x - xb.x + dm.x, xa.y - xb.y + dm.y, xa.z - xb.z + dm.z);
            const double x_ab_length = vlen<LM>(x_ab);
            const double delta_n = x_ab_length - (radius_a + xb.w);
            if (delta_n < 0.0) {
                r.nev = 0;
                const d3 vel_b = xyz(vb4);
                const d3 h0 = xyz(h4);
                d3 nd;
                if (MIXED) {
                    const MixedPair mp = mixed_pair(x_ab, x_ab_length, delta_n, vel_a, vel_b,
                                                    tof(angvel_a), xyzf(wb4), radius_a, xb.w);
                    if (cm == 2) nd = contact_linear_mixed(P, dt, r, mp, h0);
                    else nd = contact_hertz_mixed(P, dt, r, mp, h0);
                } else {
                    const d3 angvel_b = xyz(wb4);
                    if (cm == 2)
                        nd = contact_linear<LM>(P, dt, r, vel_a, vel_b, angvel_a, angvel_b,
                                                radius_a, xb.w, x_ab, x_ab_length, delta_n, h0);
                    else
                        nd = contact_hertz<LM>(P, dt, r, vel_a, vel_b, angvel_a, angvel_b,
                                               radius_a, xb.w, x_ab, x_ab_length, delta_n, h0);
                }
                hist[s] = make_double4(nd.x, nd.y, nd.z, 0.0);
            } else {
                slots[s] = EMPTY;
                hist[s] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
        }
        put_rec(S, (int)threadIdx.x, r);
        __syncwarp();
        // this lane's sphere: its entries of this round, in slot order
        const uint32_t lo = max(excl, base), hi = min(incl, base + 32u);
        for (uint32_t e = lo; e < hi; ++e) {
            const ContactRec o = get_rec(S, wbase + (int)(e - base));
            if (o.nev >= 0) replay(acc, o);
        }
        __syncwarp();
    }
    if (valid) A.csum[i_own] = acc;
}

template <int LM>
__global__ void __launch_bounds__(FINISH_THREADS, 4) k_finish(StepArgs A)
{
    // original order: every access of this kernel is to the sphere's own
    // entries, so they are all coalesced (x, vel, angvel still hold the
    // state at the start of the step: only this thread rewrites them)
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const DevBox &B = A.boxes[box_index(A, i)];
    const double4 xa = A.x[i];
    const double4 va4 = A.vel[i];
    const double4 wa4 = A.angvel[i];
    Acc acc;
    acc.F = mk(0.0, 0.0, 0.0);
    acc.T = mk(0.0, 0.0, 0.0);
    acc.es_dot = 0.0;
    acc.ev_dot = 0.0;
    acc.p = 0.0;
    acc = A.csum[i];   // the contacts' sums, added in slot order by k_contacts
    const double w0_force = walls_and_bonds<LM>(A, B, i, xa, xyz(va4), xyz(wa4), acc);
    store_sums(A, B, i, acc, w0_force);
    integrate_particle(A, B, i, xa, va4, wa4, acc.F, acc.T);
}

// Launch variants of k_interact (INTERACT_VARIANTS): the minimum resident
// blocks per SM given to the compiler (register budget 255, 128 and 80 per
// thread), chosen per handle by sph_autotune.  The arithmetic is the same
// in every variant.

template <bool MIXED, int LM, bool FUSED>
inline void launch_interact_lm(const StepArgs &A, cudaStream_t st, unsigned grid, int variant)
{
    if (variant == 0) k_interact<LM, FUSED, MIXED, 1><<<grid, INTERACT_THREADS, 0, st>>>(A);
    else if (variant == 2) k_interact<LM, FUSED, MIXED, 6><<<grid, INTERACT_THREADS, 0, st>>>(A);
    else k_interact<LM, FUSED, MIXED, 4><<<grid, INTERACT_THREADS, 0, st>>>(A);
}

template <bool MIXED>
inline void launch_contacts(const StepArgs &A, cudaStream_t st, unsigned grid, int lm, bool pdl)
{
    if (lm == SPH_LEN_FP64) launch_k(pdl, k_contacts<SPH_LEN_FP64, MIXED>, grid, CONTACT_THREADS, st, A);
    else launch_k(pdl, k_contacts<SPH_LEN_REFERENCE, MIXED>, grid, CONTACT_THREADS, st, A);
}

template <bool MIXED>
inline void launch_interact(const StepArgs &A, cudaStream_t st, unsigned grid, bool fused, int lm,
                            int variant)
{
    if (fused) {
        if (lm == SPH_LEN_FP64) launch_interact_lm<MIXED, SPH_LEN_FP64, true>(A, st, grid, variant);
        else launch_interact_lm<MIXED, SPH_LEN_REFERENCE, true>(A, st, grid, variant);
    } else {
        if (lm == SPH_LEN_FP64) launch_interact_lm<MIXED, SPH_LEN_FP64, false>(A, st, grid, variant);
        else launch_interact_lm<MIXED, SPH_LEN_REFERENCE, false>(A, st, grid, variant);
    }
}

}  // namespace sph
