// sph_kernels.cu -- FP64 kernels of the B200 DEM step.
//
// Compiled with -fmad=false: together with the operand order kept in
// sph_device.cuh this makes the FP64 step reproduce the reference's
// arithmetic bit for bit.
//
// One step (see launch_step):
//   memset cell_count
//   k_hash          cell id + atomic slot within the cell  (sorting.cuh:7-51)
//   scan (3)        exclusive scan of cell counts -> cell_off
//   k_scatter       perm[cell_off[c] + slot] = i
//   k_cellsort      order each cell by original index: the stable order of
//                   thrust::sort_by_key (device.cu:1075)
//   k_reorder       sorted copies of x, vel, angvel + rank  (sorting.cuh:56-132)
//   k_bonds         bond forces into per-bond buffers       (cohesion.cuh:8-233)
//   k_interact      topology + interact + walls + bond gather + integrate
//                   (contactsearch.cuh:329-726, integration.cuh:14-305)
//   k_block_sums    per-256 partial sums of the wall force  (integration.cuh:309-341)
//   k_box_step      integrateWalls + time/grid/velocity-step state
//                   (integration.cuh:344-450, device.cu:1050, 2455-2462, 2536)
// Boxes with a shear-stress top wall (wmode 3) need a global sum of forces
// between interact and integrate (device.cu:2427-2452); they use the
// unfused kernels k_interact<FUSED=false>, k_shear_stress, k_block_sums,
// k_tau_final and k_integrate.
#include <cstdint>
#include <cstdio>

#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

static inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------ sorting

// sorting.cuh:7-51 calcParticleCellID + device.cu:241-276 position checks
__global__ void k_hash(StepArgs A)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const DevBox &B = A.boxes[A.box_of[i]];
    const double4 x = A.x[i];
    const double xv[3] = {x.x, x.y, x.z};
    uint32_t c[3];
    bool nonfinite = !isfinite(x.x) || !isfinite(x.y) || !isfinite(x.z);
    bool outside = false;
    for (int d = 0; d < 3; ++d) {
        double f = floor((xv[d] - B.origo[d]) / (B.L[d] / B.num[d]));
        if (!(f >= 0.0)) { outside = true; f = 0.0; }
        if (f >= (double)B.num[d]) { outside = true; f = (double)(B.num[d] - 1); }
        c[d] = (uint32_t)f;
    }
    if (nonfinite) raise_flag(A.err, SPH_ERR_NAN);
    else if (outside || x.x > B.L[0] || x.y > B.L[1] || x.z > B.L[2])
        raise_flag(A.err, SPH_ERR_OUT_OF_GRID);
    const uint32_t cell = B.cell_base + (c[2] * B.num[1]) * B.num[0] + c[1] * B.num[0] + c[0];
    A.cell_id[i] = cell;
    A.local_off[i] = atomicAdd(&A.cell_count[cell], 1u);
}

// Exclusive scan of n uint32 (3 launches): per-block totals, a one-block
// scan of the totals, then per-block scans with the block offset.
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *smem,
                                                         uint32_t *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? smem[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        smem[lane] = wi - w;
        if (lane == 31) smem[32] = wi;
    }
    __syncthreads();
    const uint32_t r = smem[warp] + incl - v;
    *total = smem[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t *in, uint64_t n,
                                                              uint32_t *bsum)
{
    __shared__ uint32_t smem[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_exclusive_scan(s, smem, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_top(uint32_t *bsum, uint32_t nb)
{
    __shared__ uint32_t smem[33];
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const uint32_t idx = threadIdx.x * SCAN_ITEMS + k;
        v[k] = idx < nb ? bsum[idx] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t off = block_exclusive_scan(s, smem, &total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const uint32_t idx = threadIdx.x * SCAN_ITEMS + k;
        if (idx < nb) bsum[idx] = off;
        off += v[k];
    }
    if (threadIdx.x == 0) bsum[nb] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const uint32_t *in, uint64_t n,
                                                            const uint32_t *bsum, uint32_t nb,
                                                            uint32_t *out)
{
    __shared__ uint32_t smem[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t off = block_exclusive_scan(s, smem, &total) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = bsum[nb];
}

__global__ void k_scatter(StepArgs A)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    A.perm[A.cell_off[A.cell_id[i]] + A.local_off[i]] = i;
}

// Within each cell, order particles by original index (insertion sort of
// the short segment); the result is the stable sort by cell id.
__global__ void k_cellsort(StepArgs A)
{
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= A.ncells) return;
    const uint32_t s = A.cell_off[c], e = A.cell_off[c + 1];
    for (uint32_t j = s + 1; j < e; ++j) {
        const uint32_t v = A.perm[j];
        uint32_t k = j;
        while (k > s) {
            const uint32_t u = A.perm[k - 1];
            if (u <= v) break;
            A.perm[k] = u;
            --k;
        }
        A.perm[k] = v;
    }
}

// sorting.cuh:118-130: sorted copies of x, vel, angvel; rank = inverse of perm
__global__ void k_reorder(StepArgs A)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= A.ntot) return;
    const uint32_t i = A.perm[j];
    A.xs[j] = A.x[i];
    A.vs[j] = A.vel[i];
    A.ws[j] = A.angvel[i];
    A.rank[i] = j;
}

// -------------------------------------------------------------------- bonds

// cohesion.cuh:8-233 bondsLinear.  Forces go to per-bond buffers (w = 1
// when applied this step) and are added to the particles in ascending bond
// order by k_interact, instead of the reference's racing scatter-add.  A
// bond broken during the run stays broken (the reference re-activates it
// when nb0 < np, cohesion.cuh:30 and :205).
template <int LM>
__global__ void k_bonds(StepArgs A)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= A.nbonds) return;
    const DevBox &B = A.boxes[A.bond_box[k]];
    const SphParams &P = B.P;
    const double dt = B.dt;
    const uint2 bd = A.bonds[k];
    A.bf[k] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (!(bd.x < B.np) || A.bbroken[k]) return;
    if (!(bd.y < B.np)) { raise_flag(A.err, SPH_ERR_INPUT); return; }
    const uint32_t gi = B.p_base + bd.x, gj = B.p_base + bd.y;
    const double4 d4 = A.bdelta[k], o4 = A.bomega[k];
    d3 delta0_t = xyz(d4);
    const double delta0_n = d4.w;
    d3 omega0_t = xyz(o4);
    const double omega0_n = o4.w;
    const double4 x_i = A.x[gi], x_j = A.x[gj];
    const d3 vel_i = xyz(A.vel[gi]), vel_j = xyz(A.vel[gj]);
    const d3 angvel_i = xyz(A.angvel[gi]), angvel_j = xyz(A.angvel[gj]);
    const double R_bar = P.lambda_bar * fmin(x_i.w, x_j.w);
    const double Ar = PI * R_bar * R_bar;
    const double I = 0.25 * PI * R_bar * R_bar * R_bar * R_bar;
    const double J = I * 2.0;
    const d3 x = mk(x_i.x - x_j.x, x_i.y - x_j.y, x_i.z - x_j.z);
    const double x_length = vlen<LM>(x);
    const double overlap = fmin(0.0, x_length - (x_i.w + x_j.w));
    const d3 n = divs(x, x_length);
    delta0_t = vsub(delta0_t, muls(n, dot(n, delta0_t)));
    const d3 ddelta = muls(vadd(vadd(vsub(vel_i, vel_j), smul(x_i.w + overlap / 2.0, cross(n, angvel_i))),
                                smul(x_j.w + overlap / 2.0, cross(n, angvel_j))),
                           dt);
    const double ddelta_n = -dot(ddelta, n);
    const double delta_n = delta0_n + ddelta_n;
    const d3 ddelta_t = vsub(ddelta, muls(n, dot(n, ddelta)));
    const d3 delta_t = vadd(delta0_t, ddelta_t);
    const d3 f_n = smul(P.k_n * Ar * delta_n + P.gamma_n * ddelta_n / dt, n);
    const d3 f_t = vsub(smul(-P.k_t * Ar, delta_t), divs(smul(P.gamma_t, ddelta_t), dt));
    const d3 f = vadd(f_n, f_t);
    const d3 nn = vneg(n);
    omega0_t = vsub(omega0_t, muls(nn, dot(omega0_t, nn)));
    const d3 domega = muls(vsub(angvel_j, angvel_i), dt);
    const double domega_n = dot(domega, nn);
    const double omega_n = omega0_n + domega_n;
    const d3 domega_t = vsub(domega, smul(domega_n, nn));
    const d3 omega_t = vadd(omega0_t, domega_t);
    const d3 t_n = smul(-P.k_t * J * omega_n, nn);
    const d3 t_t = smul(-P.k_n * I, omega_t);
    const d3 t_j = vadd(t_n, t_t);
    const double sigma_max = vlen<LM>(f_n) / Ar + vlen<LM>(t_t) * R_bar / I;
    const double tau_max = vlen<LM>(f_t) / Ar + vlen<LM>(t_n) * R_bar / J;
    if (sigma_max >= P.sigma_b || tau_max >= P.tau_b) {
        A.bonds[k].x = B.nb0;
        A.bbroken[k] = 1;
        return;
    }
    A.bdelta[k] = make_double4(delta_t.x, delta_t.y, delta_t.z, delta_n);
    A.bomega[k] = make_double4(omega_t.x, omega_t.y, omega_t.z, omega_n);
    A.bf[k] = make_double4(f.x, f.y, f.z, 1.0);
    A.bt[k] = make_double4(t_j.x, t_j.y, t_j.z, 0.0);
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

// ------------------------------------------------------------------ interact

constexpr int INTERACT_THREADS = 128;

// Fused topology + interact + walls + bond gather (+ integrate when FUSED)
// for the particle at sorted position a.  Neighbour data is read from the
// sorted copies only, so writing the particle's new state in place is safe.
// The particle's contact row is staged in shared memory (slot-major, one
// column per thread); only live slots are processed, empty slots keep a
// zero tangential history by construction.
template <int LM, bool FUSED>
__global__ void __launch_bounds__(INTERACT_THREADS) k_interact(StepArgs A)
{
    __shared__ uint32_t s_row[NC * INTERACT_THREADS];
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ntot) return;
    uint32_t *row = s_row + threadIdx.x;
    const int RS = INTERACT_THREADS;
    const uint32_t i = A.perm[a];
    const DevBox &B = A.boxes[A.box_of[i]];
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

    if (cm == 2 || cm == 3) {
        // ---- topology: contactsearch.cuh:329-371 and :194-322
        int nc = 0;
        for (int dz = -1; dz < 2; ++dz)
            for (int dy = -1; dy < 2; ++dy)
                for (int dx = -1; dx < 2; ++dx) {
                    int tx = g[0] + dx, ty = g[1] + dy, sx, sy;
                    const int tz = g[2] + dz;
                    if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                    const d3 dm = shift_vec(B, sx, sy);
                    const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                    const uint32_t start = A.cell_off[cell], end = A.cell_off[cell + 1];
                    for (uint32_t b = start; b < end; ++b) {
                        if (b == a) continue;
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
                                row[cpos * RS] = b_orig | (shift_code(sx, sy) << CODE_SHIFT);
                                dirty = true;
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

        // ---- interact over the contact row: contactsearch.cuh:484-559
        double4 *hist = A.hist + (size_t)i * NC;
        for (int s = 0; s < NC; ++s) {
            const uint32_t w = row[s * RS];
            if (w == EMPTY) continue;
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
                const d3 angvel_b = xyz(A.ws[bs]);
                const d3 h0 = xyz(hist[s]);
                d3 nd;
                if (cm == 2)
                    nd = contact_linear<LM>(P, dt, acc, vel_a, vel_b, angvel_a, angvel_b, radius_a,
                                            xb.w, x_ab, x_ab_length, delta_n, h0);
                else
                    nd = contact_hertz<LM>(P, dt, acc, vel_a, vel_b, angvel_a, angvel_b, radius_a,
                                           xb.w, x_ab, x_ab_length, delta_n, h0);
                hist[s] = make_double4(nd.x, nd.y, nd.z, 0.0);
            } else {
                row[s * RS] = EMPTY;
                dirty = true;
                hist[s] = make_double4(0.0, 0.0, 0.0, 0.0);
            }
        }
    } else if (cm == 1) {
        // ---- contact model 1: contactsearch.cuh:564-598 and :91-186
        for (int dz = -1; dz < 2; ++dz)
            for (int dy = -1; dy < 2; ++dy)
                for (int dx = -1; dx < 2; ++dx) {
                    int tx = g[0] + dx, ty = g[1] + dy, sx, sy;
                    const int tz = g[2] + dz;
                    if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                    const d3 dm = shift_vec(B, sx, sy);
                    const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                    const uint32_t start = A.cell_off[cell], end = A.cell_off[cell + 1];
                    for (uint32_t b = start; b < end; ++b) {
                        if (b == a) continue;
                        const double4 xb = A.xs[b];
                        const double kappa = P.kappa;
                        d3 x_ab = mk(xa.x - xb.x, xa.y - xb.y, xa.z - xb.z);
                        x_ab = vadd(x_ab, dm);
                        const double x_ab_length = vlen<LM>(x_ab);
                        const double delta_ab = x_ab_length - (radius_a + xb.w);
                        if (delta_ab < 0.0) {
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

    // ---- walls: contactsearch.cuh:428-465 and :602-701
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

    if (dirty) {
        uint4 *wrow = reinterpret_cast<uint4 *>(A.slots + (size_t)i * NC);
#pragma unroll
        for (int q = 0; q < NC / 4; ++q)
            wrow[q] = make_uint4(row[(4 * q) * RS], row[(4 * q + 1) * RS], row[(4 * q + 2) * RS],
                                 row[(4 * q + 3) * RS]);
    }

    // ---- contactsearch.cuh:707-724
    A.force[i] = make_double4(acc.F.x, acc.F.y, acc.F.z, 0.0);
    A.torque[i] = make_double4(acc.T.x, acc.T.y, acc.T.z, 0.0);
    A.es_dot[i] = acc.es_dot;
    A.ev_dot[i] = acc.ev_dot;
    A.es[i] += acc.es_dot * dt;
    A.ev[i] += acc.ev_dot * dt;
    A.p[i] = acc.p;
    if (nw > 0) A.wf_pp[i] = w0_force;

    if (FUSED) integrate_particle(A, B, i, xa, va4, wa4, acc.F, acc.T);
}

// Unfused integrate (boxes with a shear-stress wall).
__global__ void k_integrate(StepArgs A)
{
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ntot) return;
    const uint32_t i = A.perm[a];
    const DevBox &B = A.boxes[A.box_of[i]];
    const double4 f = A.force[i], t = A.torque[i];
    integrate_particle(A, B, i, A.xs[a], A.vs[a], A.ws[a], xyz(f), xyz(t));
}

// integration.cuh:457-484 findShearStressOnFixedMovingParticles
__global__ void k_shear_stress(StepArgs A)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const DevBox &B = A.boxes[A.box_of[i]];
    if (!(B.nw > 0 && B.wmode[0] == 3)) return;
    const double z = A.x[i].z;
    const double fixvel = A.vel[i].w;
    const double force_x = A.force[i].x;
    double f_x = 0.0;
    if (fixvel > 0.0 && z > B.L[2] * 0.5) f_x = force_x;
    A.tau_pp[i] = f_x / (B.L[0] * B.L[1]);
}

// integration.cuh:309-341 summation: one 256-thread block per partial, the
// same shared-memory tree as the reference.
__global__ void __launch_bounds__(256) k_block_sums(StepArgs A, const double *in, double *out,
                                                    int only_wmode3)
{
    __shared__ double cache[256];
    const uint32_t part = blockIdx.x;
    const DevBox &B = A.boxes[A.part_owner[part]];
    const bool active = B.nw > 0 && (!only_wmode3 || B.wmode[0] == 3);
    const uint32_t local = (part - B.part_base) * 256u + threadIdx.x;
    double temp = 0.0;
    if (active && local < B.np) temp += in[B.p_base + local];
    cache[threadIdx.x] = temp;
    __syncthreads();
    for (unsigned s = 128; s != 0; s /= 2) {
        if (threadIdx.x < s) cache[threadIdx.x] += cache[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[part] = cache[0];
}

// Sum of the shear-stress partials per box (integration.cuh:65-68), once
// per box instead of once per particle.
__global__ void k_tau_final(StepArgs A)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= A.nboxes) return;
    DevBox &B = A.boxes[b];
    double tau = 0.0;
    if (B.nw > 0 && B.wmode[0] == 3)
        for (uint32_t k = 0; k < B.nblocks; ++k) tau += A.tau_partial[B.part_base + k];
    B.tau_eff_x = tau;
}

// integration.cuh:344-450 integrateWalls, then the loop bookkeeping of
// device.cu:2536-2538, the adaptive grid of device.cu:1050 and the
// velocity-step state of device.cu:2455-2462 for the next step.
__global__ void k_box_step(StepArgs A)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= A.nboxes) return;
    DevBox &B = A.boxes[b];
    const double dt = B.dt;
    if (B.np > 0) {
        for (uint32_t w = 0; w < B.nw; ++w) {
            const int wmode = B.wmode[w];
            if (wmode == 0) continue;
            const double acc0 = B.iter == 0 ? 0.0 : B.wacc[w];
            double fsum = 0.0;
            for (uint32_t k = 0; k < B.nblocks; ++k) fsum += A.wall_partial[B.part_base + k];
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

// ------------------------------------------------------------- scene packing

// One Jacobi sweep of overlap removal (scene preparation, not part of the
// step): every overlapping pair pushes both spheres apart along the centre
// line by `alpha` times half the overlap; the floor (z = origo) and the
// ceiling z_top push spheres back inside; periodic images count as
// neighbours.  The displacement goes to A.force (free before a run) and is
// applied by k_relax_apply.  The largest overlap seen is atomically max-ed
// into *max_ov (as the bit pattern of a non-negative double).
__global__ void k_relax(StepArgs A, double alpha, double z_top, unsigned long long *max_ov)
{
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= A.ntot) return;
    const uint32_t i = A.perm[a];
    const DevBox &B = A.boxes[A.box_of[i]];
    const double4 xa = A.xs[a];
    const int nx = (int)B.num[0], ny = (int)B.num[1];
    int g[3];
    g[0] = (int)floor((xa.x - B.origo[0]) / (B.L[0] / B.num[0]));
    g[1] = (int)floor((xa.y - B.origo[1]) / (B.L[1] / B.num[1]));
    g[2] = (int)floor((xa.z - B.origo[2]) / (B.L[2] / B.num[2]));
    double dx = 0.0, dy = 0.0, dz = 0.0, worst = 0.0;
    for (int oz = -1; oz < 2; ++oz)
        for (int oy = -1; oy < 2; ++oy)
            for (int ox = -1; ox < 2; ++ox) {
                int tx = g[0] + ox, ty = g[1] + oy, sx, sy;
                if (!image_cell(B, tx, ty, g[2] + oz, sx, sy)) continue;
                const d3 dm = shift_vec(B, sx, sy);
                const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * (g[2] + oz));
                for (uint32_t b = A.cell_off[cell]; b < A.cell_off[cell + 1]; ++b) {
                    if (b == a) continue;
                    const double4 xb = A.xs[b];
                    const double rx = xa.x - xb.x + dm.x, ry = xa.y - xb.y + dm.y, rz = xa.z - xb.z + dm.z;
                    const double len = sqrt(rx * rx + ry * ry + rz * rz);
                    const double ov = xa.w + xb.w - len;
                    if (ov > 0.0 && len > 0.0) {
                        const double s = 0.5 * alpha * ov / len;
                        dx += s * rx;
                        dy += s * ry;
                        dz += s * rz;
                        worst = fmax(worst, ov);
                    }
                }
            }
    const double below = (B.origo[2] + xa.w) - xa.z;
    if (below > 0.0) { dz += below; worst = fmax(worst, below); }
    const double above = xa.z + xa.w - z_top;
    if (above > 0.0) { dz -= above; worst = fmax(worst, above); }
    A.force[i] = make_double4(dx, dy, dz, 0.0);
    atomicMax(max_ov, (unsigned long long)__double_as_longlong(worst));
}

__global__ void k_relax_apply(StepArgs A)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const DevBox &B = A.boxes[A.box_of[i]];
    double4 x = A.x[i];
    const double4 d = A.force[i];
    x.x += d.x;
    x.y += d.y;
    x.z += d.z;
    if (B.periodic == 1 || B.periodic == 2) {
        if (x.x < B.origo[0]) x.x += B.L[0] - B.origo[0];
        if (x.x >= B.L[0]) x.x -= B.L[0] - B.origo[0];
    }
    if (B.periodic == 1) {
        if (x.y < B.origo[1]) x.y += B.L[1] - B.origo[1];
        if (x.y >= B.L[1]) x.y -= B.L[1] - B.origo[1];
    }
    x.x = fmin(fmax(x.x, B.origo[0]), B.L[0] * (1.0 - 1e-12));
    x.y = fmin(fmax(x.y, B.origo[1]), B.L[1] * (1.0 - 1e-12));
    x.z = fmin(fmax(x.z, B.origo[2]), B.L[2] * (1.0 - 1e-12));
    A.x[i] = x;
}

int relax_sweep(const StepArgs &A, cudaStream_t st, double alpha, double z_top,
                unsigned long long *d_max, uint64_t *launches)
{
    cudaMemsetAsync(A.cell_count, 0, sizeof(uint32_t) * A.ncells, st);
    k_hash<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    const uint32_t nb = blocks_for(A.ncells, SCAN_TILE);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp);
    k_scan_top<<<1, SCAN_THREADS, 0, st>>>(A.scan_tmp, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp, nb, A.cell_off);
    k_scatter<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    k_cellsort<<<blocks_for(A.ncells, 256), 256, 0, st>>>(A);
    k_reorder<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st);
    k_relax<<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, alpha, z_top, d_max);
    k_relax_apply<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    if (launches) *launches += 10;
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

// Live directed contacts (non-empty slots), for the roofline byte count.
__global__ void k_count_live(const uint32_t *slots, uint64_t nslots, unsigned long long *count)
{
    unsigned long long c = 0;
    for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nslots;
         q += (uint64_t)gridDim.x * blockDim.x)
        c += slots[q] != EMPTY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

int count_live_slots(const StepArgs &A, cudaStream_t st, unsigned long long *d_count,
                     uint64_t *launches)
{
    cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
    k_count_live<<<4 * 148, 256, 0, st>>>(A.slots, (uint64_t)A.ntot * NC, d_count);
    if (launches) *launches += 1;
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

// ------------------------------------------------------------------ launch

static inline void mark(Prof *prof, cudaStream_t st, const char *name)
{
    if (!prof || prof->n >= Prof::MAX) return;
    prof->name[prof->n] = name;
    cudaEventRecord(prof->ev[prof->n + 1], st);
    prof->n++;
}

int launch_step(const StepArgs &A, const StepConfig &cfg, cudaStream_t st, uint64_t *launches,
                Prof *prof)
{
    uint64_t nl = 0;
    if (prof) {
        prof->n = 0;
        cudaEventRecord(prof->ev[0], st);
    }
    if (A.ntot > 0) {
        cudaMemsetAsync(A.cell_count, 0, sizeof(uint32_t) * A.ncells, st);
        k_hash<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
        mark(prof, st, "k_hash");
        const uint32_t nb = blocks_for(A.ncells, SCAN_TILE);
        k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp);
        k_scan_top<<<1, SCAN_THREADS, 0, st>>>(A.scan_tmp, nb);
        k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp, nb, A.cell_off);
        mark(prof, st, "k_scan(3)");
        k_scatter<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
        mark(prof, st, "k_scatter");
        k_cellsort<<<blocks_for(A.ncells, 256), 256, 0, st>>>(A);
        mark(prof, st, "k_cellsort");
        k_reorder<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
        mark(prof, st, "k_reorder");
        nl += 8;
        if (A.nbonds) {
            if (cfg.lenmode == SPH_LEN_FP64) k_bonds<SPH_LEN_FP64><<<blocks_for(A.nbonds, 128), 128, 0, st>>>(A);
            else k_bonds<SPH_LEN_REFERENCE><<<blocks_for(A.nbonds, 128), 128, 0, st>>>(A);
            mark(prof, st, "k_bonds");
            nl += 1;
        }
        const unsigned gi = blocks_for(A.ntot, INTERACT_THREADS);
        if (!cfg.unfused) {
            if (cfg.lenmode == SPH_LEN_FP64) k_interact<SPH_LEN_FP64, true><<<gi, INTERACT_THREADS, 0, st>>>(A);
            else k_interact<SPH_LEN_REFERENCE, true><<<gi, INTERACT_THREADS, 0, st>>>(A);
            mark(prof, st, "k_interact");
            nl += 1;
        } else {
            if (cfg.lenmode == SPH_LEN_FP64) k_interact<SPH_LEN_FP64, false><<<gi, INTERACT_THREADS, 0, st>>>(A);
            else k_interact<SPH_LEN_REFERENCE, false><<<gi, INTERACT_THREADS, 0, st>>>(A);
            mark(prof, st, "k_interact");
            k_shear_stress<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
            k_block_sums<<<A.npartials, 256, 0, st>>>(A, A.tau_pp, A.tau_partial, 1);
            k_tau_final<<<blocks_for(A.nboxes, 128), 128, 0, st>>>(A);
            mark(prof, st, "k_shear_stress+sums");
            k_integrate<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
            mark(prof, st, "k_integrate");
            nl += 5;
        }
        if (cfg.any_walls) {
            k_block_sums<<<A.npartials, 256, 0, st>>>(A, A.wf_pp, A.wall_partial, 0);
            mark(prof, st, "k_block_sums");
            nl += 1;
        }
    }
    k_box_step<<<blocks_for(A.nboxes, 128), 128, 0, st>>>(A);
    mark(prof, st, "k_box_step");
    nl += 1;
    if (launches) *launches += nl;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "sphere_b200: kernel launch failed: %s\n", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

}  // namespace sph
