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
//   k_scatter       unsorted[cell_off[c] + slot] = i
//   k_place         perm: each cell ordered by original index, the stable
//                   order of thrust::sort_by_key (device.cu:1075); sorted
//                   copies of x (+ vel, angvel, rank)  (sorting.cuh:56-132)
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
#include "sph_step.cuh"

namespace sph {

static inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------ sorting

// sorting.cuh:7-51 calcParticleCellID + device.cu:241-276 position checks
__global__ void k_hash(StepArgs A)
{
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i0 < A.ntot;
    const uint32_t i = valid ? i0 : 0u;
    const DevBox &B = A.boxes[A.nboxes == 1 ? 0u : A.box_of[i]];
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
    if (valid) {
        if (nonfinite) raise_flag(A.err, SPH_ERR_NAN);
        else if (outside || x.x > B.L[0] || x.y > B.L[1] || x.z > B.L[2])
            raise_flag(A.err, SPH_ERR_OUT_OF_GRID);
    }
    const uint32_t cell = B.cell_base + (c[2] * B.num[1]) * B.num[0] + c[1] * B.num[0] + c[0];
    // lanes of the warp in the same cell take consecutive slots with one
    // atomic (the slot order within a cell is free: k_place orders by index)
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(0xffffffffu, valid ? cell : 0xffffffffu);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (valid && (int)lane == leader) base = atomicAdd(&A.cell_count[cell], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!valid) return;
    A.cell_id[i] = cell;
    if (A.cellc) A.cellc[i] = pack_cell(c[0], c[1], c[2]);
    A.local_off[i] = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
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
    grid_dependency_wait();
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
    grid_dependency_wait();
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
    grid_dependency_wait();
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
    grid_dependency_wait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    A.unsorted[A.cell_off[A.cell_id[i]] + A.local_off[i]] = i;
}

// The stable sort by cell id and the sorted copies (sorting.cuh:118-130)
// in one pass over the particles in original order: particle i goes to
// cell_off[c] + (the number of particles of its cell with a smaller index),
// so each cell is ordered by original index.  rank = inverse of perm.
// ALL = false for the split step, which reads velocities and partners in
// original order and needs only the sorted positions and rank (the
// neighbour-list build and the cell-search fallback).
template <bool ALL>
__global__ void k_place(StepArgs A)
{
    grid_dependency_wait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ntot) return;
    const uint32_t c = A.cell_id[i];
    const uint32_t s = A.cell_off[c], e = A.cell_off[c + 1];
    uint32_t j = s;
    for (uint32_t k = s; k < e; ++k) j += A.unsorted[k] < i ? 1u : 0u;
    A.perm[j] = i;
    const double4 x = A.x[i];
    A.xs[j] = x;
    A.xf[j] = make_float4((float)x.x, (float)x.y, (float)x.z, (float)x.w);
    A.rank[i] = j;
    if (ALL) {
        A.vs[j] = A.vel[i];
        A.ws[j] = A.angvel[i];
    }
}

// --------------------------------------------------------- neighbour lists

constexpr int VLIST_THREADS = 128;

// Neighbour lists for the contact search of contact models 2 and 3: for the
// sphere at sorted position a, the ids of all spheres within
// ra + rb + vskin among the +-vrange cells around it (FP32 test widened by
// the prefilter margin, so the list may hold a few more), ascending and
// without repeats.  A sphere that moves less than vskin / 2 (checked in the
// integration against xref) keeps every sphere it can touch in its list.
// Runs only when vflag[0] is set; a list that overflows vcap (<= VL_MAX) is
// marked VL_MAX + 1 and that sphere uses the cell search.  Entry k of
// sphere i goes to vlist[i * row_stride + k * k_stride] (rows of VL_MAX for
// the FP64 form's lists, entry-major for the list step's).
__device__ __forceinline__ void vlist_build_one(const StepArgs &A, uint32_t a, uint32_t *lst,
                                                uint32_t *vlist, uint32_t *vcount, uint32_t cap,
                                                uint32_t row_stride, uint32_t k_stride)
{
    const int RS = VLIST_THREADS;
    const uint32_t i = A.perm[a];
    const DevBox &B = A.boxes[A.box_of[i]];
    const float4 xaf = A.xf[a];
    A.xref[i] = xaf;
    const int R = B.vrange;
    const uint32_t cm = B.P.contactmodel;
    if (R < 1 || (cm != 2 && cm != 3)) {
        vcount[i] = VL_MAX + 1;
        return;
    }
    int g0, g1, g2;
    unpack_cell(A.cellc[i], g0, g1, g2);
    const int nx = (int)B.num[0], ny = (int)B.num[1];
    const float reach = B.pre_margin + B.vskin;
    const float Lf0 = (float)B.L[0], Lf1 = (float)B.L[1];
    int n = 0;
    bool over = false;
    for (int dz = -R; dz <= R && !over; ++dz)
        for (int dy = -R; dy <= R && !over; ++dy)
            for (int dx = -R; dx <= R && !over; ++dx) {
                int tx = g0 + dx, ty = g1 + dy, sx, sy;
                const int tz = g2 + dz;
                if (!image_cell(B, tx, ty, tz, sx, sy)) continue;
                const float fsx = sx == 0 ? 0.f : (sx > 0 ? Lf0 : -Lf0);
                const float fsy = sy == 0 ? 0.f : (sy > 0 ? Lf1 : -Lf1);
                const uint32_t cell = B.cell_base + (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                const uint32_t start = A.cell_off[cell], end = A.cell_off[cell + 1];
                for (uint32_t b = start; b < end; ++b) {
                    if (b == a) continue;
                    if (!maybe_touching(xaf, A.xf[b], fsx, fsy, reach)) continue;
                    const uint32_t bo = A.perm[b];
                    int q = n;
                    while (q > 0 && lst[(q - 1) * RS] > bo) --q;
                    if (q > 0 && lst[(q - 1) * RS] == bo) continue;   // another image
                    if (n == (int)cap) {
                        over = true;
                        break;
                    }
                    for (int k = n; k > q; --k) lst[k * RS] = lst[(k - 1) * RS];
                    lst[q * RS] = bo;
                    ++n;
                }
            }
    if (over) {
        vcount[i] = VL_MAX + 1;
        return;
    }
    uint32_t *out = vlist + (size_t)i * row_stride;
    for (int k = 0; k < n; ++k) out[(size_t)k * k_stride] = lst[k * RS];
    vcount[i] = (uint32_t)n;
}

// A grid of a few blocks per SM that strides over the spheres, so that the
// launch costs little on the steps that build nothing.
constexpr unsigned VLIST_BLOCKS = 148u * 8u;

__global__ void __launch_bounds__(VLIST_THREADS) k_vlist_build(StepArgs A)
{
    grid_dependency_wait();
    if (A.vflag[0] == 0u) return;
    __shared__ uint32_t s_list[VL_MAX * VLIST_THREADS];
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < A.ntot;
         a += gridDim.x * blockDim.x)
        vlist_build_one(A, a, s_list + threadIdx.x, A.vlist, A.vcount, A.vcap, VL_MAX, 1u);
}

// The list step's rebuild (sph_pair.cu): its current positions into A.x for
// the cell sort, and its lists built at full capacity into the buffers not
// in use.
__global__ void k_pair_sync_x(StepArgs A, PairArgs P)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < A.ntot) A.x[i] = P.xr[*P.pp][i];
}

__global__ void __launch_bounds__(VLIST_THREADS) k_pair_vlist(StepArgs A, PairArgs P)
{
    __shared__ uint32_t s_list[VL_MAX * VLIST_THREADS];
    const uint32_t alt = *P.lsel ^ 1u;
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < A.ntot) vlist_build_one(A, a, s_list + threadIdx.x, P.ids[alt], P.cnt[alt], VL_MAX, 1u, P.nrow);
}

// After the (possible) build: clear the request, count builds.
__global__ void k_vlist_done(StepArgs A)
{
    grid_dependency_wait();
    if (A.vflag[0] != 0u) {
        A.vflag[0] = 0u;
        A.vflag[1] += 1u;
    }
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

// Per-box kernels: one block per box, partials staged in BOX_STAGE chunks.
constexpr int BOX_THREADS = 256;
constexpr int BOX_STAGE = 2048;

// In-order sum of cnt doubles staged in shared memory, by one thread, its
// loads issued eight at a time ahead of the additions.
__device__ __forceinline__ double ordered_sum(const double *v_s, uint32_t cnt, double acc)
{
    uint32_t k = 0;
    for (; k + 8 <= cnt; k += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = v_s[k + q];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc += v[q];
    }
    for (; k < cnt; ++k) acc += v_s[k];
    return acc;
}

// Sum of the shear-stress partials per box (integration.cuh:65-68), once
// per box instead of once per particle: one block per box stages the
// partials in shared memory with coalesced loads and thread 0 adds them in
// block order, the reference's order.
__global__ void __launch_bounds__(BOX_THREADS) k_tau_final(StepArgs A)
{
    __shared__ double s_part[BOX_STAGE];
    const uint32_t b = blockIdx.x;
    if (b >= A.nboxes) return;
    DevBox &B = A.boxes[b];
    double tau = 0.0;
    if (B.nw > 0 && B.wmode[0] == 3) {
        for (uint32_t base = 0; base < B.nblocks; base += BOX_STAGE) {
            const uint32_t cnt = min((uint32_t)BOX_STAGE, B.nblocks - base);
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x)
                s_part[k] = A.tau_partial[B.part_base + base + k];
            __syncthreads();
            if (threadIdx.x == 0) tau = ordered_sum(s_part, cnt, tau);
        }
    }
    if (threadIdx.x == 0) B.tau_eff_x = tau;
}

// integration.cuh:344-450 integrateWalls, then the loop bookkeeping of
// device.cu:2536-2538, the adaptive grid of device.cu:1050 and the
// velocity-step state of device.cu:2455-2462 for the next step.
// One block per box.  The wall-force total is the sequential sum of the
// per-block partials in block order (as the reference's integrateWalls
// loop); the block stages the partials in shared memory with coalesced
// loads and thread 0 adds them in order.
__global__ void __launch_bounds__(BOX_THREADS) k_box_step(StepArgs A)
{
    __shared__ double s_part[BOX_STAGE];
    const uint32_t b = blockIdx.x;
    if (b >= A.nboxes) return;
    DevBox &B = A.boxes[b];
    bool any = false;
    for (uint32_t w = 0; w < B.nw; ++w) any = any || B.wmode[w] != 0;
    double fsum = 0.0;
    if (B.np > 0 && any) {
        for (uint32_t base = 0; base < B.nblocks; base += BOX_STAGE) {
            const uint32_t cnt = min((uint32_t)BOX_STAGE, B.nblocks - base);
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x)
                s_part[k] = A.wall_partial[B.part_base + base + k];
            __syncthreads();
            // the sequential sum of integrateWalls
            if (threadIdx.x == 0) fsum = ordered_sum(s_part, cnt, fsum);
        }
    }
    if (threadIdx.x != 0) return;
    advance_box(B, fsum);
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
    if (B.periodic == 0) {   // side walls along x
        const double lo = (B.origo[0] + xa.w) - xa.x, hi = xa.x + xa.w - B.L[0];
        if (lo > 0.0) { dx += lo; worst = fmax(worst, lo); }
        if (hi > 0.0) { dx -= hi; worst = fmax(worst, hi); }
    }
    if (B.periodic != 1) {   // side walls along y
        const double lo = (B.origo[1] + xa.w) - xa.y, hi = xa.y + xa.w - B.L[1];
        if (lo > 0.0) { dy += lo; worst = fmax(worst, lo); }
        if (hi > 0.0) { dy -= hi; worst = fmax(worst, hi); }
    }
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
    k_place<true><<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), st);
    k_relax<<<blocks_for(A.ntot, 128), 128, 0, st>>>(A, alpha, z_top, d_max);
    k_relax_apply<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    if (launches) *launches += 9;
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

// ---------------------------------------------------------------- analysis

// src/sphere.cpp:487-606 DEM::porosity, one thread per slab: the slab
// volume less the spheres' volumes inside it (with the reference's cap
// terms), spheres in index order, so that every slab's sum is the
// reference's, operation for operation.  All threads of a warp read the
// same sphere at a time (broadcast).
// One block per slab.  The slab's void volume is the reference's sequential
// subtraction over the spheres in index order (one or two subtractions per
// sphere that reaches into the slab, none otherwise); the threads compute
// the terms of 256 spheres at a time and thread 0 applies them in index
// order, skipping the spheres without a term (src/sphere.cpp:520-587).
constexpr int POR_THREADS = 256;

__global__ void __launch_bounds__(POR_THREADS) k_porosity(const double4 *x, uint32_t p0,
                                                          uint32_t np, double h_slice,
                                                          double V_slice, uint32_t nslices,
                                                          double *z_pos, double *por)
{
    __shared__ double s_t[2][POR_THREADS];
    __shared__ int s_n[POR_THREADS];
    __shared__ uint32_t s_mask[POR_THREADS / 32];
    const uint32_t iz = blockIdx.x;
    const double z_low = (double)iz * h_slice;
    const double z_high = z_low + h_slice;
    double V_void = V_slice;
    for (uint32_t base = 0; base < np; base += POR_THREADS) {
        const uint32_t i = base + threadIdx.x;
        int n = 0;
        double t0 = 0.0, t1 = 0.0;
        if (i < np) {
            const double4 p = x[p0 + i];
            const double zc = p.z, r = p.w;
            const double zl = zc - r, zh = zc + r;
            const double V_s = 4.0 / 3.0 * M_PI * r * r * r;
            if (z_low <= zl && zh <= z_high) {
                t0 = V_s;
                n = 1;
            } else {
                if (z_low >= zc && z_low <= zh) {
                    const double h = zh - z_low;
                    t0 = M_PI * h * h / 3.0 * (3.0 * r - h);
                    n = 1;
                } else if (z_low < zc && z_low > zl) {
                    const double h = z_low - zl;
                    t0 = V_s + M_PI * h * h / 3.0 * (3.0 * r - h);
                    n = 1;
                }
                double tb = 0.0;
                bool hb = false;
                if (z_high <= zc && z_high >= zl) {
                    const double h = z_high - zl;
                    tb = M_PI * h * h / 3.0 * (3.0 * r - h);
                    hb = true;
                } else if (z_high > zc && z_high < zh) {
                    const double h = zh - z_high;
                    tb = V_s + M_PI * h * h / 3.0 * (3.0 * r - h);
                    hb = true;
                }
                if (hb) {
                    if (n == 0) t0 = tb;
                    else t1 = tb;
                    ++n;
                }
            }
        }
        s_t[0][threadIdx.x] = t0;
        s_t[1][threadIdx.x] = t1;
        s_n[threadIdx.x] = n;
        const uint32_t m = __ballot_sync(0xffffffffu, n > 0);
        if ((threadIdx.x & 31) == 0) s_mask[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 0; w < POR_THREADS / 32; ++w)
                for (uint32_t b = s_mask[w]; b; b &= b - 1u) {
                    const int t = w * 32 + __ffs(b) - 1;
                    V_void -= s_t[0][t];
                    if (s_n[t] > 1) V_void -= s_t[1][t];
                }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && iz < nslices) {
        z_pos[iz] = z_low + 0.5 * h_slice;
        por[iz] = V_void / V_slice;
    }
}

int porosity_profile(const double4 *x, uint32_t p0, uint32_t np, double h_slice, double V_slice,
                     uint32_t nslices, double *z_pos, double *por, cudaStream_t st)
{
    k_porosity<<<nslices, POR_THREADS, 0, st>>>(x, p0, np, h_slice, V_slice, nslices, z_pos, por);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

// src/sphere.cpp:677-725 DEM::findOverlaps on the device: the box's spheres
// binned into its own grid (clamped cells), each sphere i testing the
// spheres j > i in the cells within +-R (no periodic images), first
// counting, then writing its pairs in ascending j after an exclusive scan
// of the counts, so that the list is the reference's, in its order.

__device__ __forceinline__ void ov_cell(const OverlapArgs &O, double4 p, int c[3])
{
    const double v[3] = {p.x, p.y, p.z};
    for (int d = 0; d < 3; ++d) {
        double f = floor((v[d] - O.origo[d]) / O.cw[d]);
        if (!(f >= 0.0)) f = 0.0;
        if (f > (double)(O.num[d] - 1)) f = (double)(O.num[d] - 1);
        c[d] = (int)f;
    }
}

__global__ void k_ov_bin(OverlapArgs O)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O.np) return;
    int c[3];
    ov_cell(O, O.x[O.p0 + i], c);
    const uint32_t cell = (uint32_t)((c[2] * O.num[1] + c[1]) * O.num[0] + c[0]);
    O.cell_of[i] = cell;
    O.slot[i] = atomicAdd(&O.count[cell], 1u);
}

__global__ void k_ov_scatter(OverlapArgs O)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O.np) return;
    O.items[O.coff[O.cell_of[i]] + O.slot[i]] = i;
}

// WRITE = false: count the pairs of sphere i; true: write them sorted by j.
template <bool WRITE>
__global__ void k_ov_pairs(OverlapArgs O)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O.np) return;
    const double4 xi = O.x[O.p0 + i];
    const bool free_i = O.vel[O.p0 + i].w == 0.0;
    int c[3];
    ov_cell(O, xi, c);
    uint32_t n = 0;
    const uint32_t base = WRITE ? O.poff[i] : 0u;
    const uint32_t cnt = WRITE ? O.npair[i] : 0u;
    for (int dz = -O.R; dz <= O.R; ++dz)
        for (int dy = -O.R; dy <= O.R; ++dy)
            for (int dx = -O.R; dx <= O.R; ++dx) {
                const int tx = c[0] + dx, ty = c[1] + dy, tz = c[2] + dz;
                if (tx < 0 || ty < 0 || tz < 0 || tx >= O.num[0] || ty >= O.num[1] ||
                    tz >= O.num[2])
                    continue;
                const uint32_t cell = (uint32_t)((tz * O.num[1] + ty) * O.num[0] + tx);
                for (uint32_t q = O.coff[cell]; q < O.coff[cell + 1]; ++q) {
                    const uint32_t j = O.items[q];
                    if (j <= i) continue;
                    const double4 xj = O.x[O.p0 + j];
                    const double ddx = xj.x - xi.x, ddy = xj.y - xi.y, ddz = xj.z - xi.z;
                    const double len = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                    const double d = len - (xi.w + xj.w);
                    if (!(d < 0.0 && free_i && O.vel[O.p0 + j].w == 0.0)) continue;
                    if (WRITE && n < cnt) {
                        // insertion by j into this sphere's part of the list
                        uint32_t k = n;
                        while (k > 0 && O.pairs[2 * (size_t)(base + k - 1) + 1] > j) {
                            O.pairs[2 * (size_t)(base + k)] = O.pairs[2 * (size_t)(base + k - 1)];
                            O.pairs[2 * (size_t)(base + k) + 1] =
                                O.pairs[2 * (size_t)(base + k - 1) + 1];
                            O.delta[base + k] = O.delta[base + k - 1];
                            --k;
                        }
                        O.pairs[2 * (size_t)(base + k)] = i;
                        O.pairs[2 * (size_t)(base + k) + 1] = j;
                        O.delta[base + k] = d;
                    }
                    ++n;
                }
            }
    if (!WRITE) O.npair[i] = n;
}

int find_overlaps(OverlapArgs O, uint32_t ncells, uint32_t *scan_tmp, cudaStream_t st,
                  int stage)
{
    const unsigned gb = blocks_for(O.np, 256);
    if (stage == 0) {
        cudaMemsetAsync(O.count, 0, sizeof(uint32_t) * ncells, st);
        k_ov_bin<<<gb, 256, 0, st>>>(O);
        const uint32_t nb = blocks_for(ncells, SCAN_TILE);
        k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(O.count, ncells, scan_tmp);
        k_scan_top<<<1, SCAN_THREADS, 0, st>>>(scan_tmp, nb);
        k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(O.count, ncells, scan_tmp, nb, O.coff);
        k_ov_scatter<<<gb, 256, 0, st>>>(O);
        k_ov_pairs<false><<<gb, 256, 0, st>>>(O);
        const uint32_t np_b = blocks_for(O.np, SCAN_TILE);
        k_scan_reduce<<<np_b, SCAN_THREADS, 0, st>>>(O.npair, O.np, scan_tmp);
        k_scan_top<<<1, SCAN_THREADS, 0, st>>>(scan_tmp, np_b);
        k_scan_down<<<np_b, SCAN_THREADS, 0, st>>>(O.npair, O.np, scan_tmp, np_b, O.poff);
    } else {
        k_ov_pairs<true><<<gb, 256, 0, st>>>(O);
    }
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

// Record a profiling event on st.  Under stream capture the record must be
// external, or it only orders the capture and is never timed.
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

// FP64 interact launcher (bit-exact form).
static void interact_fp64(const StepArgs &A, cudaStream_t st, unsigned grid, bool fused, int lm,
                          int variant)
{
    launch_interact<false>(A, st, grid, fused, lm, variant);
}

static void contacts_fp64(const StepArgs &A, cudaStream_t st, unsigned grid, int lm, bool pdl)
{
    launch_contacts<false>(A, st, grid, lm, pdl);
}

void launch_pair_sort_build(const StepArgs &A, const PairArgs &P, cudaStream_t st)
{
    k_pair_sync_x<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A, P);
    cudaMemsetAsync(A.cell_count, 0, sizeof(uint32_t) * A.ncells, st);
    k_hash<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    const uint32_t nb = blocks_for(A.ncells, SCAN_TILE);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp);
    k_scan_top<<<1, SCAN_THREADS, 0, st>>>(A.scan_tmp, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(A.cell_count, A.ncells, A.scan_tmp, nb, A.cell_off);
    k_scatter<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    k_place<false><<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
    k_pair_vlist<<<blocks_for(A.ntot, VLIST_THREADS), VLIST_THREADS, 0, st>>>(A, P);
}

int launch_step(const StepArgs &A, const StepConfig &cfg, cudaStream_t st, uint64_t *launches,
                Prof *prof)
{
    return launch_step_with(A, cfg, st, launches, prof, interact_fp64, contacts_fp64);
}

int launch_step_with(const StepArgs &A, const StepConfig &cfg, cudaStream_t st,
                     uint64_t *launches, Prof *prof, InteractLauncher interact,
                     ContactLauncher contact)
{
    uint64_t nl = 0;
    // programmatic dependent launches along the step's chain of kernels,
    // except where events are recorded between them (profiling)
    const bool pdl = prof == nullptr;
    if (prof) {
        prof->n = 0;
        record(prof->ev[0], st);
    }
    // the wall stage: wall-force partial sums and integrateWalls, time and
    // box state (integration.cuh:309-450, device.cu:2504-2537)
    auto wall_stage = [&](cudaStream_t s) {
        if (A.ntot > 0 && cfg.any_walls) {
            k_block_sums<<<A.npartials, 256, 0, s>>>(A, A.wf_pp, A.wall_partial, 0);
            mark(prof, s, "k_block_sums");
            nl += 1;
        }
        k_box_step<<<A.nboxes, BOX_THREADS, 0, s>>>(A);
        mark(prof, s, "k_box_step");
        nl += 1;
    };
    if (cfg.phase == STEP_TAIL) {
        wall_stage(st);
        if (launches) *launches += nl;
        return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
    }
    const bool overlap = cfg.phase == STEP_OVERLAP;
    if (overlap) {
        cudaEventRecord(cfg.fork, st);
        cudaStreamWaitEvent(cfg.side, cfg.fork, 0);
        wall_stage(cfg.side);
        cudaEventRecord(cfg.join, cfg.side);
    }
    if (A.ntot > 0) {
        cudaMemsetAsync(A.cell_count, 0, sizeof(uint32_t) * A.ncells, st);
        k_hash<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
        mark(prof, st, "k_hash");
        const uint32_t nb = blocks_for(A.ncells, SCAN_TILE);
        launch_k(pdl, k_scan_reduce, nb, SCAN_THREADS, st, (const uint32_t *)A.cell_count,
                 A.ncells, A.scan_tmp);
        launch_k(pdl, k_scan_top, 1, SCAN_THREADS, st, A.scan_tmp, nb);
        launch_k(pdl, k_scan_down, nb, SCAN_THREADS, st, (const uint32_t *)A.cell_count, A.ncells,
                 (const uint32_t *)A.scan_tmp, nb, A.cell_off);
        mark(prof, st, "k_scan(3)");
        launch_k(pdl, k_scatter, blocks_for(A.ntot, 256), 256, st, A);
        mark(prof, st, "k_scatter");
        const bool split = cfg.variant == SPLIT_VARIANT && !cfg.unfused && cfg.all_cm23 &&
                           A.vlist && A.csum;
        if (split) launch_k(pdl, k_place<false>, blocks_for(A.ntot, 256), 256, st, A);
        else launch_k(pdl, k_place<true>, blocks_for(A.ntot, 256), 256, st, A);
        mark(prof, st, "k_place");
        nl += 7;
        if (A.vlist) {
            const unsigned gv = blocks_for(A.ntot, VLIST_THREADS);
            launch_k(pdl, k_vlist_build, gv < VLIST_BLOCKS ? gv : VLIST_BLOCKS, VLIST_THREADS, st, A);
            launch_k(pdl, k_vlist_done, 1, 1, st, A);
            mark(prof, st, "k_vlist");
            nl += 2;
        }
        if (A.nbonds) {
            if (cfg.lenmode == SPH_LEN_FP64) k_bonds<SPH_LEN_FP64><<<blocks_for(A.nbonds, 128), 128, 0, st>>>(A);
            else k_bonds<SPH_LEN_REFERENCE><<<blocks_for(A.nbonds, 128), 128, 0, st>>>(A);
            mark(prof, st, "k_bonds");
            nl += 1;
        }
        const unsigned gi = blocks_for(A.ntot, INTERACT_THREADS);
        if (split) {
            const unsigned gs = blocks_for(A.ntot, SEARCH_THREADS);
            // after k_bonds (when there are bonds) an ordinary launch
            const bool pdl_s = pdl && !A.nbonds;
            if (cfg.lenmode == SPH_LEN_FP64)
                launch_k(pdl_s, k_search<SPH_LEN_FP64>, gs, SEARCH_THREADS, st, A);
            else
                launch_k(pdl_s, k_search<SPH_LEN_REFERENCE>, gs, SEARCH_THREADS, st, A);
            mark(prof, st, "k_search");
            contact(A, st, blocks_for(A.ntot, CONTACT_THREADS), cfg.lenmode, pdl);
            mark(prof, st, "k_contacts");
            if (overlap) cudaStreamWaitEvent(st, cfg.join, 0);
            if (cfg.lenmode == SPH_LEN_FP64)
                k_finish<SPH_LEN_FP64><<<blocks_for(A.ntot, FINISH_THREADS), FINISH_THREADS, 0, st>>>(A);
            else
                k_finish<SPH_LEN_REFERENCE><<<blocks_for(A.ntot, FINISH_THREADS), FINISH_THREADS, 0, st>>>(A);
            mark(prof, st, "k_finish");
            nl += 3;
        } else if (!cfg.unfused) {
            if (overlap) cudaStreamWaitEvent(st, cfg.join, 0);
            interact(A, st, gi, true, cfg.lenmode,
                     cfg.variant == SPLIT_VARIANT ? 1 : cfg.variant);
            mark(prof, st, "k_interact");
            nl += 1;
        } else {
            if (overlap) cudaStreamWaitEvent(st, cfg.join, 0);
            interact(A, st, gi, false, cfg.lenmode,
                     cfg.variant == SPLIT_VARIANT ? 1 : cfg.variant);
            mark(prof, st, "k_interact");
            if (cfg.darcy) {
                // device.cu:1891-2419, between interact and integrate
                const int ds = launch_darcy(A, *cfg.darcy, cfg, st, &nl, prof);
                if (ds != SPH_OK) return ds;
            }
            k_shear_stress<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
            k_block_sums<<<A.npartials, 256, 0, st>>>(A, A.tau_pp, A.tau_partial, 1);
            k_tau_final<<<A.nboxes, BOX_THREADS, 0, st>>>(A);
            mark(prof, st, "k_shear_stress+sums");
            k_integrate<<<blocks_for(A.ntot, 256), 256, 0, st>>>(A);
            mark(prof, st, "k_integrate");
            nl += 5;
        }
    } else if (overlap) {
        cudaStreamWaitEvent(st, cfg.join, 0);
    }
    if (A.ntot == 0 && cfg.darcy) {
        // a fluid without spheres (the reference's pure-fluid runs)
        const int ds = launch_darcy(A, *cfg.darcy, cfg, st, &nl, prof);
        if (ds != SPH_OK) return ds;
    }
    if (cfg.phase == STEP_WHOLE) wall_stage(st);
    if (cfg.darcy) {
        launch_darcy_tick(A, *cfg.darcy, st);
        nl += 1;
    }
    if (launches) *launches += nl;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "sphere_b200: kernel launch failed: %s\n", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}

}  // namespace sph
