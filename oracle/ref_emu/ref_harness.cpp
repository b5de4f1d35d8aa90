/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own DEM step kernels on the CPU.  The kernels are
 * #included unmodified from the reference sources (src/sorting.cuh,
 * src/contactmodels.cuh, src/cohesion.cuh, src/contactsearch.cuh,
 * src/integration.cuh) through cuda_host_shim.h, and launched here in the
 * order of the reference's step loop for fluid == 0 (src/device.cu:1031-2538).
 * The result (libsphere_ref.so, built by oracle/ref_emu/Makefile into
 * oracle/_ref/) pins the restatement in oracle/sphere_oracle.c: both read and
 * write the same OrState.
 *
 * Launch emulation: every block of a launch runs its threads one after the
 * other in thread order, which is exact for these kernels because no thread
 * reads what another thread of the same launch writes, with three
 * exceptions handled explicitly:
 *  - reorderArrays (sorting.cuh:56-132) reads the key that the previous
 *    thread stored in shared memory; in-order execution provides it;
 *  - summation (integration.cuh:309-341) is a shared-memory tree reduction
 *    with barriers; its threads run as cooperative fibers that switch at
 *    every __syncthreads();
 *  - bondsLinear (cohesion.cuh:8-233) adds into shared particles without
 *    atomics; it runs serially, in ascending bond order.
 * thrust::sort_by_key (device.cu:1075) is a stable radix sort for 32-bit
 * keys; std::stable_sort is used here.
 * The harness is built with -ftrivial-auto-var-init=zero so that the
 * reference's one uninitialised local (contactmodels.cuh:320) reads as zero.
 */
#include "cuda_host_shim.h"
#include "helper_math.h"

#include "vector_arithmetic.h"
#include "constants.cuh"
#include "sorting.cuh"
#include "contactmodels.cuh"
#include "cohesion.cuh"
#include "contactsearch.cuh"
#include "integration.cuh"
/* the reference's Darcy kernels (src/darcy.cuh) and the helpers they take
 * from src/navierstokes.cuh, extracted by oracle/Makefile */
#include "darcy_kernels.inc"

#include <ucontext.h>
#include <algorithm>
#include <functional>
#include <utility>
#include <vector>

#include "../sphere_oracle.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
/* dynamic shared memory of reorderArrays (sorting.cuh:70) */
thread_local unsigned int shared_data[4096];

static thread_local bool g_fiber_mode = false;
static thread_local ucontext_t g_sched;
static thread_local ucontext_t *g_cur = nullptr;
static thread_local const std::function<void()> *g_body = nullptr;
static thread_local bool g_finished = false;

void __syncthreads(void)
{
    if (g_fiber_mode) swapcontext(g_cur, &g_sched);
}

static void fiber_entry(void)
{
    (*g_body)();
    g_finished = true;
}

/* Sequential launch: blocks in parallel (optional), threads in order. */
static void launch_seq(unsigned grid, unsigned block, const std::function<void()> &body,
                       bool parallel_blocks)
{
    auto run_block = [&](unsigned b) {
        blockIdx = make_uint3(b, 0, 0);
        blockDim = dim3(block, 1, 1);
        gridDim = dim3(grid, 1, 1);
        for (unsigned t = 0; t < block; ++t) {
            threadIdx = make_uint3(t, 0, 0);
            body();
        }
    };
    if (parallel_blocks) {
#pragma omp parallel for schedule(dynamic, 4)
        for (long b = 0; b < (long)grid; ++b) run_block((unsigned)b);
    } else {
        for (unsigned b = 0; b < grid; ++b) run_block(b);
    }
}

/* Fiber launch: threads of a block switch at every barrier. */
static void launch_fibers(unsigned grid, unsigned block, const std::function<void()> &body)
{
    const size_t stack_size = 64 * 1024;
    std::vector<ucontext_t> ctx(block);
    std::vector<std::vector<char>> stacks(block, std::vector<char>(stack_size));
    std::vector<char> done(block);
    g_body = &body;
    g_fiber_mode = true;
    blockDim = dim3(block, 1, 1);
    gridDim = dim3(grid, 1, 1);
    for (unsigned b = 0; b < grid; ++b) {
        blockIdx = make_uint3(b, 0, 0);
        for (unsigned t = 0; t < block; ++t) {
            getcontext(&ctx[t]);
            ctx[t].uc_stack.ss_sp = stacks[t].data();
            ctx[t].uc_stack.ss_size = stack_size;
            ctx[t].uc_link = &g_sched;
            makecontext(&ctx[t], fiber_entry, 0);
            done[t] = 0;
        }
        unsigned live = block;
        while (live > 0) {
            for (unsigned t = 0; t < block; ++t) {
                if (done[t]) continue;
                threadIdx = make_uint3(t, 0, 0);
                g_cur = &ctx[t];
                g_finished = false;
                swapcontext(&g_sched, &ctx[t]);
                if (g_finished) { done[t] = 1; --live; }
            }
        }
    }
    g_fiber_mode = false;
}

static inline Float4 *F4(double *p) { return reinterpret_cast<Float4 *>(p); }
/* src/darcy.cpp:64-76 DEM::d_idx */
static inline unsigned d_idx_host(unsigned nx, unsigned ny, int x, int y, int z)
{
    return (x + 1) + (nx + 2) * (y + 1) + (nx + 2) * (ny + 2) * (z + 1);
}
static inline Float3 *F3(double *p) { return reinterpret_cast<Float3 *>(p); }

/* 3-D launch on the fluid grid (src/device.cu:865-869: 8 x 8 x 8 threads
 * per block, blocks covering grid.num), blocks and threads in order.  None
 * of the Darcy kernels reads what another thread of the same launch
 * writes, so the order is immaterial. */
static void launch_fluid(const std::function<void()> &body)
{
    const unsigned gx = (devC_grid.num[0] + 7) / 8, gy = (devC_grid.num[1] + 7) / 8;
    const unsigned gz = (devC_grid.num[2] + 7) / 8;
    gridDim = dim3(gx, gy, gz);
    blockDim = dim3(8, 8, 8);
    for (unsigned bz = 0; bz < gz; ++bz)
        for (unsigned by = 0; by < gy; ++by)
            for (unsigned bx = 0; bx < gx; ++bx) {
                blockIdx = make_uint3(bx, by, bz);
                for (unsigned tz = 0; tz < 8; ++tz)
                    for (unsigned ty = 0; ty < 8; ++ty)
                        for (unsigned tx = 0; tx < 8; ++tx) {
                            threadIdx = make_uint3(tx, ty, tz);
                            body();
                        }
            }
}

/* The Darcy part of the step loop, src/device.cu:1891-2419, with the
 * host's residual check (src/darcy.cpp:266-293, every nijacnorm = 10
 * iterations, src/debug.h:16) and conv.log bookkeeping as entries of the
 * state's log; a NaN residual raises SPH_ERR_NAN instead of exit(1). */
static void ref_darcy(OrState *s, unsigned iter, unsigned blocksPerGrid, unsigned threadsPerBlock,
                      Float4 *dev_x, Float4 *dev_x_sorted, Float4 *dev_vel_sorted, Float4 *dev_force)
{
    OrDarcy *D = s->darcy;
    const SphDarcy &d = D->prm;
    const unsigned np = s->box.np;
    const unsigned nx = devC_grid.num[0], ny = devC_grid.num[1], nz = devC_grid.num[2];
    if (s->box.walls.nw > 0 && (s->box.walls.wmode[0] == 1 || s->box.walls.wmode[0] == 3))
        D->wall0_iz = D->wall_w_host / (devC_grid.L[2] / devC_grid.num[2]);
    const unsigned wall0_iz = D->wall0_iz;
    Float *p = D->p, *p_old = D->p_old, *p_new = D->p_new, *dp_expl = D->dp_expl;
    Float *phi = D->phi, *dphi = D->dphi, *norm = D->norm, *k = D->k, *div_v_p = D->div_v_p;
    Float3 *v = F3(D->v), *vp_avg = F3(D->vp_avg), *grad_k = F3(D->grad_k), *grad_p = F3(D->grad_p);
    int *p_constant = D->p_constant;
    if (np > 0) {
        launch_fluid([&] { setDarcyGhostNodes<Float>(p, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
        launch_fluid([&] { findDarcyPressureGradient(p, grad_p); });
        launch_fluid([&] { setDarcyGhostNodes<Float3>(grad_p, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
        launch_seq(blocksPerGrid, threadsPerBlock,
                   [&] {
                       findDarcyPressureForceLinear(dev_x, grad_p, phi, wall0_iz, d.rho_f, d.bc_top,
                                                    dev_force, F4(D->f_p));
                   },
                   false);
    }
    if ((iter % d.ndem) != 0) return;
    launch_fluid([&] {
        findDarcyPorositiesLinear(s->cell_start, s->cell_end, dev_x_sorted, dev_vel_sorted, iter,
                                  d.ndem, np, d.c_phi, phi, dphi, div_v_p, vp_avg);
    });
    if (devC_grid.periodic == 2) {
        launch_fluid([&] { copyDarcyPorositiesToEdges(phi, dphi, div_v_p, vp_avg); });
        launch_fluid([&] { copyDarcyPorositiesToBottom(phi, dphi, div_v_p, vp_avg); });
    }
    if ((d.p_mod_A > 1.0e-5 || d.p_mod_A < -1.0e-5) && d.p_mod_f > 1.0e-7) {
        const Float new_pressure =
            D->p_top_orig + d.p_mod_A * sin(2.0 * M_PI * d.p_mod_f * s->box.t_current + d.p_mod_phi);
        /* the launch grid's threads past nx or ny write too; keep those
         * writes inside the array */
        std::vector<Float> pad((size_t)(nx + 2) * (ny + 2) * (nz + 2) + 16 * (nx + ny + 64), 0.0);
        std::memcpy(pad.data(), p, sizeof(Float) * (size_t)(nx + 2) * (ny + 2) * (nz + 2));
        launch_fluid([&] { setDarcyTopPressure(new_pressure, pad.data(), wall0_iz); });
        std::memcpy(p, pad.data(), sizeof(Float) * (size_t)(nx + 2) * (ny + 2) * (nz + 2));
        launch_fluid([&] { setDarcyTopWallPressure(new_pressure, wall0_iz, p); });
    }
    launch_fluid([&] { findDarcyPermeabilities(d.k_c, phi, k); });
    launch_fluid([&] { setDarcyGhostNodes<Float>(phi, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
    launch_fluid([&] { setDarcyGhostNodes<Float>(k, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
    launch_fluid([&] { findDarcyPermeabilityGradients(k, grad_k); });
    if (iter == 0) {
        launch_fluid([&] { setDarcyNormZero(norm); });
        launch_fluid([&] { copyValues<Float>(p, p_old); });
    }
    if (d.bc_bot == 4 || d.bc_top == 4)
        launch_fluid([&] { setDarcyGhostNodesFlux<Float>(p, d.bc_bot, d.bc_top, d.bc_bot_flux, d.bc_top_flux, k, d.mu); });
    unsigned nijac = 0, ok = 0;
    for (nijac = 0; nijac < d.maxiter; ++nijac) {
        if (nijac == 0) launch_fluid([&] { copyValues<Float>(p, p_old); });
        launch_fluid([&] { setDarcyGhostNodes<Float>(p, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
        if (nijac == 0)
            launch_fluid([&] {
                firstDarcySolution(p, k, phi, dphi, div_v_p, vp_avg, grad_k, d.beta_f, d.mu, d.bc_xn,
                                   d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top, d.ndem, wall0_iz,
                                   p_constant, dp_expl);
            });
        launch_fluid([&] {
            updateDarcySolution(p_old, dp_expl, p, k, phi, dphi, div_v_p, vp_avg, grad_k, d.beta_f, d.mu,
                                d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top, d.ndem, wall0_iz,
                                p_constant, p_new, norm);
        });
        if (d.bc_top == 1) {
            /* a wall at or above the top of the grid indexes past the padded
             * array: the kernel runs on a copy with room to spare, whose
             * part past the array is dropped (reads there see zeros) */
            const size_t nc = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
            std::vector<Float> pad(nc + (size_t)(nx + 2) * (ny + 2) * 16, 0.0);
            std::memcpy(pad.data(), p, sizeof(Float) * nc);
            launch_fluid([&] { setDarcyTopWallFixedFlow(wall0_iz, pad.data()); });
            std::memcpy(p, pad.data(), sizeof(Float) * nc);
        }
        if (d.bc_bot == 4 || d.bc_top == 4)
            launch_fluid([&] { setDarcyGhostNodesFlux<Float>(p, d.bc_bot, d.bc_top, d.bc_bot_flux, d.bc_top_flux, k, d.mu); });
        launch_fluid([&] { copyValues<Float>(p_new, p); });
        if (nijac % 10 == 0) {
            double max_norm_res = -1.0e9;
            bool nan = false;
            for (unsigned z = 0; z < nz && !nan; ++z)
                for (unsigned y = 0; y < ny && !nan; ++y)
                    for (unsigned x = 0; x < nx; ++x) {
                        const double r = fabs(norm[d_idx_host(nx, ny, x, y, z)]);
                        if (r != r) { nan = true; break; }
                        if (r > max_norm_res) max_norm_res = r;
                    }
            if (nan) {
                s->error_flags |= 1 << SPH_ERR_NAN;
                break;
            }
            if (max_norm_res <= d.tolerance) { ok = 1; break; }
        }
        if (nijac == d.maxiter - 1) break;
    }
    if (D->log_n < D->log_cap) {
        D->log_step[D->log_n] = (uint64_t)iter + 1;
        D->log_iters[D->log_n] = nijac;
        D->log_ok[D->log_n] = ok;
        D->log_n++;
    }
    if (D->filetimeclock + s->box.dt < d.file_dt)
        launch_fluid([&] { setDarcyZeros<Float>(dphi); });
    launch_fluid([&] { setDarcyGhostNodes<Float>(p, d.bc_xn, d.bc_xp, d.bc_yn, d.bc_yp, d.bc_bot, d.bc_top); });
    launch_fluid([&] { findDarcyVelocities(p, phi, k, d.mu, v); });
}

extern "C" int ref_step(OrState *s, uint64_t nsteps)
{
    const unsigned np = s->box.np;
    const unsigned nw = s->box.walls.nw;
    const unsigned nb0 = s->box.nb0;
    const unsigned threadsPerBlock = 256;                          /* device.cu:853 */
    const unsigned blocksPerGrid = (np + threadsPerBlock - 1) / threadsPerBlock;
    const unsigned blocksPerGridBonds = (nb0 + threadsPerBlock - 1) / threadsPerBlock;

    /* constant memory, device.cu:324-340 */
    devC_nd = 3;
    devC_np = np;
    devC_nw = nw;
    devC_nc = NC;
    devC_dt = s->box.dt;
    devC_nb0 = nb0;
    const SphParams &P = s->box.params;
    for (int d = 0; d < 3; ++d) devC_params.g[d] = P.g[d];
    devC_params.k_n = P.k_n;
    devC_params.k_t = P.k_t;
    devC_params.k_r = P.k_r;
    devC_params.E = P.E;
    devC_params.gamma_n = P.gamma_n;
    devC_params.gamma_t = P.gamma_t;
    devC_params.gamma_r = P.gamma_r;
    devC_params.mu_s = P.mu_s;
    devC_params.mu_d = P.mu_d;
    devC_params.mu_r = P.mu_r;
    devC_params.gamma_wn = P.gamma_wn;
    devC_params.gamma_wt = P.gamma_wt;
    devC_params.mu_ws = P.mu_ws;
    devC_params.mu_wd = P.mu_wd;
    devC_params.rho = P.rho;
    devC_params.contactmodel = P.contactmodel;
    devC_params.kappa = P.kappa;
    devC_params.db = P.db;
    devC_params.V_b = P.V_b;
    devC_params.lambda_bar = P.lambda_bar;
    devC_params.nb0 = nb0;
    devC_params.sigma_b = P.sigma_b;
    devC_params.tau_b = P.tau_b;
    devC_params.sigma0_A = P.sigma0_A;
    devC_params.sigma0_f = P.sigma0_f;

    /* aligned device-array stand-ins for walls and per-block partials */
    std::vector<Float4> w_nx(nw ? nw : 1), w_mvfd(nw ? nw : 1);
    std::vector<int> w_mode(nw ? nw : 1);
    std::vector<Float> w_acc(nw ? nw : 1), w_tau_x(nw ? nw : 1);
    for (unsigned i = 0; i < nw; ++i) {
        w_nx[i] = make_double4(s->box.walls.nx[i][0], s->box.walls.nx[i][1],
                               s->box.walls.nx[i][2], s->box.walls.nx[i][3]);
        w_mvfd[i] = make_double4(s->box.walls.mvfd[i][0], s->box.walls.mvfd[i][1],
                                 s->box.walls.mvfd[i][2], s->box.walls.mvfd[i][3]);
        w_mode[i] = s->box.walls.wmode[i];
        w_acc[i] = s->walls_acc[i];
        w_tau_x[i] = s->box.walls.tau_x;
    }
    std::vector<Float> force_pp((size_t)(nw ? nw : 1) * (np ? np : 1));
    std::vector<Float> force_partial((size_t)(blocksPerGrid ? blocksPerGrid : 1) * (nw ? nw : 1));
    std::vector<Float> tau_pp((size_t)(nw ? nw : 1) * (np ? np : 1));
    std::vector<Float> tau_partial((size_t)(blocksPerGrid ? blocksPerGrid : 1) * (nw ? nw : 1));
    std::vector<unsigned> keys(np ? np : 1), index(np ? np : 1);
    std::vector<std::pair<unsigned, unsigned>> kv(np);
    std::vector<Float4> vel0(np ? np : 1), angvel0(np ? np : 1);
    uint2 *bonds = reinterpret_cast<uint2 *>(s->bonds);

    Float4 *dev_x = F4(s->x), *dev_vel = F4(s->vel), *dev_angvel = F4(s->angvel);
    Float4 *dev_x_sorted = F4(s->x_sorted), *dev_vel_sorted = F4(s->vel_sorted);
    Float4 *dev_angvel_sorted = F4(s->angvel_sorted);
    Float4 *dev_force = F4(s->force), *dev_torque = F4(s->torque);

    int velocity_state = s->velocity_state;
    for (uint64_t step = 0; step < nsteps; ++step) {
        const unsigned iter = (unsigned)s->iter;
        /* device.cu:1050-1052 updateGridSize */
        if (s->box.grid.adaptive == 1 && nw > 0) s->box.grid.L[2] = w_nx[0].w;
        for (int d = 0; d < 3; ++d) {
            devC_grid.origo[d] = s->box.grid.origo[d];
            devC_grid.L[d] = s->box.grid.L[d];
            devC_grid.num[d] = s->box.grid.num[d];
        }
        devC_grid.periodic = s->box.grid.periodic;
        devC_grid.adaptive = s->box.grid.adaptive;
        const size_t ncells = (size_t)devC_grid.num[0] * devC_grid.num[1] * devC_grid.num[2];

        if (np > 0) {
            /* device.cu:1059 */
            launch_seq(blocksPerGrid, threadsPerBlock,
                       [&] { calcParticleCellID(keys.data(), index.data(), dev_x); }, true);
            std::memcpy(s->cell_id, keys.data(), np * sizeof(unsigned));
            /* device.cu:1075-1078 */
            for (unsigned i = 0; i < np; ++i) kv[i] = std::make_pair(keys[i], index[i]);
            std::stable_sort(kv.begin(), kv.end(),
                             [](const std::pair<unsigned, unsigned> &a,
                                const std::pair<unsigned, unsigned> &b) { return a.first < b.first; });
            for (unsigned i = 0; i < np; ++i) { keys[i] = kv[i].first; index[i] = kv[i].second; }
            /* device.cu:1089-1090 */
            std::memset(s->cell_start, 0xff, ncells * sizeof(unsigned));
            /* device.cu:1099 */
            launch_seq(blocksPerGrid, threadsPerBlock,
                       [&] {
                           reorderArrays(s->cell_start, s->cell_end, keys.data(), index.data(),
                                         dev_x, dev_vel, dev_angvel, dev_x_sorted,
                                         dev_vel_sorted, dev_angvel_sorted);
                       },
                       true);
            std::memcpy(s->perm, index.data(), np * sizeof(unsigned));
            /* device.cu:1119-1128 */
            if (P.contactmodel == 2 || P.contactmodel == 3)
                launch_seq(blocksPerGrid, threadsPerBlock,
                           [&] {
                               topology(s->cell_start, s->cell_end, index.data(), dev_x_sorted,
                                        s->contacts, F4(s->distmod));
                           },
                           true);
            /* device.cu:1146-1167 */
            launch_seq(blocksPerGrid, threadsPerBlock,
                       [&] {
                           interact(index.data(), s->cell_start, s->cell_end, dev_x, dev_x_sorted,
                                    dev_vel_sorted, dev_angvel_sorted, dev_vel, dev_angvel,
                                    dev_force, dev_torque, s->es_dot, s->ev_dot, s->es, s->ev,
                                    s->p, w_nx.data(), w_mvfd.data(), force_pp.data(),
                                    s->contacts, F4(s->distmod), F4(s->delta_t));
                       },
                       true);
            /* device.cu:1180-1191 */
            if (nb0 > 0)
                launch_seq(blocksPerGridBonds, threadsPerBlock,
                           [&] {
                               bondsLinear(bonds, F4(s->bonds_delta), F4(s->bonds_omega), dev_x,
                                           dev_vel, dev_angvel, dev_force, dev_torque);
                           },
                           false);
        }
        /* device.cu:1891-2419 */
        if (s->darcy)
            ref_darcy(s, iter, blocksPerGrid, threadsPerBlock, dev_x, dev_x_sorted, dev_vel_sorted,
                      dev_force);
        if (np > 0) {
            /* device.cu:2427-2452 */
            if (nw > 0 && w_mode[0] == 3) {
                launch_seq(blocksPerGrid, threadsPerBlock,
                           [&] {
                               findShearStressOnFixedMovingParticles(dev_x, dev_vel, dev_force,
                                                                     tau_pp.data());
                           },
                           true);
                launch_fibers(blocksPerGrid, threadsPerBlock,
                              [&] { summation(tau_pp.data(), tau_partial.data()); });
            }
            /* device.cu:2455-2462 */
            int change_velocity_state = 0;
            if (s->box.t_current >= 10.0 && s->box.t_current < 15.0 && velocity_state == 1) {
                change_velocity_state = 1;
                velocity_state = 2;
            } else if (s->box.t_current >= 15.0 && velocity_state == 2) {
                change_velocity_state = -1;
                velocity_state = 1;
            }
            /* device.cu:2467-2490 */
            launch_seq(blocksPerGrid, threadsPerBlock,
                       [&] {
                           integrate(dev_x_sorted, dev_vel_sorted, dev_angvel_sorted, dev_x,
                                     dev_vel, dev_angvel, dev_force, dev_torque, F4(s->angpos),
                                     F4(s->acc), F4(s->angacc), vel0.data(), angvel0.data(),
                                     F4(s->xyzsum), index.data(), iter, w_mode.data(),
                                     w_mvfd.data(), tau_partial.data(), w_tau_x.data(),
                                     s->box.walls.tau_x, change_velocity_state, 10.0,
                                     blocksPerGrid);
                       },
                       true);
            /* device.cu:2503-2526 */
            if (nw > 0) {
                launch_fibers(blocksPerGrid, threadsPerBlock,
                              [&] { summation(force_pp.data(), force_partial.data()); });
                launch_seq(1, nw,
                           [&] {
                               integrateWalls(w_nx.data(), w_mvfd.data(), w_mode.data(),
                                              force_partial.data(), w_acc.data(), blocksPerGrid,
                                              s->box.t_current, iter);
                           },
                           false);
            }
        }
        /* device.cu:2536-2538 */
        s->box.t_current += s->box.dt;
        /* device.cu:2537, 2569, 2672: the file clock; the output's transfer
         * (device.cu:805) refreshes the host copy of the walls */
        if (s->darcy) {
            s->darcy->filetimeclock += s->box.dt;
            if (s->darcy->filetimeclock >= s->darcy->prm.file_dt) {
                s->darcy->filetimeclock = 0.0;
                if (nw > 0) s->darcy->wall_w_host = w_nx[0].w;
            }
        }
        s->iter++;
    }
    s->velocity_state = velocity_state;
    for (unsigned i = 0; i < nw; ++i) {
        s->box.walls.nx[i][0] = w_nx[i].x; s->box.walls.nx[i][1] = w_nx[i].y;
        s->box.walls.nx[i][2] = w_nx[i].z; s->box.walls.nx[i][3] = w_nx[i].w;
        s->box.walls.mvfd[i][0] = w_mvfd[i].x; s->box.walls.mvfd[i][1] = w_mvfd[i].y;
        s->box.walls.mvfd[i][2] = w_mvfd[i].z; s->box.walls.mvfd[i][3] = w_mvfd[i].w;
        s->walls_acc[i] = w_acc[i];
    }
    for (size_t i = 0; i < (size_t)nw * np && s->walls_force_pp; ++i) s->walls_force_pp[i] = force_pp[i];
    for (size_t i = 0; i < blocksPerGrid && s->walls_force_partial && nw > 0; ++i)
        s->walls_force_partial[i] = force_partial[i];
    return 0;
}
