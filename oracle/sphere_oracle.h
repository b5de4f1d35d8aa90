/*
 * sphere_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * State layout shared by the two CPU oracles used by the tests and by the
 * cpu_baseline leg of bench.py:
 *   - oracle/sphere_oracle.c: a plain-C FP64 restatement of the reference's
 *     DEM step (libsphere_oracle.so);
 *   - oracle/ref_emu/ref_harness.cpp: the reference's own kernels compiled
 *     for the CPU (oracle/_ref/libsphere_ref.so).
 * The product library (sphere_b200) never links or calls either.
 *
 * Arrays use the reference's device layouts (src/datatypes.h:16-37):
 * Float4 = 4 doubles per particle, contact rows of NC slots per particle
 * indexed by the original particle index (src/device.cu:428-432).
 */
#ifndef SPHERE_ORACLE_H_
#define SPHERE_ORACLE_H_

#include <stdint.h>
#include "../include/sphere_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrState {
    SphBox box;            /* grid, params, walls, dt, t_current, np, nb0 */
    int32_t length_mode;   /* SphLengthMode */
    int32_t velocity_state;/* src/device.cu:994, starts at 1 */
    uint64_t iter;         /* TY3 step counter of this run (src/device.cu:919) */
    int32_t error_flags;   /* bit (1 << SphStatus) for each condition seen */
    int32_t nthreads;      /* OpenMP threads (0: default) */
    /* particle state, [np][4] doubles unless noted */
    double *x, *xyzsum, *vel, *force, *angpos, *angvel, *torque, *acc, *angacc;
    double *es_dot, *es, *ev_dot, *ev, *p;          /* [np] */
    /* contact bookkeeping, [np*NC] and [np*NC][4] */
    uint32_t *contacts;
    double *distmod, *delta_t;
    /* bonds: pairs [nb0][2], delta/omega [nb0][4] (xyz tangential, w normal) */
    uint32_t *bonds;
    double *bonds_delta, *bonds_omega;
    uint8_t *bonds_broken;  /* [nb0] bonds broken during this run */
    double walls_acc[SPH_MAXWALLS];
    /* products of the last step / scratch */
    uint32_t *cell_id, *perm, *cell_start, *cell_end;   /* [np],[np],[ncells],[ncells] */
    double *x_sorted, *vel_sorted, *angvel_sorted;      /* [np][4] */
    double *walls_force_pp;                             /* [nw*np] */
    double *walls_force_partial;                        /* [ceil(np/256)] */
    double *tau_eff_x_pp, *tau_eff_x_partial;           /* [np], [ceil(np/256)] */
    struct OrDarcy *darcy;                              /* NULL: fluid == 0 */
} OrState;

/* Darcy coupling (fluid == 1, cfd_solver == 1).  Cell fields are padded
 * with one ghost layer on every side, (nx+2)(ny+2)(nz+2) cells indexed
 * (x+1) + (nx+2)(y+1) + (nx+2)(ny+2)(z+1) (src/darcy.cpp:64-76); vector
 * fields hold three doubles per cell (Float3).  The file clock and the
 * host's copy of the top wall position (refreshed when an output is
 * written) are the reference's host variables (src/device.cu:918, 1001,
 * 1903, 2537, 2569-2672).  The log keeps one entry per fluid step. */
typedef struct OrDarcy {
    SphDarcy prm;
    double *p, *p_old, *p_new, *dp_expl, *phi, *dphi, *norm, *k, *div_v_p;
    double *v, *vp_avg, *grad_k, *grad_p;
    int32_t *p_constant;
    double *f_p;              /* [np][4] */
    double p_top_orig;
    double filetimeclock;
    double wall_w_host;
    uint32_t wall0_iz;
    uint32_t log_cap, log_n;
    uint64_t *log_step;
    uint32_t *log_iters, *log_ok;
} OrDarcy;

/* Run nsteps iterations of the fluid == 0 step loop.  Returns the OR of the
 * error flags raised (0 = clean). */
int or_step(OrState *s, uint64_t nsteps);

/* Analysis (TEST INFRASTRUCTURE ONLY), restated from src/sphere.cpp.
 * x: [np][4] (x, y, z, r); vel: [np][4] (fixvel in w).
 * or_porosity: DEM::porosity (:487-606); returns -1 when a slab is not
 * thicker than 2 r_max (the reference exits), else 0.
 * or_overlaps: DEM::findOverlaps (:677-725); writes up to max_pairs pairs
 * (i, j) and their delta_n, returns the total count. */
int or_porosity(const double *x, uint32_t np, double top, double origo_z, double L0, double L1,
                uint32_t z_slices, double *z_pos, double *porosity);
uint64_t or_overlaps(const double *x, const double *vel, uint32_t np, uint64_t max_pairs,
                     uint32_t *pairs, double *delta_n);
/* Ray tracer (TEST INFRASTRUCTURE ONLY), restated from src/raytracer.cuh:
 * DEM::render (:379-560) with its camera (:291-333) and kernels (:14-288),
 * every sphere tested for every pixel.  x, vel, angvel, angpos, xyzsum:
 * [np][4]; p: [np]; L: grid.L; rgb: width * height * 3 bytes, row-major. */
void or_render(const double *x, const double *vel, const double *angvel, const double *angpos,
               const double *xyzsum, const double *p, uint32_t np, const double *L, int method,
               float maxval, float lower_cutoff, uint32_t width, uint32_t height, uint8_t *rgb);
/* Packing sweeps of the project's scene preparation (sph_relax), restated
 * for one box (TEST INFRASTRUCTURE, and the CPU packer of bench.py's
 * reference arm): x4 [np][4] updated in place, *max_ov = the largest overlap
 * of the last sweep. */
void or_relax(double *x4, uint32_t np, const double origo[3], const double L[3],
              const uint32_t num[3], int periodic, uint32_t sweeps, double alpha, double z_top,
              int nthreads, double *max_ov);
int ref_step(OrState *s, uint64_t nsteps);
/* Darcy set-up at the start of a run (src/device.cu:1003-1016): p_top_orig
 * from the top cell's pressure, the host wall copy from wall 0. */
void or_darcy_start(OrState *s);

#ifdef __cplusplus
}
#endif
#endif
