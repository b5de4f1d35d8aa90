/*
 * sphere_b200.h -- C ABI of the B200-native DEM time step.
 *
 * The reference (19revey/sphere) has no library boundary for its time step:
 * python/sphere.py:4482-4540 (sim.run) writes input/<sid>.bin and executes the
 * `sphere` binary, whose DEM::startTime loop (src/device.cu:826-2677) runs the
 * step kernels.  This header is the in-process replacement for that process
 * boundary.  Each entry point below names the reference code it replaces.
 *
 * Conventions
 *  - Plain C types only; every pointer is a caller-owned HOST buffer that is
 *    read or written only during the call.
 *  - Array layouts are the .bin v2.15 block layouts (src/file_io.cpp:420-731):
 *    x = [np][4] (x, y, z, radius), vel = [np][4] (vx, vy, vz, fixvel),
 *    xyzsum/force/angpos/angvel/torque = [np][3], energies = [np].
 *  - Every function returns an SphStatus code (0 = OK) and never calls exit().
 *  - One handle is bound to one device and one CUDA stream; calls on a handle
 *    must not overlap.  Handles are independent of each other.
 *  - Several independent boxes ("ensemble") may share one handle: their
 *    particles are concatenated in box order and stepped by the same kernel
 *    launches.  A single simulation is the nboxes == 1 case.
 */
#ifndef SPHERE_B200_H_
#define SPHERE_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH_NC 32          /* contact slots per particle, src/constants.h:21 (NC) */
#define SPH_MAXWALLS 6     /* src/constants.h:12 (MAXWALLS) */
#define SPH_BIN_VERSION 2.15 /* src/version.h:5 (VERSION) */

typedef enum SphStatus {
    SPH_OK = 0,
    SPH_ERR_INPUT = 1,        /* invalid argument or scene (src/sphere.cpp:145-345 checks) */
    SPH_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    SPH_ERR_NC_OVERFLOW = 3,  /* a particle had more than SPH_NC contacts */
    SPH_ERR_OUT_OF_GRID = 4,  /* a particle left the sorting grid */
    SPH_ERR_NAN = 5,          /* a non-finite particle position */
    SPH_ERR_NOMEM = 6,        /* device or host allocation failed */
    SPH_ERR_STATE = 7,        /* call out of order (e.g. step before upload) */
    SPH_ERR_UNSUPPORTED = 8,  /* feature outside this library's scope */
    SPH_ERR_TIMEOUT = 9       /* a device-side wait gave up (the step's state is undefined) */
} SphStatus;

/* Arithmetic of the step. */
typedef enum SphPrecision {
    SPH_PREC_FP64 = 0,   /* all state and contact arithmetic in FP64 */
    SPH_PREC_MIXED = 1   /* FP64 geometry, history and integration; FP32 contact law */
} SphPrecision;

/* How vector lengths are evaluated.  The reference's length()
 * (src/vector_arithmetic.h:317-324) is sqrtf() of an FP64 dot product, i.e. the
 * length is rounded to FP32.  SPH_LEN_REFERENCE reproduces that bit for bit;
 * SPH_LEN_FP64 takes the square root in FP64. */
typedef enum SphLengthMode {
    SPH_LEN_REFERENCE = 0,
    SPH_LEN_FP64 = 1
} SphLengthMode;

/* Global physical parameters: src/datatypes.h:74-101 (struct Params), same
 * field order, without nb0 (a per-box count below). */
typedef struct SphParams {
    double g[3];
    double k_n, k_t, k_r, E;
    double gamma_n, gamma_t, gamma_r;
    double mu_s, mu_d, mu_r;
    double gamma_wn, gamma_wt, mu_ws, mu_wd;
    double rho;
    uint32_t contactmodel;  /* 1, 2 or 3 */
    uint32_t pad0;
    double kappa, db, V_b;
    double lambda_bar, sigma_b, tau_b;
    double sigma0_A, sigma0_f;
} SphParams;

/* Sorting grid: src/datatypes.h:44-50 (struct Grid). */
typedef struct SphGrid {
    double origo[3];
    double L[3];
    uint32_t num[3];
    int32_t periodic;   /* 0: walls, 1: x and y periodic, 2: x periodic */
    int32_t adaptive;   /* 1: L[2] follows wall 0 (src/device.cu:363-393) */
    int32_t pad0;
} SphGrid;

/* Dynamic walls: src/datatypes.h:103-109 (struct Walls).  nx[i] = normal xyz
 * and position; mvfd[i] = mass, velocity, force, normal stress. */
typedef struct SphWalls {
    uint32_t nw;
    int32_t wmode[SPH_MAXWALLS];   /* 0 fixed, 1 stress, 2 velocity, 3 stress + shear */
    uint32_t pad0;
    double nx[SPH_MAXWALLS][4];
    double mvfd[SPH_MAXWALLS][4];
    double tau_x;
} SphWalls;

/* One independent simulation box. */
typedef struct SphBox {
    SphGrid grid;
    SphParams params;
    SphWalls walls;
    double dt;          /* time.dt */
    double t_current;   /* time.current at the start of the next step */
    uint32_t np;        /* particles in this box */
    uint32_t nb0;       /* bonds in this box (params.nb0) */
} SphBox;

/* Host particle arrays (all boxes concatenated), .bin block layouts. */
typedef struct SphParticles {
    double *x;       /* [np][4] */
    double *xyzsum;  /* [np][3] */
    double *vel;     /* [np][4] */
    double *force;   /* [np][3] */
    double *angpos;  /* [np][3] */
    double *angvel;  /* [np][3] */
    double *torque;  /* [np][3] */
    double *es_dot, *es, *ev_dot, *ev, *p;  /* [np] */
} SphParticles;

/* Host bond arrays (all boxes concatenated), .bin layouts
 * (src/file_io.cpp:228-250).  Particle indexes are local to the box. */
typedef struct SphBonds {
    uint32_t *pairs;   /* [nb0][2] */
    double *delta_n;   /* [nb0] */
    double *delta_t;   /* [nb0][3] */
    double *omega_n;   /* [nb0] */
    double *omega_t;   /* [nb0][3] */
} SphBonds;

typedef struct SphHandle SphHandle;

/* Create a handle for `nboxes` boxes on CUDA device `device` (-1: current).
 * Replaces DEM::DEM + initializeGPU + transferToConstantDeviceMemory +
 * allocateGlobalDeviceMemory (src/sphere.cpp:16-95, src/device.cu:58-480),
 * with checkValues (src/sphere.cpp:145-345) applied to every box. */
int sph_create(const SphBox *boxes, uint32_t nboxes, int precision,
               int length_mode, int device, SphHandle **out);

/* Copy particle (and bond, may be NULL when no box has bonds) state to the
 * device; contact lists are emptied and tangential histories zeroed.
 * Replaces transferToGlobalDeviceMemory (src/device.cu:660-746).  The
 * input is checked as checkValues does (src/sphere.cpp:145-345) while the
 * copies run; when a check fails (SPH_ERR_INPUT) the handle holds no
 * particle state until an upload succeeds (sph_step: SPH_ERR_STATE).  The
 * caller's arrays are only read during the call. */
int sph_upload(SphHandle *h, const SphParticles *p, const SphBonds *b);

/* Run `nsteps` iterations of the DEM::startTime loop body for fluid == 0
 * (src/device.cu:1039-1200 and 2423-2538): cell hash, sort, reorder,
 * topology, interact, bonds, integrate, wall sums and integrateWalls, then
 * time.current += dt.  Returns the first device error seen in these steps;
 * a step that overflowed a contact list is still completed. */
int sph_step(SphHandle *h, uint64_t nsteps);

/* As sph_step, without waiting: the steps are queued on the handle's stream
 * and their device errors are reported by the next sph_sync or sph_step. */
int sph_step_async(SphHandle *h, uint64_t nsteps);

/* Wait for queued steps; returns the first device error they raised. */
int sph_sync(SphHandle *h);

/* Run the steps on `cuda_stream` (a cudaStream_t of the handle's device)
 * instead of the handle's own stream; NULL restores the own stream.  The
 * legacy default stream has the handle value NULL too, so a caller that
 * wants ordering with its own work passes a stream it created. */
int sph_set_stream(SphHandle *h, void *cuda_stream);

/* Per-kernel timing, the counterpart of the reference's PROFILING
 * breakdown (src/device.cu:947-987, 2711-2808).  While enabled, steps run
 * from a ring of 8 captured step graphs that record CUDA events between
 * kernels; sph_profile_read returns the mean milliseconds per kernel group
 * over the (up to 8) most recent steps in ms[] and the groups' names as a
 * comma-separated list in names. */
int sph_profile(SphHandle *h, int enable);
int sph_profile_read(SphHandle *h, char *names, size_t names_len, double *ms,
                     int max_kernels, int *nkernels);

/* Output-cadence driver for a single box, replacing the loop control of
 * src/device.cu:1031, 2536-2537 and 2569: runs steps while
 * *time_current <= time_total, adding dt to *time_current and *filetimeclock
 * after each step exactly as the reference does, and returns after the step
 * where *filetimeclock >= file_dt (the caller then writes an output file and
 * zeroes *filetimeclock) or when the run is over.  *steps_done receives the
 * number of steps run; at most max_steps are run. */
int sph_advance(SphHandle *h, double time_total, double file_dt,
                double *time_current, double *filetimeclock,
                uint64_t max_steps, uint64_t *steps_done);

/* Copy the current particle/bond state to host arrays (any pointer may be
 * NULL to skip it).  Replaces transferFromGlobalDeviceMemory
 * (src/device.cu:747-822). */
int sph_download(SphHandle *h, SphParticles *p, SphBonds *b);

/* Current per-box grid, walls and time (wall positions, velocities and
 * forces after integrateWalls; L[2] after an adaptive-grid update). */
int sph_get_boxes(SphHandle *h, SphBox *boxes);

/* The same box state read back without waiting (no counterpart in the
 * reference, whose loop stops for every read).  A state is the raw device
 * box table, sph_box_state_bytes long.  sph_get_boxes_async queues, on the
 * handle's stream after the steps queued so far, a copy of it into
 * `staging`; sph_step_async_states queues nsteps steps as sph_step_async
 * does and the state after step s into states + s * sph_box_state_bytes
 * (states_bytes >= nsteps times that).  Pinned host memory keeps the copies
 * asynchronous.  After sph_sync, sph_boxes_from_staging turns nstates
 * consecutive states into nstates x nbox SphBox records (state-major), as
 * sph_get_boxes returns them.  Lets a caller read
 * every step's result while the steps run back to back. */
int sph_box_state_bytes(const SphHandle *h, uint64_t *bytes);
int sph_get_boxes_async(SphHandle *h, void *staging, uint64_t staging_bytes);
int sph_step_async_states(SphHandle *h, uint64_t nsteps, void *states, uint64_t states_bytes);
int sph_boxes_from_staging(SphHandle *h, const void *staging, uint64_t nstates, SphBox *boxes);

/* Contact bookkeeping in the reference's slot form (src/device.cu:428-432):
 * contacts [np][NC] (partner index local to the box, np_box = empty),
 * delta_t [np][NC][4], distmod [np][NC][4] (periodic shift xyz, partner
 * radius).  Any pointer may be NULL. */
int sph_get_contacts(SphHandle *h, uint32_t *contacts, double *delta_t,
                     double *distmod);
/* The inverse of sph_get_contacts, after sph_upload (no counterpart in the
 * reference, whose .bin files carry no contact history, so that a restart
 * begins with empty contact lists): contacts [np][NC] (partner index local
 * to the box, np_box = empty slot) and delta_t [np][NC][4] (NULL: zero
 * histories) become the handle's contact rows; each pair's periodic image
 * is the nearest one at the current positions.  A partner index that is
 * not a sphere of the box, or the sphere itself, is SPH_ERR_INPUT and
 * changes nothing. */
int sph_set_contacts(SphHandle *h, const uint32_t *contacts, const double *delta_t);

/* Cell-sort products of the last step (src/sorting.cuh:25-132,
 * src/device.cu:1059-1107): per-particle cell id [np] (in original order),
 * sorted permutation [np] (gridParticleIndex), cellStart/cellEnd
 * [total cells] with 0xffffffff for empty cells.  Indexes are global over
 * the concatenated boxes; cell ids are offset by the box's first cell. */
int sph_get_sort(SphHandle *h, uint32_t *cell_id, uint32_t *perm,
                 uint32_t *cell_start, uint32_t *cell_end);
uint64_t sph_total_cells(const SphHandle *h);

/* Live directed contacts after the last step (each pair counted twice,
 * once per particle row); used for the roofline byte count. */
int sph_count_contacts(SphHandle *h, uint64_t *ncontacts);

/* Kernel launches issued by this handle since creation. */
uint64_t sph_kernel_launches(const SphHandle *h);

/* Scene preparation (no counterpart in the reference's step; it stands in
 * for the long gravity-settling runs sphere's scripts use to make dense
 * packs): `sweeps` Jacobi sweeps of geometric overlap removal on the
 * uploaded positions -- each overlapping pair is pushed apart by alpha/2 of
 * its overlap per sweep, spheres are kept between the floor and z_top.
 * *max_overlap receives the largest overlap of the last sweep.  Velocities
 * and contact lists are untouched; download the positions afterwards. */
int sph_relax(SphHandle *h, uint32_t sweeps, double alpha, double z_top,
              double *max_overlap);

/* Differentiable steps (no counterpart in the reference).
 *
 * sph_adjoint_forward runs `nsteps` steps as sph_step does and keeps a
 * device checkpoint of the full state at the start of every `ckpt` steps
 * and at the end (held by the handle until the backward pass or
 * sph_destroy).  forward_ms (may be NULL) gets the device time.
 *
 * sph_adjoint_backward takes dx_final [np][3] = dLoss/d(final positions)
 * and returns grad_params[3] = dLoss/dk_n, dLoss/dgamma_n, dLoss/dmu (mu_s
 * and mu_d tied; k_t held fixed) and grad_v0 [np][3] = dLoss/d(velocities
 * at the start of the forward); either may be NULL.  Each segment is
 * recomputed from its checkpoint while a tape of the contact rows and
 * tangential histories is recorded, then its steps are reversed with the
 * contact set of each step frozen and each contact law differentiated on
 * the branch it took (normal force on/off, stick/slip).  adjoint_ms gets
 * the device time of recompute + reverse; the CUDA graphs of the segments
 * (one per segment length and kind) are captured before that time is
 * taken, as the forward's step graph is built before forward_ms is taken.
 * Afterwards the handle holds the
 * forward's final state and the checkpoints are released.
 *
 * Scope: one box, SPH_PREC_FP64 with SPH_LEN_FP64, contact model 2, E = 0,
 * kappa = 0, no bonds, no dynamic walls, fixed grid (adaptive 0),
 * gamma_wt = 0 (SPH_ERR_UNSUPPORTED otherwise). */
int sph_adjoint_forward(SphHandle *h, uint64_t nsteps, uint32_t ckpt, double *forward_ms);
int sph_adjoint_backward(SphHandle *h, const double *dx_final, double *grad_params,
                         double *grad_v0, double *adjoint_ms);

/* Neighbour lists of the contact search (contact models 2 and 3; no
 * counterpart in the reference, whose search scans the 27 neighbour cells
 * every step): each sphere keeps the ids of the spheres within
 * r_a + r_b + 0.1 r_min, rebuilt when a sphere has moved half that skin;
 * the contacts found, and their order, are those of the cell search.
 * capacity = list entries per sphere (1..48, default 48; a sphere with
 * more neighbours uses the cell search), 0 = lists off (cell search for
 * all).  Takes effect at the next step. */
int sph_set_neighbor_lists(SphHandle *h, uint32_t capacity);
/* stats[5] as of the last step: spheres using their list, spheres whose
 * list overflowed (they use the cell search), list entries in use, longest
 * list, list builds so far. */
int sph_neighbor_stats(SphHandle *h, uint64_t *stats);

/* Launch variants of the interact stage (no counterpart in the
 * reference).  0, 1, 2 = the fused kernel compiled for up to 255, 128 and
 * 80 registers per thread (different occupancy); 3 = the split step
 * (contact search, one thread per contact for the contact laws, one thread
 * per sphere for the sums and integration), for contact models 2 and 3
 * with neighbour lists on, which allocates 332 B per sphere when first
 * chosen.  Variants 0-3 have the same arithmetic and results.
 * 4 = the list step of the FP32-mixed form (SPH_PREC_MIXED only; contact
 * models 2 and 3, neighbour lists on, no bonds, no shear-stress wall, no
 * adaptive grid; other handles run variant 1 when it is chosen): the
 * tangential history of a touching pair is kept with its neighbour-list
 * entry instead of an NC slot, each sphere's contacts are summed in list
 * order, and one kernel per step runs the contact laws, walls and
 * integration on compact state (FP32 where the mixed form allows); it
 * allocates about 2.7 kB per sphere when first chosen.  Its contacts are
 * those of the other variants (the same FP64 overlap test); sph_get_contacts
 * returns them in list order in slots 0, 1, ...; its results are held to
 * the mixed form's stated error, not to the other variants' bits.
 * sph_autotune times `steps` steps with each applicable variant from the
 * current state, keeps the fastest for this handle and puts the state back
 * as it was (ms_per_step[SPH_TUNE_VARIANTS] may be NULL; -1 for a variant
 * not tried).  sph_set_variant picks one directly.  Default 1. */
#define SPH_TUNE_VARIANTS 5
int sph_autotune(SphHandle *h, uint32_t steps, double *ms_per_step, int *chosen);
int sph_set_variant(SphHandle *h, int variant);
/* Launch shape of the list step (variant 4): threads per block x resident
 * blocks per SM, i.e. its register budget, and for shapes 5-8 the number
 * of list entries whose partner data each thread has in flight (staged in
 * shared memory) -- 0: 128 x 4, 1: 128 x 5, 2: 128 x 6, 3: 64 x 8,
 * 4: 256 x 2, 5: 64 x 8 staging 4, 6: 64 x 8 staging 6, 7: 128 x 4
 * staging 4, 8: 64 x 10 staging 3, 9: persistent 64 x 8, 10: persistent
 * 128 x 4; shapes 11 and 12 load each list entry at its turn instead of
 * one entry ahead (fewer registers, more resident warps) -- 11: 64 x 10,
 * 12: 64 x 12 (SPH_PAIR_SHAPES).  The results do
 * not depend on the shape.  sph_autotune tries every shape of variant 4
 * and reports the best in ms_per_step[4]; sph_get_tuning returns the
 * variant and shape in use. */
#define SPH_PAIR_SHAPES 13
int sph_set_launch_shape(SphHandle *h, int shape);
int sph_get_tuning(const SphHandle *h, int *variant, int *shape);
/* The last sph_autotune's time per step (ms) of the list step at each
 * launch shape, into ms[0 .. n-1] (-1: not tried, or past
 * SPH_PAIR_SHAPES).  sph_autotune times every candidate twice, in two
 * rounds over all of them, and keeps each one's better time. */
int sph_get_shape_times(const SphHandle *h, double *ms, int n);

/* Shapes 9 (64 x 8) and 10 (128 x 4) of the list step are persistent: one
 * cooperative launch per step whose blocks (all resident) take the spheres
 * in turn, then meet at a grid-wide barrier, sum the wall forces, meet
 * again and advance the walls.  A block waits at a barrier at most 1 s; a
 * wait that runs out raises SPH_ERR_TIMEOUT (the launch ends, the device
 * stays usable, the handle needs sph_upload).  sph_barrier_check runs
 * `rounds` such barriers among `blocks` resident blocks of 32 threads on
 * the current device, each waiting for `expected` arrivals for at most
 * limit_s seconds: SPH_OK when they all open, SPH_ERR_TIMEOUT when
 * expected > blocks (no barrier can open; every block gives up after the
 * limit), SPH_ERR_INPUT for blocks outside 1 .. the number of SMs or a
 * limit outside (0, 10] s. */
int sph_barrier_check(uint32_t blocks, uint32_t expected, uint32_t rounds, double limit_s);

/* Output snapshot, the output path of the reference's loop
 * (transferFromGlobalDeviceMemory before each output file,
 * src/device.cu:747-822 and 2569-2590) without stopping the steps:
 * sph_snapshot enqueues on the handle's stream, after the steps already
 * queued, a device copy of everything sph_download and sph_get_boxes
 * return, and returns at once; steps queued later do not change it.
 * sph_snapshot_read waits for that copy only (not for later steps) and
 * fills p and b as sph_download and boxes[nboxes] as sph_get_boxes (each
 * may be NULL); it returns the first device error raised by the steps
 * before the snapshot and after the previous one.  One snapshot is held at
 * a time; a new sph_snapshot replaces an unread one.  The copies take
 * 272 B per sphere and 72 B per bond of device memory, allocated at the
 * first call. */
int sph_snapshot(SphHandle *h);
int sph_snapshot_read(SphHandle *h, SphParticles *p, SphBonds *b, SphBox *boxes);

/* Porosity profile of box `box` in z_slices horizontal slabs from the
 * current state: DEM::porosity (src/sphere.cpp:487-606, the reference's
 * `porosity` program), the same arithmetic in the same order; the top is
 * wall 0's position when the box has walls, else L[2].  z_pos and porosity
 * are host arrays of z_slices.  Slabs not thicker than 2 r_max:
 * SPH_ERR_INPUT (the reference exits). */
int sph_porosity(SphHandle *h, uint32_t box, uint32_t z_slices, double *z_pos, double *porosity);

/* Overlapping sphere pairs of box `box` in the current state:
 * DEM::findOverlaps (src/sphere.cpp:677-725, behind `sphere --contacts`):
 * pairs (i, j) of box-local indexes with i < j, ascending in i then j,
 * |x_j - x_i| - (r_i + r_j) < 0 without periodic images, both spheres free
 * (fixvel 0), delta_n = that distance.  Writes up to max_pairs entries of
 * pairs [max_pairs][2] and delta_n [max_pairs] (either may be NULL) and the
 * total count in *npairs. */
int sph_overlaps(SphHandle *h, uint32_t box, uint64_t max_pairs, uint32_t *pairs, double *delta_n,
                 uint64_t *npairs);

/* Ray-traced image of box `box` in the current state: DEM::render
 * (src/raytracer.cuh:379-560, behind `sphere --render`) with its camera
 * (eye at (2.3 L0, -5 L1, 1.3 L2), looking at maxPos()/2, image plane
 * 1.35 L0 wide), its rays (including the row index taken modulo the width)
 * and its shading.  method: 0 uniform colour, 1 pressure, 2 |vel|,
 * 3 |angvel|, 4 xyzsum.x, 5 |angpos| (colour map from 0 to maxval);
 * lower_cutoff > 0 hides spheres of methods 1-5 at or below it and spheres
 * with a fixed velocity.  focal_length is accepted and unused, as in the
 * reference.  rgb: host array of width * height * 3 bytes, written row by
 * row (the body of the reference's PPM file, src/file_io.cpp:734-757).
 * Arithmetic: the reference's FP32 expressions in its order, without FMA
 * contraction, with IEEE division and square root and a normalisation by
 * 1 / sqrtf.  Other methods or a zero width or height: SPH_ERR_INPUT. */
int sph_render(SphHandle *h, uint32_t box, int method, float maxval, float lower_cutoff,
               float focal_length, uint32_t width, uint32_t height, uint8_t *rgb);

/* Message of the last error on this handle (or a static message for a NULL
 * handle).  Returns the number of characters written. */
int sph_last_error(const SphHandle *h, char *buf, size_t n);
const char *sph_status_string(int status);

void sph_destroy(SphHandle *h);

/* sizeof of SphParams, SphGrid, SphWalls, SphBox, SphParticles, SphBonds
 * (6 entries), for binding checks. */
int sph_struct_sizes(uint64_t *sizes);

/* Cell-offset scan that allocates nothing (no counterpart in the
 * reference; it is the cellStart/cellEnd construction of the contact
 * search, src/sorting.cuh:56-116 reorderArrays, as a stand-alone call):
 * offsets[k] = counts[0] + ... + counts[k-1] for k = 0..n (n + 1 words;
 * offsets[n] is the total), on device pointers, enqueued on `stream` (a
 * cudaStream_t of the current device, else SPH_ERR_INPUT; NULL = default
 * stream).  For callers that must not allocate device
 * memory at the call (a framework that owns all device memory, a
 * steady-state loop where an allocation could block or fail): the scratch
 * is a fixed file-scope device array of SPH_SCAN_STATIC_MAX / 4096 + 1
 * words (16 KiB + 4 B), so n > SPH_SCAN_STATIC_MAX returns
 * SPH_ERR_UNSUPPORTED.  The scratch needs no initial value.  The first call
 * on each device (and the first after a device reset) looks up the array's
 * address with the device current (cudaGetSymbolAddress, which may load
 * the module, and the driver may allocate device memory for it): make that
 * first call at initialisation, before any stream capture begins; later
 * calls allocate nothing.  Calls on one device share the array, so calls
 * that may overlap in time (other streams or host threads without ordering
 * between them) race and give wrong offsets. */
#define SPH_SCAN_STATIC_MAX 16777216u
int sph_cell_offsets_static(const uint32_t *counts, uint64_t n, uint32_t *offsets, void *stream);

/* Darcy flow coupling (fluid == 1, cfd_solver == 1): the Darcy struct of
 * src/datatypes.h:157-190 without its arrays, plus the output interval.
 * Boundary codes as the reference's: 0 fixed pressure (Dirichlet), 1 no
 * flow (Neumann), 2 periodic, 4 prescribed flux (bot/top only). */
typedef struct SphDarcy {
    double mu;            /* fluid dynamic viscosity */
    double rho_f;         /* fluid density */
    double beta_f;        /* adiabatic fluid compressibility */
    double k_c;           /* Kozeny-Carman permeability prefactor */
    double c_phi;         /* porosity scaling coefficient */
    double tolerance;     /* largest normalized residual of a converged solve */
    double p_mod_A;       /* top pressure modulation: amplitude, */
    double p_mod_f;       /* frequency */
    double p_mod_phi;     /* and phase */
    double bc_bot_flux;   /* normal flux through the bottom (bc_bot == 4) */
    double bc_top_flux;   /* and the top (bc_top == 4) */
    double file_dt;       /* time.file_dt: the output interval */
    uint32_t maxiter;     /* Jacobi iterations per fluid step at most */
    uint32_t ndem;        /* DEM steps per fluid step */
    int32_t bc_xn, bc_xp, bc_yn, bc_yp, bc_bot, bc_top;
    int32_t free_slip_bot, free_slip_top;   /* kept for the .bin file only */
} SphDarcy;

/* Turn the Darcy coupling on for a one-box FP64 handle and set its state.
 * The fluid grid is the box's cell grid (nx, ny, nz = grid.num, not
 * adaptive); p, phi, dphi and p_constant hold nx*ny*nz cells and v three
 * doubles per cell, x fastest (the .bin fluid block order,
 * src/file_io.cpp:347-404); f_p is [np][3] (may be NULL: zero).  Replaces
 * initDarcyMem + initDarcyMemDev + transferDarcyToGlobalDeviceMemory and
 * the start-of-run set-up of DEM::startTime (src/darcy.cpp:17-36,
 * src/darcy.cuh:17-104, src/device.cu:1003-1016).  From then on every step
 * runs the Darcy part of the step loop (src/device.cu:1891-2419) between
 * interact and integrate: the pressure force on the spheres, and every ndem
 * steps the porosities, permeabilities, the Jacobi solve of the pressure
 * (on the device: no host round trip per iteration) and the velocities.
 * The file clock and the host's copy of the top wall position that the
 * reference keeps (refreshed at each output) are kept on the device from
 * this call on, so that results do not depend on how the steps are split
 * into calls.  SPH_ERR_UNSUPPORTED for more than one box, the FP32-mixed
 * form or an adaptive grid. */
int sph_darcy_set(SphHandle *h, const SphDarcy *d, const double *p, const double *v,
                  const double *phi, const double *dphi, const int32_t *p_constant,
                  const double *f_p);

/* The fluid state after the steps run so far (any pointer may be NULL):
 * p, phi, dphi, k [cells], v [cells][3], f_p [np][3].  Replaces
 * transferDarcyFromGlobalDeviceMemory (src/darcy.cuh:106-129). */
int sph_darcy_get(SphHandle *h, double *p, double *v, double *phi, double *dphi, double *k,
                  double *f_p);

/* The Jacobi solves since the last call, one entry per fluid step: the
 * step (iter + 1, as the reference's conv.log writes it), the iterations
 * run (the last nijac) and whether the solve converged.  Up to
 * SPH_DARCY_LOG entries are kept between calls (older ones are dropped);
 * *n receives the number written (at most cap).  The reference writes
 * "step nijac" to output/<sid>-conv.log for converged solves at every
 * tenth step and for every solve that did not converge
 * (src/device.cu:2349-2370). */
#define SPH_DARCY_LOG 4096u
int sph_darcy_log(SphHandle *h, uint64_t *step, uint32_t *iterations, uint32_t *converged,
                  uint32_t cap, uint32_t *n);

/* sizeof(SphDarcy), for binding checks. */
int sph_darcy_struct_size(uint64_t *size);

#ifdef __cplusplus
}
#endif
#endif /* SPHERE_B200_H_ */
