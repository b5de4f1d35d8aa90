// sph_internal.h -- kernel argument block shared by the step kernels and the
// C-ABI host code.  Not part of the public interface.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "sphere_b200.h"

namespace sph {

struct DevBox;
struct Acc;

// Device pointers of one handle, passed by value to every step kernel.
struct StepArgs {
    DevBox *boxes;
    uint32_t nboxes;
    uint32_t ntot;        // particles over all boxes
    uint64_t ncells;      // cells over all boxes
    uint32_t nbonds;      // bonds over all boxes
    uint32_t npartials;   // per-256-particle partial sums over all boxes
    // particle state, original order
    double4 *x, *vel, *angvel, *angpos, *xyzsum, *acc, *angacc, *force, *torque;
    double *es_dot, *es, *ev_dot, *ev, *p;
    const uint32_t *box_of;
    // cell sort
    uint32_t *cell_id, *local_off, *cell_count, *cell_off, *scan_tmp, *perm, *rank;
    uint32_t *unsorted;        // ids by cell in arrival order (k_scatter)
    double4 *xs, *vs, *ws;     // sorted copies
    float4 *xf;                // sorted FP32 copy of x+r for the candidate prefilter
    // contact rows: slot word = partner | image code << 28, EMPTY when free
    uint32_t *slots;
    double4 *hist;             // tangential displacement per slot (w unused)
    // walls and shear stress
    double *wf_pp, *wall_partial, *tau_pp, *tau_partial;
    const uint32_t *part_owner;
    // bonds
    uint2 *bonds;
    double4 *bdelta, *bomega, *bf, *bt;
    uint8_t *bbroken;
    const uint32_t *bond_box;
    const uint32_t *bcsr_off, *bcsr_ent;
    uint32_t *err;
    // neighbour lists (contact models 2 and 3; vlist null = off): per
    // sphere (original order) up to vcap partner ids in ascending order,
    // vcount = their number (VL_MAX + 1 when the list overflowed: that
    // sphere uses the cell search), xref = position at the list build; cellc = packed cell
    // coordinates of the current step (k_hash); vflag[0] != 0 requests a
    // rebuild before the next contact search, vflag[1] counts rebuilds
    uint32_t *vlist, *vcount, *vflag;
    float4 *xref;
    uint64_t *cellc;
    uint32_t vcap;             // list capacity in use (<= VL_MAX)
    // split step (k_search / k_contacts / k_finish): per warp of 32
    // original indexes, a region of 32 * NC entries holding the warp's live
    // contacts from its start, sphere after sphere, each in slot order
    // (slot word; original index | slot << 27); per sphere their
    // number and the sums of its contacts, all by original index (null until
    // the split step is first used)
    uint2 *lent;
    uint32_t *nlive;
    Acc *csum;
    // adjoint tape of the current step (null outside a recorded segment):
    // contact rows at kernel entry and after the contact search, and the
    // tangential histories the interact pass reads
    uint32_t *tape_rows_pre, *tape_rows_post;
    double4 *tape_hist;
};

constexpr int VL_MAX = 48;   // neighbour-list capacity per sphere
constexpr int INTERACT_VARIANTS = 5;   // launch variants of the interact stage (sph_autotune)
constexpr int SPLIT_VARIANT = 3;       // the split step (k_search / k_contacts / k_finish)
constexpr int PAIR_VARIANT = 4;        // the list step of the FP32-mixed form (sph_pair.cu)
constexpr uint32_t SPLIT_ID_MASK = 0x07ffffffu;   // sphere index bits of a live entry

// The list step of the FP32-mixed form (launch variant 4, sph_pair.cu).
// Its state lives in compact arrays of its own while it steps; the FP64
// arrays of StepArgs are brought up to date from them (pair_flush) before
// anything else reads them, and the compact arrays are loaded from them
// (pair_load) before the first list step after anything wrote them.
//  - ping-pong (selected by *pp: the current step reads [*pp], writes
//    [*pp ^ 1]; k_pair_box flips *pp at the end of the step): what the
//    contact laws read of a partner, x+r in FP64 (xr) and velocity and
//    angular velocity in FP32 (vw: two float4 per sphere, (v, 0) and
//    (w, 0));
//  - the sphere's own state, read and written by its own thread only:
//    velocity+fixvel FP64, angpos, acc, angacc (w: angacc_w), force,
//    torque FP32, es_dot/ev_dot/p FP32 (epp), es/ev FP64 (eacc);
//  - the contact lists, double buffered (selected by *lsel, flipped by a
//    rebuild): per sphere up to VL_MAX neighbour ids in ascending order
//    (ids, cnt), the tangential-displacement history of each entry (hist,
//    three FP64 per entry) and a bit per entry that is set while the pair
//    touches (live);
//  - the wall force of each sphere (A.wf_pp) summed over chunks of
//    PAIR_CHUNK spheres of one box (chunk_part), then per box.
struct PairArgs {
    double4 *xr[2];
    float4 *vw[2];
    double4 *vel;
    float4 *angpos, *acc, *angacc, *force, *torque, *epp;
    double2 *eacc;
    double4 *xyzsum;
    // the lists and histories, entry-major (entry k of every sphere side by
    // side): sphere i's entry k at ids[k * nrow + i], its history component
    // c at hist[(3 k + c) * nrow + i] (nrow = the spheres of the handle), so
    // that the threads of a warp read entry k of their lists from a few
    // lines instead of one line each
    uint32_t *ids[2], *cnt[2];
    uint64_t *live[2];
    double *hist[2];
    uint32_t nrow;
    // the order in which the step kernel's threads take the spheres: within
    // each group of PAIR_ORDER_GROUP consecutive spheres, by list length
    // (built with each list), so that a warp's lists are of similar length
    uint32_t *order[2];
    uint32_t *pp, *lsel;
    uint32_t *from_rows;       // != 0: the next rebuild takes histories from A.slots / A.hist
    uint32_t *bar;             // grid-barrier words of the persistent shapes: count, generation
    double *chunk_part;        // [nchunks]
    const uint32_t *chunk_box; // box of each chunk
    uint32_t nchunks;
    uint32_t chunk_log2;       // chunk = 1 << chunk_log2 spheres of one box
    const uint32_t *box_chunk0;   // first chunk of each box
};
constexpr int PAIR_CHUNK_LOG2 = 11;

// A grid-wide barrier among the blocks of one cooperative launch: arrival
// count and generation words in device memory, and the longest a block
// waits before it gives up (SPH_ERR_TIMEOUT).
struct GridSync {
    uint32_t *count, *gen;
    unsigned long long limit_ns;
};
constexpr unsigned long long BARRIER_LIMIT_NS = 1000000000ull;   // 1 s
constexpr int PAIR_SHAPES = 13;
// Shapes 9 and 10 are the persistent kernel, which does the wall stage
// itself; every other shape is followed by k_pair_chunks and k_pair_box.
inline bool pair_shape_persistent(int shape) { return shape == 9 || shape == 10; }
constexpr int PAIR_ORDER_GROUP = 128;   // launch shapes of the list-step kernel (sph_pair.cu)

// Overlap search of one box (sph_overlaps): positions and velocities, the
// box's spheres [p0, p0 + np), its grid (origin, cell widths, cell counts),
// the search range R in cells, and scratch / output arrays.
struct OverlapArgs {
    const double4 *x, *vel;
    uint32_t p0, np;
    double origo[3], cw[3];
    int num[3], R;
    uint32_t *cell_of, *slot, *count, *coff, *items, *npair, *poff;
    uint32_t *pairs;
    double *delta;
};

// Parts of a step a captured graph holds.  A step ends with the wall stage
// (wall-force partial sums, integrateWalls, time and state of the box),
// which the next step's sort and contact search do not read: in a run of
// steps the wall stage of step t can run beside step t+1 up to its
// integration.  STEP_WHOLE: the whole step; STEP_HEAD: the step without
// its wall stage; STEP_OVERLAP: the previous step's wall stage on the side
// stream beside this step's head, joined before the integration;
// STEP_TAIL: the wall stage alone.
enum StepPhase { STEP_WHOLE = 0, STEP_HEAD = 1, STEP_OVERLAP = 2, STEP_TAIL = 3 };

// The Darcy coupling (fluid == 1, cfd_solver == 1, sph_darcy.cu).  Cell
// fields are padded with one ghost layer on every side, (nx+2)(ny+2)(nz+2)
// cells indexed (x+1) + (nx+2)(y+1) + (nx+2)(ny+2)(z+1) as the reference's
// (src/darcy.cpp:64-76); vector fields hold three doubles per cell.
constexpr uint32_t DARCY_RING = 65536;   // queued top pressures (steps)
struct DarcyState {
    double filetimeclock;          // the reference's host file clock
    double wall_w_host;            // its host copy of walls.nx[0].w (refreshed at outputs)
    unsigned long long qstep;      // steps run since sph_darcy_set (top-pressure ring index)
    unsigned long long log_head;   // Jacobi log entries written
    uint32_t wall0_iz;             // src/device.cu:1001, 1903
    uint32_t active;               // this step runs the fluid update (iter % ndem == 0)
    uint32_t nijac;                // the last iteration of the last solve
};
struct DarcyArgs {
    SphDarcy prm;
    int periodic;                  // grid.periodic of the box
    int nx, ny, nz;
    double dx, dy, dz;
    uint32_t ncell;                // padded cells
    double *p, *p_old, *p_new, *dp_expl, *phi, *dphi, *norm, *k, *div_v_p;
    double *v, *vp_avg, *grad_k, *grad_p;
    int32_t *p_constant;
    double4 *f_p;
    DarcyState *st;
    const double *pmod;            // top pressure per queued step (DARCY_RING), null: no modulation
    uint64_t *log_step;            // the Jacobi log, a ring of SPH_DARCY_LOG entries
    uint32_t *log_iters, *log_ok;
    // the Jacobi loop's cooperative launch: the arrival counter of its grid
    // barrier (zeroed before each launch, only grows during it) and the
    // per-block largest |residual| and NaN flag of a checked iteration
    unsigned long long *bar;
    unsigned long long *part_max;
    uint32_t *part_nan;
    // per interior cell (x fastest), field-major, the parts of the pressure
    // change that stay fixed during a solve (DARCY_COEF doubles per cell)
    double *coef;
};
constexpr int DARCY_COEF = 9;
constexpr uint32_t DARCY_PARTS = 8192;   // blocks of the Jacobi launch at most

struct StepConfig {
    int lenmode;
    bool unfused;     // some box has a shear-stress (wmode 3) top wall
    bool any_walls;   // some box has nw > 0
    int variant = 1;  // interact launch variant (sph_autotune)
    int pair_shape = 0;   // register budget of the list-step kernel (sph_autotune)
    bool all_cm23 = false;   // every box uses contact model 2 or 3
    int phase = STEP_WHOLE;
    cudaStream_t side = nullptr;                       // STEP_OVERLAP only
    cudaEvent_t fork = nullptr, join = nullptr;        // STEP_OVERLAP only
    const DarcyArgs *darcy = nullptr;                  // the Darcy coupling, null: off
};

// Per-kernel timing of an un-graphed step (the counterpart of the
// reference's PROFILING breakdown, src/device.cu:947-987 and 2711-2808):
// an event is recorded on the stream after each kernel.
struct Prof {
    static constexpr int MAX = 32;
    cudaEvent_t ev[MAX + 1];
    const char *name[MAX];
    int n = 0;
};

// The Darcy part of a step (between interact and integrate; needs
// cfg.side under stream capture for the Jacobi loop's body) and the file
// clock after the step's wall stage (sph_darcy.cu).
int launch_darcy(const StepArgs &A, const DarcyArgs &D, const StepConfig &cfg, cudaStream_t st,
                 uint64_t *launches, Prof *prof);
void launch_darcy_tick(const StepArgs &A, const DarcyArgs &D, cudaStream_t st);

// Enqueue one step on `st`; adds the number of kernel launches to
// *launches.  Capturable in a CUDA graph (events in prof become event-record
// nodes).  launch_step runs the FP64 form; launch_step_with takes the
// launcher of the fused interact kernel (FP64 or FP32-mixed variant).
typedef void (*InteractLauncher)(const StepArgs &A, cudaStream_t st, unsigned grid, bool fused,
                                 int lenmode, int variant);
int launch_step(const StepArgs &A, const StepConfig &cfg, cudaStream_t st, uint64_t *launches,
                Prof *prof = nullptr);
typedef void (*ContactLauncher)(const StepArgs &A, cudaStream_t st, unsigned grid, int lenmode,
                                bool pdl);

// Launch kern<<<grid, block, 0, st>>>(args...); with pdl, as a programmatic
// dependent launch: the grid may be scheduled while the kernel before it
// in the stream finishes, and waits (grid_dependency_wait) before reading
// what that kernel wrote.
template <typename... P, typename... Q>
inline void launch_k(bool pdl, void (*kern)(P...), unsigned grid, unsigned block,
                     cudaStream_t st, Q... args)
{
    if (!pdl) {
        kern<<<grid, block, 0, st>>>(args...);
        return;
    }
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3(grid);
    c.blockDim = dim3(block);
    c.dynamicSmemBytes = 0;
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    c.attrs = at;
    c.numAttrs = 1;
    cudaLaunchKernelEx(&c, kern, args...);
}
int launch_step_with(const StepArgs &A, const StepConfig &cfg, cudaStream_t st,
                     uint64_t *launches, Prof *prof, InteractLauncher interact,
                     ContactLauncher contact);
int launch_step_mixed(const StepArgs &A, const StepConfig &cfg, cudaStream_t st,
                      uint64_t *launches, Prof *prof);

// The list step (sph_pair.cu): one step; the public FP64 arrays from the
// compact state and back; the number of touching list entries.
int launch_step_pair(const StepArgs &A, const PairArgs &P, const StepConfig &cfg, cudaStream_t st,
                     uint64_t *launches, Prof *prof);
int pair_load(const StepArgs &A, const PairArgs &P, cudaStream_t st);
int pair_flush(const StepArgs &A, const PairArgs &P, cudaStream_t st);
int pair_count_live(const StepArgs &A, const PairArgs &P, cudaStream_t st,
                    unsigned long long *d_count);
// Self-check of the grid barrier (sph_barrier_check): `rounds` barriers of
// `expected` arrivals among `blocks` resident blocks; error bits in *err.
int barrier_check(uint32_t blocks, uint32_t expected, uint32_t rounds,
                  unsigned long long limit_ns, uint32_t *d_words, uint32_t *d_err,
                  cudaStream_t st);
// Sort and neighbour lists for a rebuild of the list step's lists
// (sph_kernels.cu): the positions of the current state (xr[*pp]) into A.x,
// the cell sort, and the lists into the buffers not in use
// (ids / cnt [*lsel ^ 1]).
void launch_pair_sort_build(const StepArgs &A, const PairArgs &P, cudaStream_t st);

// Ray-traced image of one box (sph_render): tiles of the screen, entries of
// the tile lists, kernels launched.
struct RenderStats {
    uint32_t tiles = 0, entries = 0;
    int launches = 0;
};
// Renders spheres [p0, p0 + np) into d_img (width * height * 3 bytes,
// row-major RGB).  d_L is the box's grid.L in device memory.  Allocates and
// frees its own scratch; synchronises st once (to size the tile lists) and
// at the end.
int render_image(const StepArgs &A, uint32_t p0, uint32_t np, const double *d_L, int method,
                 float maxval, float lower_cutoff, uint32_t width, uint32_t height,
                 uint8_t *d_img, cudaStream_t st, RenderStats *stats);

}  // namespace sph
