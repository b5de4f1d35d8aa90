// sph_capi.cu -- C ABI of include/sphere_b200.h: handle, device memory,
// host<->device transfers and the CUDA-graph step driver.
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sph_device.cuh"
#include "sph_internal.h"

using sph::DevBox;
using sph::StepArgs;
using sph::StepConfig;

namespace sph {
int count_live_slots(const StepArgs &A, cudaStream_t st, unsigned long long *d_count,
                     uint64_t *launches);
int launch_step_mixed(const StepArgs &A, const StepConfig &cfg, cudaStream_t st,
                      uint64_t *launches, Prof *prof);
int relax_sweep(const StepArgs &A, cudaStream_t st, double alpha, double z_top,
                unsigned long long *d_max, uint64_t *launches);
int porosity_profile(const double4 *x, uint32_t p0, uint32_t np, double h_slice, double V_slice,
                     uint32_t nslices, double *z_pos, double *por, cudaStream_t st);
int find_overlaps(OverlapArgs O, uint32_t ncells, uint32_t *scan_tmp, cudaStream_t st, int stage);
int adjoint_step(const DevBox *box, uint32_t n, uint64_t iter, const double4 *x,
                 const double4 *vel, const double4 *angvel, const uint32_t *rows_pre,
                 const uint32_t *rows_post, const double4 *hist, const double4 *const lnext[5],
                 double4 *const lcur[5], double4 *lH, double *gparam, cudaStream_t st);
}

struct SphHandle {
    int device = 0;
    cudaStream_t stream = nullptr;   // stream the steps run on (own or caller's)
    cudaStream_t own = nullptr;      // stream created by the handle (graph capture)
    int precision = SPH_PREC_FP64;
    int lenmode = SPH_LEN_REFERENCE;
    std::vector<SphBox> boxes;       // as created
    std::vector<DevBox> dbox;        // host image of the device box table
    std::vector<double> t_host;      // host mirror of each box's time.current
    uint32_t nbox = 0;
    uint64_t ntot = 0, ncells = 0, nbonds = 0, npartials = 0;
    StepArgs A{};
    StepConfig cfg{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    // runs of steps: head of the first step, then steps that overlap the
    // previous step's wall stage (side stream), then the last wall stage
    // (indexed by sph::StepPhase; [0] unused)
    cudaGraph_t pgraph_ph[4] = {};
    cudaGraphExec_t pexec_ph[4] = {};
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    uint64_t launches_per_step = 0;
    uint64_t launches = 0;
    // the last sph_autotune's time per step of the list step at each launch
    // shape (-1: not tried)
    double shape_ms[sph::PAIR_SHAPES] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
    static_assert(sph::PAIR_SHAPES == 13, "one initial value per launch shape");
    // profiling: a ring of captured step graphs with event-record nodes
    static constexpr int PR = 8;
    bool prof_on = false;
    cudaGraph_t pgraph[PR] = {};
    cudaGraphExec_t pexec[PR] = {};
    sph::Prof prof[PR];
    bool prof_events = false;
    int pnext = 0;
    uint64_t pcount = 0;
    bool uploaded = false;
    std::string err;
    std::vector<void *> allocs;
    unsigned long long *d_count = nullptr;
    uint32_t *vlist_mem = nullptr;   // neighbour-list storage (A.vlist is null when off)
    std::vector<double> rmax_box;    // largest radius per box (at upload)
    double *stage = nullptr;         // [np][3] staging of the host 3-vector layout
    // output snapshot (sph_snapshot): device copies of what sph_download and
    // sph_get_boxes return, the error word, an event after the copies and a
    // stream for reading them back
    StepArgs snap{};
    bool snap_alloc = false, snap_pending = false;
    cudaEvent_t snap_ev = nullptr;
    cudaStream_t snap_stream = nullptr;
    // adjoint: checkpoints of the last sph_adjoint_forward (null when none)
    char *adj_snaps = nullptr;
    uint64_t adj_nsteps = 0, adj_iter0 = 0;
    uint32_t adj_ckpt = 0;
    // the list step of the FP32-mixed form (launch variant 4): its compact
    // state (allocated when the variant is first chosen); pair_valid: the
    // compact arrays hold the current state; pair_ahead: the FP64 arrays
    // of A are behind them (brought up to date by sync_public)
    sph::PairArgs P{};
    bool pair_alloc = false, pair_valid = false, pair_ahead = false;
    // steps launched kernel by kernel instead of as captured graphs
    // (SPHERE_B200_EAGER=1 at sph_create): for profilers that cannot see
    // into graphs with conditional nodes; the list step then reads its
    // rebuild request on the host each step
    bool eager = false;
    // the Darcy coupling (sph_darcy_set): its device fields and state
    // (D.st null until set), the host mirror of the device's step count
    // (the top-pressure ring index), the Jacobi log entries read so far and
    // the top pressure at the start of the run
    sph::DarcyArgs D{};
    bool darcy_on = false;
    uint64_t darcy_qstep = 0, darcy_log_tail = 0;
    double darcy_p_top_orig = 0.0;
};

static int fail(SphHandle *h, int code, const std::string &msg)
{
    if (h) h->err = msg;
    return code;
}

#define CUDA_TRY(h, call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), e_ == cudaErrorMemoryAllocation ? SPH_ERR_NOMEM : SPH_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                \
    } while (0)

template <typename T>
static int dalloc(SphHandle *h, T **p, uint64_t count)
{
    if (count == 0) count = 1;
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * count);
    if (e != cudaSuccess)
        return fail(h, SPH_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    h->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return SPH_OK;
}

// Whether the list step (launch variant 4) can run this handle: the
// FP32-mixed form, contact models 2/3 in every box, no shear-stress wall,
// no bonds, no adaptive grid, neighbour lists on and possible in every
// populated box (set at sph_upload).
static bool pair_eligible(const SphHandle *h)
{
    if (h->precision != SPH_PREC_MIXED || !h->cfg.all_cm23 || h->cfg.unfused || !h->A.vlist ||
        h->nbonds != 0 || h->ntot == 0 || !h->uploaded)
        return false;
    for (uint32_t k = 0; k < h->nbox; ++k) {
        if (h->boxes[k].grid.adaptive) return false;
        if (h->dbox[k].np > 0 && h->dbox[k].vrange < 1) return false;
    }
    return true;
}

static bool pair_active(const SphHandle *h)
{
    return h->cfg.variant == sph::PAIR_VARIANT && pair_eligible(h);
}

static int ensure_pair(SphHandle *h)
{
    if (h->pair_alloc) return SPH_OK;
    const uint64_t n = h->ntot;
    sph::PairArgs &P = h->P;
    std::vector<uint32_t> cbox, c0(h->nbox);
    for (uint32_t k = 0; k < h->nbox; ++k) {
        c0[k] = (uint32_t)cbox.size();
        const uint32_t nch = (h->dbox[k].np + (1u << sph::PAIR_CHUNK_LOG2) - 1) >> sph::PAIR_CHUNK_LOG2;
        for (uint32_t c = 0; c < nch; ++c) cbox.push_back(k);
    }
    uint32_t *chunk_box = nullptr, *box_chunk0 = nullptr, *words = nullptr;
    int st;
    if ((st = dalloc(h, &P.xr[0], n)) || (st = dalloc(h, &P.xr[1], n)) ||
        (st = dalloc(h, &P.vw[0], 2 * n)) || (st = dalloc(h, &P.vw[1], 2 * n)) ||
        (st = dalloc(h, &P.vel, n)) || (st = dalloc(h, &P.angpos, n)) ||
        (st = dalloc(h, &P.acc, n)) || (st = dalloc(h, &P.angacc, n)) ||
        (st = dalloc(h, &P.force, n)) || (st = dalloc(h, &P.torque, n)) ||
        (st = dalloc(h, &P.epp, n)) || (st = dalloc(h, &P.eacc, n)) ||
        (st = dalloc(h, &P.xyzsum, n)) ||
        (st = dalloc(h, &P.ids[0], n * sph::VL_MAX)) || (st = dalloc(h, &P.ids[1], n * sph::VL_MAX)) ||
        (st = dalloc(h, &P.cnt[0], n)) || (st = dalloc(h, &P.cnt[1], n)) ||
        (st = dalloc(h, &P.live[0], n)) || (st = dalloc(h, &P.live[1], n)) ||
        (st = dalloc(h, &P.order[0], n)) || (st = dalloc(h, &P.order[1], n)) ||
        (st = dalloc(h, &P.hist[0], 3 * n * sph::VL_MAX)) ||
        (st = dalloc(h, &P.hist[1], 3 * n * sph::VL_MAX)) || (st = dalloc(h, &words, 5)) ||
        (st = dalloc(h, &P.chunk_part, cbox.size())) || (st = dalloc(h, &chunk_box, cbox.size())) ||
        (st = dalloc(h, &box_chunk0, h->nbox)))
        return st;
    P.pp = words;
    P.lsel = words + 1;
    P.from_rows = words + 2;
    P.bar = words + 3;
    P.chunk_box = chunk_box;
    P.box_chunk0 = box_chunk0;
    P.nchunks = (uint32_t)cbox.size();
    P.chunk_log2 = sph::PAIR_CHUNK_LOG2;
    P.nrow = (uint32_t)n;
    CUDA_TRY(h, cudaMemset(words, 0, 5 * sizeof(uint32_t)));
    for (int b = 0; b < 2; ++b) {
        CUDA_TRY(h, cudaMemset(P.cnt[b], 0, sizeof(uint32_t) * n));
        CUDA_TRY(h, cudaMemset(P.live[b], 0, sizeof(uint64_t) * n));
    }
    if (!cbox.empty())
        CUDA_TRY(h, cudaMemcpy(chunk_box, cbox.data(), 4 * cbox.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(box_chunk0, c0.data(), 4 * c0.size(), cudaMemcpyHostToDevice));
    h->pair_alloc = true;
    return SPH_OK;
}

// Bring the FP64 arrays of A up to date with the list step's compact state
// (before anything reads them); synchronises the handle's stream.
static int sync_public(SphHandle *h)
{
    if (!h->pair_ahead) return SPH_OK;
    int st = sph::pair_flush(h->A, h->P, h->stream);
    if (st != SPH_OK) return fail(h, st, "list-step state flush failed");
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->pair_ahead = false;
    return SPH_OK;
}

// The FP64 arrays were written: the compact state no longer holds the
// current state.
static void invalidate_pair(SphHandle *h)
{
    h->pair_valid = false;
    h->pair_ahead = false;
}

// Before steps of the active launch variant are queued: the list step
// loads its compact state when that is stale; every other variant needs
// the FP64 arrays current, and leaves the compact state stale.
static int prepare_steps(SphHandle *h)
{
    if (pair_active(h)) {
        int st = ensure_pair(h);
        if (st != SPH_OK) return st;
        if (!h->pair_valid) {
            st = sph::pair_load(h->A, h->P, h->stream);
            if (st != SPH_OK) return fail(h, st, "list-step state load failed");
            h->pair_valid = true;
        }
        h->pair_ahead = true;
        return SPH_OK;
    }
    int st = sync_public(h);
    if (st != SPH_OK) return st;
    h->pair_valid = false;
    return SPH_OK;
}

// src/sphere.cpp:145-345 checkValues, parts that do not need particle data.
static int check_box(SphHandle *h, const SphBox &b, uint32_t k)
{
    char buf[256];
    const SphGrid &g = b.grid;
    if (g.origo[0] < 0.0 || g.origo[1] < 0.0 || g.origo[2] < 0.0) {
        snprintf(buf, sizeof buf, "box %u: negative values in grid.origo", k);
        return fail(h, SPH_ERR_INPUT, buf);
    }
    if (!(g.L[0] > 0.0) || !(g.L[1] > 0.0) || !(g.L[2] > 0.0)) {
        snprintf(buf, sizeof buf, "box %u: grid.L must be positive", k);
        return fail(h, SPH_ERR_INPUT, buf);
    }
    if (g.num[0] == 0 || g.num[1] == 0 || g.num[2] == 0) {
        snprintf(buf, sizeof buf, "box %u: grid.num must be positive", k);
        return fail(h, SPH_ERR_INPUT, buf);
    }
    if (g.periodic == 2 && g.num[0] < 3) {
        snprintf(buf, sizeof buf, "box %u: periodic x needs at least 3 cells along x", k);
        return fail(h, SPH_ERR_INPUT, buf);
    }
    if (g.periodic == 1 && (g.num[0] < 3 || g.num[1] < 3)) {
        snprintf(buf, sizeof buf, "box %u: periodic x/y needs at least 3 cells along x and y", k);
        return fail(h, SPH_ERR_INPUT, buf);
    }
    if (!(b.params.k_n > 0.0)) return fail(h, SPH_ERR_INPUT, "k_n must be positive");
    if (b.params.E < 0.0) return fail(h, SPH_ERR_INPUT, "E must not be negative");
    if (!(b.params.rho > 0.0)) return fail(h, SPH_ERR_INPUT, "rho must be positive");
    if (b.params.contactmodel < 1 || b.params.contactmodel > 3)
        return fail(h, SPH_ERR_INPUT, "contact model must be 1, 2 or 3");
    if (b.walls.nw > SPH_MAXWALLS) return fail(h, SPH_ERR_INPUT, "nw exceeds MAXWALLS (6)");
    if (!(b.dt > 0.0)) return fail(h, SPH_ERR_INPUT, "time.dt must be positive");
    return SPH_OK;
}

static void init_dev_box(DevBox &d, const SphBox &b)
{
    memset(&d, 0, sizeof d);
    d.P = b.params;
    for (int k = 0; k < 3; ++k) {
        d.origo[k] = b.grid.origo[k];
        d.L[k] = b.grid.L[k];
        d.num[k] = b.grid.num[k];
    }
    d.periodic = b.grid.periodic;
    d.adaptive = b.grid.adaptive;
    d.np = b.np;
    d.nb0 = b.nb0;
    d.nblocks = (b.np + 255) / 256;
    d.nw = b.walls.nw;
    for (uint32_t w = 0; w < SPH_MAXWALLS; ++w) {
        d.wmode[w] = b.walls.wmode[w];
        for (int k = 0; k < 4; ++k) {
            d.wnx[w][k] = b.walls.nx[w][k];
            d.wmvfd[w][k] = b.walls.mvfd[w][k];
        }
        d.wacc[w] = 0.0;
    }
    d.tau_x = b.walls.tau_x;
    d.tau_eff_x = 0.0;
    d.dt = b.dt;
    d.t_current = b.t_current;
    d.iter = 0;
    // device.cu:994 and 2455-2462: velocity-step state of the first step
    d.velocity_state = 1;
    d.change_velocity_state = 0;
    if (d.t_current >= 10.0 && d.t_current < 15.0) {
        d.change_velocity_state = 1;
        d.velocity_state = 2;
    }
    // device.cu:1050-1052: adaptive grid height of the first step
    d.L2_out = d.L[2];
    if (d.adaptive == 1 && d.nw > 0) d.L[2] = d.wnx[0][3];
}

extern "C" {

int sph_darcy_struct_size(uint64_t *size)
{
    if (!size) return SPH_ERR_INPUT;
    *size = sizeof(SphDarcy);
    return SPH_OK;
}

int sph_struct_sizes(uint64_t *sizes)
{
    if (!sizes) return SPH_ERR_INPUT;
    sizes[0] = sizeof(SphParams);
    sizes[1] = sizeof(SphGrid);
    sizes[2] = sizeof(SphWalls);
    sizes[3] = sizeof(SphBox);
    sizes[4] = sizeof(SphParticles);
    sizes[5] = sizeof(SphBonds);
    return SPH_OK;
}

const char *sph_status_string(int status)
{
    switch (status) {
    case SPH_OK: return "ok";
    case SPH_ERR_INPUT: return "invalid input";
    case SPH_ERR_CUDA: return "CUDA error";
    case SPH_ERR_NC_OVERFLOW: return "a particle had more contacts than the contact list holds (NC = 32)";
    case SPH_ERR_OUT_OF_GRID: return "a particle left the computational grid";
    case SPH_ERR_NAN: return "a particle position is not finite";
    case SPH_ERR_NOMEM: return "out of memory";
    case SPH_ERR_STATE: return "call out of order";
    case SPH_ERR_UNSUPPORTED: return "unsupported";
    case SPH_ERR_TIMEOUT: return "a device-side wait gave up (grid barrier time limit)";
    default: return "unknown status";
    }
}

int sph_last_error(const SphHandle *h, char *buf, size_t n)
{
    const char *m = h ? h->err.c_str() : "no handle";
    if (!buf || n == 0) return 0;
    size_t k = strlen(m);
    if (k >= n) k = n - 1;
    memcpy(buf, m, k);
    buf[k] = 0;
    return (int)k;
}

void sph_destroy(SphHandle *h)
{
    if (!h) return;
    if (h->device >= 0) cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    for (int k = 1; k < 4; ++k) {
        if (h->pexec_ph[k]) cudaGraphExecDestroy(h->pexec_ph[k]);
        if (h->pgraph_ph[k]) cudaGraphDestroy(h->pgraph_ph[k]);
    }
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    for (int r = 0; r < SphHandle::PR; ++r) {
        if (h->pexec[r]) cudaGraphExecDestroy(h->pexec[r]);
        if (h->pgraph[r]) cudaGraphDestroy(h->pgraph[r]);
        if (h->prof_events)
            for (int k = 0; k <= sph::Prof::MAX; ++k) cudaEventDestroy(h->prof[r].ev[k]);
    }
    if (h->adj_snaps) cudaFree(h->adj_snaps);
    if (h->snap_ev) cudaEventDestroy(h->snap_ev);
    if (h->snap_stream) cudaStreamDestroy(h->snap_stream);
    for (void *p : h->allocs) cudaFree(p);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
}

int sph_create(const SphBox *boxes, uint32_t nboxes, int precision, int length_mode, int device,
               SphHandle **out)
{
    if (!out) return SPH_ERR_INPUT;
    *out = nullptr;
    SphHandle *h = new SphHandle();
    int st = SPH_OK;
    auto bail = [&](int code) {
        sph_destroy(h);
        return code;
    };
    if (!boxes || nboxes == 0) return bail(SPH_ERR_INPUT);
    if (precision != SPH_PREC_FP64 && precision != SPH_PREC_MIXED) return bail(SPH_ERR_INPUT);
    if (length_mode != SPH_LEN_REFERENCE && length_mode != SPH_LEN_FP64) return bail(SPH_ERR_INPUT);
    h->precision = precision;
    h->lenmode = length_mode;
    h->nbox = nboxes;
    h->boxes.assign(boxes, boxes + nboxes);
    h->dbox.resize(nboxes);
    h->t_host.resize(nboxes);
    bool any_walls = false, unfused = false;
    uint64_t pb = 0, cb = 0, bb = 0, qb = 0;
    for (uint32_t k = 0; k < nboxes; ++k) {
        if ((st = check_box(h, boxes[k], k)) != SPH_OK) {
            fprintf(stderr, "sphere_b200: %s\n", h->err.c_str());
            return bail(st);
        }
        DevBox &d = h->dbox[k];
        init_dev_box(d, boxes[k]);
        d.p_base = (uint32_t)pb;
        d.cell_base = (uint32_t)cb;
        d.b_base = (uint32_t)bb;
        d.part_base = (uint32_t)qb;
        pb += boxes[k].np;
        cb += (uint64_t)boxes[k].grid.num[0] * boxes[k].grid.num[1] * boxes[k].grid.num[2];
        bb += boxes[k].nb0;
        qb += d.nblocks;
        if (boxes[k].walls.nw > 0) any_walls = true;
        if (boxes[k].walls.nw > 0 && boxes[k].walls.wmode[0] == 3) unfused = true;
        h->t_host[k] = boxes[k].t_current;
    }
    h->ntot = pb;
    h->ncells = cb;
    h->nbonds = bb;
    h->npartials = qb;
    if (pb >= sph::ID_MASK) return bail(SPH_ERR_UNSUPPORTED);
    if (cb >= 0xffffffffull || cb > 4096ull * 4096ull) return bail(SPH_ERR_UNSUPPORTED);
    h->cfg.lenmode = length_mode;
    h->cfg.unfused = unfused;
    h->cfg.any_walls = any_walls;
    h->cfg.all_cm23 = true;
    for (uint32_t k = 0; k < nboxes; ++k)
        if (boxes[k].params.contactmodel != 2 && boxes[k].params.contactmodel != 3)
            h->cfg.all_cm23 = false;

    if (device >= 0) {
        if (cudaSetDevice(device) != cudaSuccess) return bail(SPH_ERR_CUDA);
        h->device = device;
    } else {
        cudaGetDevice(&h->device);
    }
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess)
        return bail(SPH_ERR_CUDA);
    h->stream = h->own;
    {
        const char *e = getenv("SPHERE_B200_EAGER");
        h->eager = e && e[0] == '1';
    }

    StepArgs &A = h->A;
    A.nboxes = nboxes;
    A.ntot = (uint32_t)h->ntot;
    A.ncells = h->ncells;
    A.nbonds = (uint32_t)h->nbonds;
    A.npartials = (uint32_t)h->npartials;
    const uint64_t n = h->ntot, nb = h->nbonds;
    uint32_t *box_of = nullptr, *part_owner = nullptr, *bond_box = nullptr, *bcsr_off = nullptr,
             *bcsr_ent = nullptr;
    const uint32_t scan_blocks = (uint32_t)((h->ncells + 4095) / 4096);
    if ((st = dalloc(h, &A.boxes, nboxes)) || (st = dalloc(h, &A.x, n)) ||
        (st = dalloc(h, &A.vel, n)) || (st = dalloc(h, &A.angvel, n)) ||
        (st = dalloc(h, &A.angpos, n)) || (st = dalloc(h, &A.xyzsum, n)) ||
        (st = dalloc(h, &A.acc, n)) || (st = dalloc(h, &A.angacc, n)) ||
        (st = dalloc(h, &A.force, n)) || (st = dalloc(h, &A.torque, n)) ||
        (st = dalloc(h, &A.es_dot, n)) || (st = dalloc(h, &A.es, n)) ||
        (st = dalloc(h, &A.ev_dot, n)) || (st = dalloc(h, &A.ev, n)) ||
        (st = dalloc(h, &A.p, n)) || (st = dalloc(h, &box_of, n)) ||
        (st = dalloc(h, &A.cell_id, n)) || (st = dalloc(h, &A.local_off, n)) ||
        (st = dalloc(h, &A.unsorted, n)) ||
        (st = dalloc(h, &A.cell_count, h->ncells)) || (st = dalloc(h, &A.cell_off, h->ncells + 1)) ||
        (st = dalloc(h, &A.scan_tmp, scan_blocks + 1)) || (st = dalloc(h, &A.perm, n)) ||
        (st = dalloc(h, &A.rank, n)) || (st = dalloc(h, &A.xs, n)) || (st = dalloc(h, &A.vs, n)) ||
        (st = dalloc(h, &A.ws, n)) || (st = dalloc(h, &A.xf, n)) ||
        (st = dalloc(h, &A.slots, n * sph::NC)) ||
        (st = dalloc(h, &A.hist, n * sph::NC)) || (st = dalloc(h, &A.wf_pp, n)) ||
        (st = dalloc(h, &A.wall_partial, h->npartials)) || (st = dalloc(h, &A.tau_pp, n)) ||
        (st = dalloc(h, &A.tau_partial, h->npartials)) ||
        (st = dalloc(h, &part_owner, h->npartials)) || (st = dalloc(h, &A.bonds, nb)) ||
        (st = dalloc(h, &A.bdelta, nb)) || (st = dalloc(h, &A.bomega, nb)) ||
        (st = dalloc(h, &A.bf, nb)) || (st = dalloc(h, &A.bt, nb)) ||
        (st = dalloc(h, &A.bbroken, nb)) || (st = dalloc(h, &bond_box, nb)) ||
        (st = dalloc(h, &bcsr_off, n + 1)) || (st = dalloc(h, &bcsr_ent, 2 * nb)) ||
        (st = dalloc(h, &A.err, 1)) || (st = dalloc(h, &h->d_count, 1)) ||
        (st = dalloc(h, &A.vlist, n * sph::VL_MAX)) || (st = dalloc(h, &A.vcount, n)) ||
        (st = dalloc(h, &A.vflag, 2)) || (st = dalloc(h, &A.xref, n)) ||
        (st = dalloc(h, &A.cellc, n))) {
        fprintf(stderr, "sphere_b200: %s\n", h->err.c_str());
        return bail(st);
    }
    A.vcap = sph::VL_MAX;
    h->vlist_mem = A.vlist;
    A.box_of = box_of;
    A.part_owner = part_owner;
    A.bond_box = bond_box;
    A.bcsr_off = bcsr_off;
    A.bcsr_ent = bcsr_ent;

    std::vector<uint32_t> hb(n ? n : 1), hp(h->npartials ? h->npartials : 1), hbb(nb ? nb : 1);
    for (uint32_t k = 0; k < nboxes; ++k) {
        const DevBox &d = h->dbox[k];
        for (uint32_t j = 0; j < d.np; ++j) hb[d.p_base + j] = k;
        for (uint32_t j = 0; j < d.nblocks; ++j) hp[d.part_base + j] = k;
        for (uint32_t j = 0; j < d.nb0; ++j) hbb[d.b_base + j] = k;
    }
    if (cudaMemcpy(box_of, hb.data(), sizeof(uint32_t) * (n ? n : 1), cudaMemcpyHostToDevice) ||
        cudaMemcpy(part_owner, hp.data(), sizeof(uint32_t) * hp.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(bond_box, hbb.data(), sizeof(uint32_t) * hbb.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(A.boxes, h->dbox.data(), sizeof(DevBox) * nboxes, cudaMemcpyHostToDevice) ||
        cudaMemset(A.err, 0, sizeof(uint32_t)))
        return bail(SPH_ERR_CUDA);
    *out = h;
    return SPH_OK;
}

// The checks of one particle range [j0, j1) of a box: the first failing
// particle (bad, with kind 1 radius, 2 NaN, 3 outside the grid) stops the
// range; otherwise the range's largest z and largest/smallest radius.
struct CheckRange {
    uint32_t bad = UINT32_MAX;
    int kind = 0;
    double zmax = 0.0, rmax = 0.0, rmin = HUGE_VAL;
};

static void check_range(const SphParticles *p, const SphBox &b, uint64_t base, uint32_t j0,
                        uint32_t j1, CheckRange &r)
{
    for (uint32_t j = j0; j < j1; ++j) {
        const double *x = p->x + 4 * (size_t)(base + j);
        const double *v = p->vel + 4 * (size_t)(base + j);
        r.rmax = fmax(r.rmax, x[3]);
        r.rmin = fmin(r.rmin, x[3]);
        int kind = 0;
        if (!(x[3] > 0.0)) kind = 1;
        else {
            for (int c = 0; c < 4; ++c)
                if (x[c] != x[c] || v[c] != v[c]) kind = 2;
            if (!kind && (x[0] < b.grid.origo[0] || x[1] < b.grid.origo[1] ||
                          x[2] < b.grid.origo[2] || x[0] > b.grid.L[0] || x[1] > b.grid.L[1] ||
                          x[2] > b.grid.L[2]))
                kind = 3;
        }
        if (kind) {
            r.bad = j;
            r.kind = kind;
            return;
        }
        if (x[2] > r.zmax) r.zmax = x[2];
    }
}

// One pass over the particles (split over host threads for large boxes),
// which also gives each box's largest and smallest radius (0 for an empty
// box).  The error reported is that of the first failing particle in index
// order, as a sequential pass finds it.
static int check_particles(SphHandle *h, const SphParticles *p, std::vector<double> &rmax_box,
                           std::vector<double> &rmin_box)
{
    char buf[256];
    rmax_box.assign(h->nbox, 0.0);
    rmin_box.assign(h->nbox, 0.0);
    const unsigned hw = std::thread::hardware_concurrency();
    for (uint32_t k = 0; k < h->nbox; ++k) {
        const DevBox &d = h->dbox[k];
        const SphBox &b = h->boxes[k];
        const uint32_t nt = d.np >= (1u << 17) ? std::max(1u, std::min(8u, hw)) : 1u;
        std::vector<CheckRange> res(nt);
        const uint32_t per = (d.np + nt - 1) / nt;
        std::vector<std::thread> pool;
        for (uint32_t t = 1; t < nt; ++t) {
            const uint32_t j0 = std::min(d.np, t * per), j1 = std::min(d.np, (t + 1) * per);
            try {
                pool.emplace_back(check_range, p, std::cref(b), (uint64_t)d.p_base, j0, j1,
                                  std::ref(res[t]));
            } catch (...) {
                check_range(p, b, d.p_base, j0, j1, res[t]);   // no thread to be had
            }
        }
        check_range(p, b, d.p_base, 0, std::min(d.np, per), res[0]);
        for (auto &th : pool) th.join();
        double zmax = 0.0, rmax = 0.0, rmin = HUGE_VAL;
        for (const CheckRange &r : res) {
            if (r.kind == 1) {
                snprintf(buf, sizeof buf, "box %u particle %u has a radius of %g m", k, r.bad,
                         p->x[4 * (size_t)(d.p_base + r.bad) + 3]);
                return fail(h, SPH_ERR_INPUT, buf);
            }
            if (r.kind == 2) {
                snprintf(buf, sizeof buf, "box %u particle %u has NaN values", k, r.bad);
                return fail(h, SPH_ERR_INPUT, buf);
            }
            if (r.kind == 3) {
                snprintf(buf, sizeof buf, "box %u particle %u is outside of the computational grid",
                         k, r.bad);
                return fail(h, SPH_ERR_INPUT, buf);
            }
            zmax = fmax(zmax, r.zmax);
            rmax = fmax(rmax, r.rmax);
            rmin = fmin(rmin, r.rmin);
        }
        rmax_box[k] = rmax;
        rmin_box[k] = d.np ? rmin : 0.0;
        if (b.walls.nw > 0 && b.walls.nx[0][3] < zmax) {
            snprintf(buf, sizeof buf,
                     "box %u: one or more particles have centres above the upper, dynamic wall", k);
            return fail(h, SPH_ERR_INPUT, buf);
        }
    }
    return SPH_OK;
}

// [np][3] host layout <-> double4 device arrays: one copy of the host
// buffer into (or out of) a device staging array, and the repacking on the
// GPU (a pinned host buffer then moves at DMA speed).
__global__ void k_unpack3(double4 *dst, const double *src, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0);
}

__global__ void k_pack3(double *dst, const double4 *src, uint64_t n)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double4 v = src[i];
        dst[3 * i] = v.x;
        dst[3 * i + 1] = v.y;
        dst[3 * i + 2] = v.z;
    }
}

// The image code of every occupied slot (sph_set_contacts): the nearest
// periodic image of the partner at the current positions.
__global__ void k_image_codes(StepArgs A, uint64_t ns)
{
    const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ns) return;
    const uint32_t w = A.slots[q];
    if (w == sph::EMPTY) return;
    const uint32_t i = (uint32_t)(q / sph::NC), b = w & sph::ID_MASK;
    const DevBox &B = A.boxes[A.nboxes == 1 ? 0u : A.box_of[i]];
    const double dx = A.x[i].x - A.x[b].x, dy = A.x[i].y - A.x[b].y;
    int sx = 0, sy = 0;
    if (B.periodic == 1 || B.periodic == 2) {
        if (dx > 0.5 * B.L[0]) sx = -1;
        else if (dx < -0.5 * B.L[0]) sx = 1;
    }
    if (B.periodic == 1) {
        if (dy > 0.5 * B.L[1]) sy = -1;
        else if (dy < -0.5 * B.L[1]) sy = 1;
    }
    A.slots[q] = b | (sph::shift_code(sx, sy) << sph::CODE_SHIFT);
}

// Staging for the [np][3] host layouts: one slot of 3 np doubles per
// 3-vector field (five fields), so that every field's copy and repacking
// can be queued before a single synchronisation.
constexpr int STAGE_SLOTS = 5;

static int ensure_stage(SphHandle *h)
{
    if (h->stage) return SPH_OK;
    return dalloc(h, &h->stage, (uint64_t)STAGE_SLOTS * 3 * h->ntot);
}

// Queue on stream s: the host [n][3] field src into slot `slot` of the
// staging array, then repacked into dst (zeros when src is NULL).
static int put3(SphHandle *h, double4 *dst, const double *src, uint64_t n, int slot,
                cudaStream_t s)
{
    if (!src || n == 0) {
        CUDA_TRY(h, cudaMemsetAsync(dst, 0, sizeof(double4) * (n ? n : 1), s));
        return SPH_OK;
    }
    int st;
    if ((st = ensure_stage(h)) != SPH_OK) return st;
    double *stage = h->stage + (size_t)slot * 3 * n;
    CUDA_TRY(h, cudaMemcpyAsync(stage, src, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    k_unpack3<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, stage, n);
    CUDA_TRY(h, cudaGetLastError());
    return SPH_OK;
}

// Queue on stream s: src repacked into staging slot `slot`, then copied to
// the host [n][3] array dst (nothing when dst is NULL).
static int get3(SphHandle *h, double *dst, const double4 *src, uint64_t n, int slot,
                cudaStream_t s)
{
    if (!dst || n == 0) return SPH_OK;
    int st;
    if ((st = ensure_stage(h)) != SPH_OK) return st;
    double *stage = h->stage + (size_t)slot * 3 * n;
    k_pack3<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(stage, src, n);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(dst, stage, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s));
    return SPH_OK;
}

static int put1(SphHandle *h, double *dst, const double *src, uint64_t n, cudaStream_t s)
{
    if (src) CUDA_TRY(h, cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    else CUDA_TRY(h, cudaMemsetAsync(dst, 0, sizeof(double) * (n ? n : 1), s));
    return SPH_OK;
}

int sph_upload(SphHandle *h, const SphParticles *p, const SphBonds *b)
{
    if (!h || !p) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    const uint64_t n = h->ntot, nb = h->nbonds;
    if (n > 0 && (!p->x || !p->vel)) return fail(h, SPH_ERR_INPUT, "x and vel are required");
    if (nb > 0 && (!b || !b->pairs)) return fail(h, SPH_ERR_INPUT, "bond pairs are required");
    int st;
    StepArgs &A = h->A;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    // The copies are queued first and run while the host checks the same
    // input (src/sphere.cpp:145-345 checkValues); a check that fails leaves
    // the handle without a state (sph_step refuses until an upload succeeds).
    h->uploaded = false;
    invalidate_pair(h);
    const cudaStream_t cs = h->stream;
    if (n > 0) {
        CUDA_TRY(h, cudaMemcpyAsync(A.x, p->x, sizeof(double4) * n, cudaMemcpyHostToDevice, cs));
        CUDA_TRY(h, cudaMemcpyAsync(A.vel, p->vel, sizeof(double4) * n, cudaMemcpyHostToDevice, cs));
    }
    if ((st = put3(h, A.xyzsum, p->xyzsum, n, 0, cs)) || (st = put3(h, A.force, p->force, n, 1, cs)) ||
        (st = put3(h, A.angpos, p->angpos, n, 2, cs)) || (st = put3(h, A.angvel, p->angvel, n, 3, cs)) ||
        (st = put3(h, A.torque, p->torque, n, 4, cs)) || (st = put1(h, A.es_dot, p->es_dot, n, cs)) ||
        (st = put1(h, A.es, p->es, n, cs)) || (st = put1(h, A.ev_dot, p->ev_dot, n, cs)) ||
        (st = put1(h, A.ev, p->ev, n, cs)) || (st = put1(h, A.p, p->p, n, cs))) {
        cudaStreamSynchronize(cs);
        return st;
    }
    CUDA_TRY(h, cudaMemsetAsync(A.acc, 0, sizeof(double4) * (n ? n : 1), cs));
    CUDA_TRY(h, cudaMemsetAsync(A.angacc, 0, sizeof(double4) * (n ? n : 1), cs));
    CUDA_TRY(h, cudaMemsetAsync(A.wf_pp, 0, sizeof(double) * (n ? n : 1), cs));
    CUDA_TRY(h, cudaMemsetAsync(A.tau_pp, 0, sizeof(double) * (n ? n : 1), cs));
    // src/device.cu:458-464: empty contact lists; histories start at zero
    if (n) {
        CUDA_TRY(h, cudaMemsetAsync(A.slots, 0xff, sizeof(uint32_t) * n * sph::NC, cs));
        CUDA_TRY(h, cudaMemsetAsync(A.hist, 0, sizeof(double4) * n * sph::NC, cs));
    }
    std::vector<double> rmax_in, rmin_in;
    if ((st = check_particles(h, p, rmax_in, rmin_in)) != SPH_OK) {
        cudaStreamSynchronize(cs);
        return st;
    }

    // bonds (local indexes) and the per-particle list of bond endpoints in
    // ascending bond order
    std::vector<uint32_t> cnt;
    if (nb > 0) {
        cnt.assign(n + 1, 0);
        std::vector<uint2> pairs(nb);
        std::vector<double4> dl(nb), om(nb);
        for (uint32_t k = 0; k < h->nbox; ++k) {
            const DevBox &d = h->dbox[k];
            for (uint32_t j = 0; j < d.nb0; ++j) {
                const uint64_t q = d.b_base + j;
                pairs[q] = make_uint2(b->pairs[2 * q], b->pairs[2 * q + 1]);
                dl[q] = make_double4(b->delta_t ? b->delta_t[3 * q] : 0.0,
                                     b->delta_t ? b->delta_t[3 * q + 1] : 0.0,
                                     b->delta_t ? b->delta_t[3 * q + 2] : 0.0,
                                     b->delta_n ? b->delta_n[q] : 0.0);
                om[q] = make_double4(b->omega_t ? b->omega_t[3 * q] : 0.0,
                                     b->omega_t ? b->omega_t[3 * q + 1] : 0.0,
                                     b->omega_t ? b->omega_t[3 * q + 2] : 0.0,
                                     b->omega_n ? b->omega_n[q] : 0.0);
                if (pairs[q].x < d.np && pairs[q].y < d.np) {
                    cnt[d.p_base + pairs[q].x + 1]++;
                    cnt[d.p_base + pairs[q].y + 1]++;
                }
            }
        }
        for (uint64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
        std::vector<uint32_t> ent(cnt[n] ? cnt[n] : 1), fill(cnt.begin(), cnt.end() - 1);
        for (uint32_t k = 0; k < h->nbox; ++k) {
            const DevBox &d = h->dbox[k];
            for (uint32_t j = 0; j < d.nb0; ++j) {
                const uint32_t q = d.b_base + j;
                if (pairs[q].x < d.np && pairs[q].y < d.np) {
                    ent[fill[d.p_base + pairs[q].x]++] = (q << 1) | 0u;
                    ent[fill[d.p_base + pairs[q].y]++] = (q << 1) | 1u;
                }
            }
        }
        CUDA_TRY(h, cudaMemcpy(A.bonds, pairs.data(), sizeof(uint2) * nb, cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(A.bdelta, dl.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemcpy(A.bomega, om.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice));
        CUDA_TRY(h, cudaMemset(A.bbroken, 0, nb));
        CUDA_TRY(h, cudaMemset(A.bf, 0, sizeof(double4) * nb));
        CUDA_TRY(h, cudaMemset(A.bt, 0, sizeof(double4) * nb));
        CUDA_TRY(h, cudaMemcpy((void *)A.bcsr_ent, ent.data(), sizeof(uint32_t) * ent.size(),
                               cudaMemcpyHostToDevice));
    }
    if (nb > 0)
        CUDA_TRY(h, cudaMemcpy((void *)A.bcsr_off, cnt.data(), sizeof(uint32_t) * (n + 1),
                               cudaMemcpyHostToDevice));
    else
        CUDA_TRY(h, cudaMemset((void *)A.bcsr_off, 0, sizeof(uint32_t) * (n + 1)));
    // a new run: time state from the boxes, TY3 iteration counter at zero
    for (uint32_t k = 0; k < h->nbox; ++k) {
        init_dev_box(h->dbox[k], h->boxes[k]);
        h->dbox[k].p_base = 0;
    }
    {
        uint64_t pb = 0, cb = 0, bb = 0, qb = 0;
        for (uint32_t k = 0; k < h->nbox; ++k) {
            DevBox &d = h->dbox[k];
            d.p_base = (uint32_t)pb;
            d.cell_base = (uint32_t)cb;
            d.b_base = (uint32_t)bb;
            d.part_base = (uint32_t)qb;
            pb += d.np;
            cb += (uint64_t)d.num[0] * d.num[1] * d.num[2];
            bb += d.nb0;
            qb += d.nblocks;
            h->t_host[k] = h->boxes[k].t_current;
            // FP32 prefilter margin: bounds the rounding of FP32 coordinates
            // (|x| <= 2 max L), their differences and periodic shifts, and
            // of the reference's FP32-rounded lengths, with room to spare.
            const double rmax = rmax_in[k];
            double lmax = 0.0;
            for (int c = 0; c < 3; ++c) lmax = fmax(lmax, fabs(d.L[c]) + fabs(d.origo[c]));
            d.pre_margin = (float)(ldexp(2.0 * lmax + 2.0 * rmax, -19));
            h->rmax_box.resize(h->nbox);
            h->rmax_box[k] = rmax;
            // neighbour lists: skin 0.1 r_min; the list is rebuilt once a
            // sphere has moved half the skin less the rounding allowance;
            // the build searches the cells that can hold a sphere within
            // 2 r_max + skin (up to +-3 cells, else lists are off)
            const double rmin = rmin_in[k];
            const double skin = 0.1 * rmin;
            const double cmin = fmin(d.L[0] / d.num[0], fmin(d.L[1] / d.num[1], d.L[2] / d.num[2]));
            const double half = 0.5 * skin - 4.0 * (double)d.pre_margin;
            const double reach = 2.0 * rmax + skin + 2.0 * (double)d.pre_margin;
            const int R = cmin > 0.0 ? (int)ceil(reach / cmin) : 99;
            d.vskin = (float)skin;
            d.vdisp2 = half > 0.0 ? (float)(half * half) : -1.0f;
            d.vrange = (half > 0.0 && R >= 1 && R <= 3) ? R : 0;
        }
    }
    CUDA_TRY(h, cudaMemcpyAsync(A.boxes, h->dbox.data(), sizeof(DevBox) * h->nbox,
                                cudaMemcpyHostToDevice, cs));
    CUDA_TRY(h, cudaMemsetAsync(A.err, 0, sizeof(uint32_t), cs));
    CUDA_TRY(h, cudaMemsetAsync(A.vflag, 0, 2 * sizeof(uint32_t), cs));
    CUDA_TRY(h, cudaMemsetAsync(A.vflag, 1, 1, cs));   // build the lists in the first step
    // the caller's buffers are read only during the call
    CUDA_TRY(h, cudaStreamSynchronize(cs));
    h->uploaded = true;
    return SPH_OK;
}

// Capture one step (optionally with event-record nodes between kernels)
// into a CUDA graph.
static int capture_step(SphHandle *h, sph::Prof *prof, cudaGraph_t *g, cudaGraphExec_t *ge,
                        uint64_t *nl, int phase = sph::STEP_WHOLE)
{
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    // an error left by an earlier failed call (already returned to its
    // caller) must not be taken for a launch error of this capture
    (void)cudaGetLastError();
    StepConfig cfg = h->cfg;
    cfg.phase = phase;
    cfg.side = h->side;
    cfg.fork = h->ev_fork;
    cfg.join = h->ev_join;
    const bool pair = pair_active(h);
    if ((pair || h->darcy_on) && !h->side) {
        // the list step captures its rebuild body, the Darcy coupling its
        // Jacobi loop's body, on the side stream
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    cfg.side = h->side;
    cfg.fork = h->ev_fork;
    cfg.join = h->ev_join;
    if (pair) {
        int st = ensure_pair(h);
        if (st != SPH_OK) return st;
        cfg.side = h->side;
    }
    CUDA_TRY(h, cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
    int st = pair ? sph::launch_step_pair(h->A, h->P, cfg, h->own, nl, prof)
             : h->precision == SPH_PREC_MIXED
                 ? sph::launch_step_mixed(h->A, cfg, h->own, nl, prof)
                 : sph::launch_step(h->A, cfg, h->own, nl, prof);
    cudaError_t e = cudaStreamEndCapture(h->own, g);
    if (st != SPH_OK) return fail(h, st, "step launch failed during graph capture");
    if (e != cudaSuccess) return fail(h, SPH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    CUDA_TRY(h, cudaGraphInstantiate(ge, *g, 0));
    return SPH_OK;
}

static int build_graph(SphHandle *h)
{
    if (h->gexec) return SPH_OK;
    uint64_t nl = 0;
    int st = capture_step(h, nullptr, &h->graph, &h->gexec, &nl);
    if (st != SPH_OK) return st;
    h->launches_per_step = nl;
    return SPH_OK;
}

// Whether runs of steps may overlap a step's wall stage with the next
// step: not when a box's grid follows its wall (the next step's cell hash
// reads L[2]) nor for the unfused kernels.
static bool overlap_ok(const SphHandle *h)
{
    if (h->cfg.unfused || pair_active(h)) return false;
    for (uint32_t k = 0; k < h->nbox; ++k)
        if (h->boxes[k].grid.adaptive) return false;
    return true;
}

static int build_phase_graphs(SphHandle *h)
{
    if (h->pexec_ph[1]) return SPH_OK;
    if (!h->side) {
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    for (int k = 1; k < 4; ++k) {
        uint64_t nl = 0;
        int st = capture_step(h, nullptr, &h->pgraph_ph[k], &h->pexec_ph[k], &nl, k);
        if (st != SPH_OK) return st;
    }
    return SPH_OK;
}

static int build_prof_graphs(SphHandle *h)
{
    if (h->pexec[0]) return SPH_OK;
    if (!h->prof_events) {
        for (int r = 0; r < SphHandle::PR; ++r)
            for (int k = 0; k <= sph::Prof::MAX; ++k) CUDA_TRY(h, cudaEventCreate(&h->prof[r].ev[k]));
        h->prof_events = true;
    }
    for (int r = 0; r < SphHandle::PR; ++r) {
        uint64_t nl = 0;
        int st = capture_step(h, &h->prof[r], &h->pgraph[r], &h->pexec[r], &nl);
        if (st != SPH_OK) return st;
    }
    return SPH_OK;
}

// Launch one step graph on the active stream (a profiled one when profiling).
static int launch_one(SphHandle *h)
{
    if (h->prof_on) {
        CUDA_TRY(h, cudaGraphLaunch(h->pexec[h->pnext], h->stream));
        h->pnext = (h->pnext + 1) % SphHandle::PR;
        h->pcount++;
    } else {
        CUDA_TRY(h, cudaGraphLaunch(h->gexec, h->stream));
    }
    for (uint32_t k = 0; k < h->nbox; ++k) h->t_host[k] += h->boxes[k].dt;
    return SPH_OK;
}

static int collect_errors(SphHandle *h)
{
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    uint32_t bits = 0;
    CUDA_TRY(h, cudaMemcpy(&bits, h->A.err, sizeof bits, cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemset(h->A.err, 0, sizeof(uint32_t)));
    if (!bits) return SPH_OK;
    static const int order[] = {SPH_ERR_TIMEOUT, SPH_ERR_NAN, SPH_ERR_OUT_OF_GRID, SPH_ERR_INPUT,
                                SPH_ERR_NC_OVERFLOW};
    for (int code : order)
        if (bits & (1u << code)) return fail(h, code, sph_status_string(code));
    return fail(h, SPH_ERR_CUDA, "unknown device error bits");
}

int sph_step(SphHandle *h, uint64_t nsteps)
{
    if (!h) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_step before sph_upload");
    int st = sph_step_async(h, nsteps);
    if (st != SPH_OK) return st;
    return collect_errors(h);
}

// The Darcy top pressure of the next n (<= DARCY_RING) queued steps
// (device.cu:2000-2008: p_top_orig + A sin(2 pi f t + phi) with the host's
// time and the C library's sin) into the device ring, in stream order.
static int fill_darcy_pmod(SphHandle *h, uint64_t n)
{
    const SphDarcy &d = h->D.prm;
    std::vector<double> v(n);
    double t = h->t_host[0];
    for (uint64_t j = 0; j < n; ++j) {
        v[j] = h->darcy_p_top_orig + d.p_mod_A * sin(2.0 * 3.14159265358979323846 * d.p_mod_f * t +
                                                     d.p_mod_phi);
        t += h->boxes[0].dt;
    }
    double *ring = const_cast<double *>(h->D.pmod);
    uint64_t done = 0;
    while (done < n) {
        const uint64_t slot = (h->darcy_qstep + done) % sph::DARCY_RING;
        const uint64_t len = std::min<uint64_t>(n - done, sph::DARCY_RING - slot);
        CUDA_TRY(h, cudaMemcpyAsync(ring + slot, v.data() + done, sizeof(double) * len,
                                    cudaMemcpyHostToDevice, h->stream));
        done += len;
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->darcy_qstep += n;
    return SPH_OK;
}

static int queue_steps_now(SphHandle *h, uint64_t nsteps, uint8_t *states);
static int drop_graphs(SphHandle *h);

// Queue nsteps steps on the handle's stream; with states, the box table
// after step s is copied to states + s * (nbox * sizeof(DevBox)) as soon as
// that step's wall stage has run.  With a modulated Darcy top pressure the
// steps are queued in runs of at most DARCY_RING, each after its pressures.
static int queue_steps(SphHandle *h, uint64_t nsteps, uint8_t *states)
{
    if (!h->darcy_on) return queue_steps_now(h, nsteps, states);
    if (!h->D.pmod) {
        h->darcy_qstep += nsteps;
        return queue_steps_now(h, nsteps, states);
    }
    const size_t bytes = sizeof(DevBox) * h->nbox;
    uint64_t done = 0;
    while (done < nsteps) {
        const uint64_t n = std::min<uint64_t>(nsteps - done, sph::DARCY_RING);
        int st = fill_darcy_pmod(h, n);
        if (st == SPH_OK) st = queue_steps_now(h, n, states ? states + done * bytes : nullptr);
        if (st != SPH_OK) return st;
        done += n;
    }
    return SPH_OK;
}

static int queue_steps_now(SphHandle *h, uint64_t nsteps, uint8_t *states)
{
    int st;
    if (h->eager) {
        // kernel by kernel on the handle's stream (no graphs)
        if ((st = prepare_steps(h)) != SPH_OK) return st;
        const size_t bytes = sizeof(DevBox) * h->nbox;
        StepConfig cfg = h->cfg;
        for (uint64_t s = 0; s < nsteps; ++s) {
            uint64_t nl = 0;
            st = pair_active(h) ? sph::launch_step_pair(h->A, h->P, cfg, h->stream, &nl, nullptr)
                 : h->precision == SPH_PREC_MIXED
                     ? sph::launch_step_mixed(h->A, cfg, h->stream, &nl, nullptr)
                     : sph::launch_step(h->A, cfg, h->stream, &nl, nullptr);
            if (st != SPH_OK) return fail(h, st, "step launch failed");
            h->launches += nl;
            for (uint32_t k = 0; k < h->nbox; ++k) h->t_host[k] += h->boxes[k].dt;
            if (states)
                CUDA_TRY(h, cudaMemcpyAsync(states + s * bytes, h->A.boxes, bytes,
                                            cudaMemcpyDeviceToHost, h->stream));
        }
        return SPH_OK;
    }
    if ((st = build_graph(h)) != SPH_OK) return st;
    if ((st = prepare_steps(h)) != SPH_OK) return st;
    const size_t bytes = sizeof(DevBox) * h->nbox;
    if (nsteps >= 2 && !h->prof_on && overlap_ok(h)) {
        // the head of step 1, steps 2..n each beside the wall stage of the
        // step before, then the wall stage of step n: every step's work, in
        // an order that respects each read of the wall stage's results.
        // Graph s (s >= 1) ends with the wall stage of step s, and the
        // heads only read the box table, so a copy after graph s holds the
        // state after step s.
        if ((st = build_phase_graphs(h)) != SPH_OK) return st;
        for (uint64_t s = 0; s <= nsteps; ++s) {
            const int ph = s == 0 ? sph::STEP_HEAD : (s < nsteps ? sph::STEP_OVERLAP : sph::STEP_TAIL);
            CUDA_TRY(h, cudaGraphLaunch(h->pexec_ph[ph], h->stream));
            if (states && s > 0)
                CUDA_TRY(h, cudaMemcpyAsync(states + (s - 1) * bytes, h->A.boxes, bytes,
                                            cudaMemcpyDeviceToHost, h->stream));
        }
        for (uint64_t s = 0; s < nsteps; ++s)
            for (uint32_t k = 0; k < h->nbox; ++k) h->t_host[k] += h->boxes[k].dt;
    } else {
        for (uint64_t s = 0; s < nsteps; ++s) {
            if ((st = launch_one(h)) != SPH_OK) return st;
            if (states)
                CUDA_TRY(h, cudaMemcpyAsync(states + s * bytes, h->A.boxes, bytes,
                                            cudaMemcpyDeviceToHost, h->stream));
        }
    }
    h->launches += nsteps * h->launches_per_step;
    return SPH_OK;
}

int sph_step_async(SphHandle *h, uint64_t nsteps)
{
    if (!h) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_step_async before sph_upload");
    cudaSetDevice(h->device);
    return queue_steps(h, nsteps, nullptr);
}

int sph_step_async_states(SphHandle *h, uint64_t nsteps, void *states, uint64_t states_bytes)
{
    if (!h || !states) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_step_async_states before sph_upload");
    if (nsteps && states_bytes / nsteps < sizeof(DevBox) * (uint64_t)h->nbox)
        return fail(h, SPH_ERR_INPUT, "states smaller than nsteps x sph_box_state_bytes");
    cudaSetDevice(h->device);
    return queue_steps(h, nsteps, static_cast<uint8_t *>(states));
}

int sph_profile(SphHandle *h, int enable)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    if (enable) {
        int st;
        if ((st = build_graph(h)) != SPH_OK || (st = build_prof_graphs(h)) != SPH_OK) return st;
        h->pnext = 0;
        h->pcount = 0;
    }
    h->prof_on = enable != 0;
    return SPH_OK;
}

int sph_profile_read(SphHandle *h, char *names, size_t names_len, double *ms, int max_kernels,
                     int *nkernels)
{
    if (!h || !ms || !nkernels) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const int nr = (int)(h->pcount < (uint64_t)SphHandle::PR ? h->pcount : SphHandle::PR);
    if (nr == 0) return fail(h, SPH_ERR_STATE, "no profiled steps ran");
    const int n = h->prof[0].n;
    std::string all;
    for (int k = 0; k < n && k < max_kernels; ++k) {
        double acc = 0.0;
        for (int r = 0; r < nr; ++r) {
            float t = 0.f;
            CUDA_TRY(h, cudaEventElapsedTime(&t, h->prof[r].ev[k], h->prof[r].ev[k + 1]));
            acc += t;
        }
        ms[k] = acc / nr;
        if (k) all += ",";
        all += h->prof[0].name[k];
    }
    *nkernels = n < max_kernels ? n : max_kernels;
    if (names && names_len) {
        size_t m = all.size() < names_len - 1 ? all.size() : names_len - 1;
        memcpy(names, all.data(), m);
        names[m] = 0;
    }
    return SPH_OK;
}

int sph_sync(SphHandle *h)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    return collect_errors(h);
}

int sph_set_stream(SphHandle *h, void *stream)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own;
    return SPH_OK;
}

int sph_advance(SphHandle *h, double time_total, double file_dt, double *time_current,
                double *filetimeclock, uint64_t max_steps, uint64_t *steps_done)
{
    if (!h || !time_current || !filetimeclock) return SPH_ERR_INPUT;
    if (h->nbox != 1) return fail(h, SPH_ERR_UNSUPPORTED, "sph_advance drives a single box");
    if (*time_current != h->t_host[0])
        return fail(h, SPH_ERR_STATE, "time_current differs from the handle's time");
    const double dt = h->boxes[0].dt;
    double cur = *time_current, ftc = *filetimeclock;
    uint64_t k = 0;
    // device.cu:1031 loop condition, :2536-2537 increments, :2569 output test
    while (cur <= time_total && k < max_steps) {
        cur += dt;
        ftc += dt;
        ++k;
        if (ftc >= file_dt) break;
    }
    int st = sph_step(h, k);
    *time_current = cur;
    *filetimeclock = ftc;
    if (steps_done) *steps_done = k;
    return st;
}

// ------------------------------------------------------------------ Darcy

int sph_darcy_set(SphHandle *h, const SphDarcy *d, const double *p, const double *v,
                  const double *phi, const double *dphi, const int32_t *p_constant,
                  const double *f_p)
{
    if (!h || !d || !p || !v || !phi || !dphi) return SPH_ERR_INPUT;
    if (h->nbox != 1 || h->precision != SPH_PREC_FP64)
        return fail(h, SPH_ERR_UNSUPPORTED, "the Darcy coupling runs one box in the FP64 form");
    const SphBox &b0 = h->boxes[0];
    if (b0.grid.adaptive)
        return fail(h, SPH_ERR_UNSUPPORTED, "the Darcy coupling on an adaptive grid");
    if (d->ndem == 0) return fail(h, SPH_ERR_INPUT, "ndem must be at least 1");
    for (int k = 0; k < 3; ++k)
        if (b0.grid.num[k] < 1) return fail(h, SPH_ERR_INPUT, "empty fluid grid");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const int nx = (int)b0.grid.num[0], ny = (int)b0.grid.num[1], nz = (int)b0.grid.num[2];
    const uint64_t ncell = (uint64_t)(nx + 2) * (ny + 2) * (nz + 2);
    if (ncell >= 0xffffffffull) return fail(h, SPH_ERR_UNSUPPORTED, "fluid grid too large");
    sph::DarcyArgs &D = h->D;
    if (!D.st) {
        int st;
        double **f1[] = {&D.p, &D.p_old, &D.p_new, &D.dp_expl, &D.phi, &D.dphi, &D.norm, &D.k,
                         &D.div_v_p};
        for (double **f : f1)
            if ((st = dalloc(h, f, ncell)) != SPH_OK) return st;
        double **f3[] = {&D.v, &D.vp_avg, &D.grad_k, &D.grad_p};
        for (double **f : f3)
            if ((st = dalloc(h, f, 3 * ncell)) != SPH_OK) return st;
        if ((st = dalloc(h, &D.p_constant, ncell)) != SPH_OK ||
            (st = dalloc(h, &D.f_p, h->ntot)) != SPH_OK || (st = dalloc(h, &D.st, 1)) != SPH_OK ||
            (st = dalloc(h, &D.log_step, SPH_DARCY_LOG)) != SPH_OK ||
            (st = dalloc(h, &D.log_iters, SPH_DARCY_LOG)) != SPH_OK ||
            (st = dalloc(h, &D.log_ok, SPH_DARCY_LOG)) != SPH_OK ||
            (st = dalloc(h, &D.bar, 1)) != SPH_OK ||
            (st = dalloc(h, &D.part_max, sph::DARCY_PARTS)) != SPH_OK ||
            (st = dalloc(h, &D.part_nan, sph::DARCY_PARTS)) != SPH_OK ||
            (st = dalloc(h, &D.coef, (uint64_t)sph::DARCY_COEF * nx * ny * nz)) != SPH_OK)
            return st;
        CUDA_TRY(h, cudaMemset(D.bar, 0, sizeof(unsigned long long)));
    }
    const bool modulated = (d->p_mod_A > 1.0e-5 || d->p_mod_A < -1.0e-5) && d->p_mod_f > 1.0e-7;
    if (modulated && !D.pmod) {
        double *ring = nullptr;
        int st = dalloc(h, &ring, sph::DARCY_RING);
        if (st != SPH_OK) return st;
        D.pmod = ring;
    }
    D.prm = *d;
    D.periodic = b0.grid.periodic;
    D.nx = nx;
    D.ny = ny;
    D.nz = nz;
    D.dx = b0.grid.L[0] / b0.grid.num[0];
    D.dy = b0.grid.L[1] / b0.grid.num[1];
    D.dz = b0.grid.L[2] / b0.grid.num[2];
    D.ncell = (uint32_t)ncell;
    if (!modulated) D.pmod = nullptr;
    // the fields with zero ghost layers, x fastest inside
    auto pad = [&](const double *src, int m) {
        std::vector<double> out((size_t)m * ncell, 0.0);
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const size_t c = (size_t)(x + 1) + (size_t)(nx + 2) * (y + 1) +
                                     (size_t)(nx + 2) * (ny + 2) * (z + 1);
                    const size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
                    for (int k = 0; k < m; ++k) out[(size_t)m * c + k] = src[(size_t)m * i + k];
                }
        return out;
    };
    const std::vector<double> hp = pad(p, 1), hv = pad(v, 3), hphi = pad(phi, 1), hd = pad(dphi, 1);
    std::vector<int32_t> hc(ncell, 0);
    if (p_constant)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                    hc[(size_t)(x + 1) + (size_t)(nx + 2) * (y + 1) + (size_t)(nx + 2) * (ny + 2) * (z + 1)] =
                        p_constant[(size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z)];
    std::vector<double4> hf(h->ntot ? h->ntot : 1, make_double4(0.0, 0.0, 0.0, 0.0));
    if (f_p)
        for (uint64_t i = 0; i < h->ntot; ++i) hf[i] = make_double4(f_p[3 * i], f_p[3 * i + 1], f_p[3 * i + 2], 0.0);
    const size_t B1 = sizeof(double) * ncell;
    CUDA_TRY(h, cudaMemcpy(D.p, hp.data(), B1, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(D.v, hv.data(), 3 * B1, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(D.phi, hphi.data(), B1, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(D.dphi, hd.data(), B1, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(D.p_constant, hc.data(), sizeof(int32_t) * ncell, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(D.f_p, hf.data(), sizeof(double4) * (h->ntot ? h->ntot : 1), cudaMemcpyHostToDevice));
    double *zero1[] = {D.p_old, D.p_new, D.dp_expl, D.norm, D.k, D.div_v_p};
    for (double *f : zero1) CUDA_TRY(h, cudaMemset(f, 0, B1));
    double *zero3[] = {D.vp_avg, D.grad_k, D.grad_p};
    for (double *f : zero3) CUDA_TRY(h, cudaMemset(f, 0, 3 * B1));
    // the start of the run (device.cu:1001, 1009-1015, 918): the top
    // pressure at t = time.current, the file clock, the host's copy of the
    // top wall as the device holds it now
    DevBox b;
    CUDA_TRY(h, cudaMemcpy(&b, h->A.boxes, sizeof(DevBox), cudaMemcpyDeviceToHost));
    h->darcy_p_top_orig = hp[(size_t)1 + (size_t)(nx + 2) * 1 + (size_t)(nx + 2) * (ny + 2) * nz] -
                          d->p_mod_A * sin(2.0 * 3.14159265358979323846 * d->p_mod_f * h->t_host[0] +
                                           d->p_mod_phi);
    sph::DarcyState ds{};
    ds.filetimeclock = 0.0;
    ds.wall_w_host = b.nw > 0 ? b.wnx[0][3] : 0.0;
    ds.wall0_iz = 10000000u;
    CUDA_TRY(h, cudaMemcpy(D.st, &ds, sizeof ds, cudaMemcpyHostToDevice));
    h->darcy_qstep = 0;
    h->darcy_log_tail = 0;
    h->darcy_on = true;
    h->cfg.darcy = &h->D;
    h->cfg.unfused = true;
    return drop_graphs(h);
}

int sph_darcy_get(SphHandle *h, double *p, double *v, double *phi, double *dphi, double *k,
                  double *f_p)
{
    if (!h) return SPH_ERR_INPUT;
    if (!h->darcy_on) return fail(h, SPH_ERR_STATE, "sph_darcy_get before sph_darcy_set");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const sph::DarcyArgs &D = h->D;
    const int nx = D.nx, ny = D.ny, nz = D.nz;
    const size_t ncell = D.ncell;
    auto get = [&](double *dst, const double *src, int m) -> int {
        if (!dst) return SPH_OK;
        std::vector<double> buf((size_t)m * ncell);
        CUDA_TRY(h, cudaMemcpy(buf.data(), src, sizeof(double) * m * ncell, cudaMemcpyDeviceToHost));
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const size_t c = (size_t)(x + 1) + (size_t)(nx + 2) * (y + 1) +
                                     (size_t)(nx + 2) * (ny + 2) * (z + 1);
                    const size_t i = (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z);
                    for (int q = 0; q < m; ++q) dst[(size_t)m * i + q] = buf[(size_t)m * c + q];
                }
        return SPH_OK;
    };
    int st;
    if ((st = get(p, D.p, 1)) || (st = get(v, D.v, 3)) || (st = get(phi, D.phi, 1)) ||
        (st = get(dphi, D.dphi, 1)) || (st = get(k, D.k, 1)))
        return st;
    if (f_p && h->ntot) {
        std::vector<double4> hf(h->ntot);
        CUDA_TRY(h, cudaMemcpy(hf.data(), D.f_p, sizeof(double4) * h->ntot, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < h->ntot; ++i) {
            f_p[3 * i] = hf[i].x;
            f_p[3 * i + 1] = hf[i].y;
            f_p[3 * i + 2] = hf[i].z;
        }
    }
    return SPH_OK;
}

int sph_darcy_log(SphHandle *h, uint64_t *step, uint32_t *iterations, uint32_t *converged,
                  uint32_t cap, uint32_t *n)
{
    if (!h || !n || (cap && (!step || !iterations || !converged))) return SPH_ERR_INPUT;
    *n = 0;
    if (!h->darcy_on) return fail(h, SPH_ERR_STATE, "sph_darcy_log before sph_darcy_set");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const sph::DarcyArgs &D = h->D;
    sph::DarcyState ds;
    CUDA_TRY(h, cudaMemcpy(&ds, D.st, sizeof ds, cudaMemcpyDeviceToHost));
    const uint64_t head = ds.log_head;
    uint64_t first = h->darcy_log_tail;
    if (head - first > SPH_DARCY_LOG) first = head - SPH_DARCY_LOG;
    const uint64_t count = std::min<uint64_t>(head - first, cap);
    if (count) {
        std::vector<uint64_t> a(SPH_DARCY_LOG);
        std::vector<uint32_t> b(SPH_DARCY_LOG), c(SPH_DARCY_LOG);
        CUDA_TRY(h, cudaMemcpy(a.data(), D.log_step, sizeof(uint64_t) * SPH_DARCY_LOG, cudaMemcpyDeviceToHost));
        CUDA_TRY(h, cudaMemcpy(b.data(), D.log_iters, sizeof(uint32_t) * SPH_DARCY_LOG, cudaMemcpyDeviceToHost));
        CUDA_TRY(h, cudaMemcpy(c.data(), D.log_ok, sizeof(uint32_t) * SPH_DARCY_LOG, cudaMemcpyDeviceToHost));
        for (uint64_t j = 0; j < count; ++j) {
            const size_t slot = (size_t)((first + j) % SPH_DARCY_LOG);
            step[j] = a[slot];
            iterations[j] = b[slot];
            converged[j] = c[slot];
        }
    }
    h->darcy_log_tail = first + count;
    *n = (uint32_t)count;
    return SPH_OK;
}

}  // extern "C"

// Copy the particle and bond state held in S (the live arrays or the
// snapshot copies) to the host layouts; cs: stream for the copies (null:
// synchronous copies).
static int download_from(SphHandle *h, const StepArgs &S, cudaStream_t cs, SphParticles *p,
                         SphBonds *b)
{
    const uint64_t n = h->ntot, nb = h->nbonds;
    const cudaStream_t s = cs ? cs : h->stream;
    auto d2h = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    };
    int st;
    if (p) {
        // every particle array queued on s (the 3-vector fields repacked in
        // their own staging slots), one synchronisation
        if (p->x && n) CUDA_TRY(h, cudaMemcpyAsync(p->x, S.x, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
        if (p->vel && n)
            CUDA_TRY(h, cudaMemcpyAsync(p->vel, S.vel, sizeof(double4) * n, cudaMemcpyDeviceToHost, s));
        if ((st = get3(h, p->xyzsum, S.xyzsum, n, 0, s)) || (st = get3(h, p->force, S.force, n, 1, s)) ||
            (st = get3(h, p->angpos, S.angpos, n, 2, s)) || (st = get3(h, p->angvel, S.angvel, n, 3, s)) ||
            (st = get3(h, p->torque, S.torque, n, 4, s))) {
            cudaStreamSynchronize(s);
            return st;
        }
        double *dst[5] = {p->es_dot, p->es, p->ev_dot, p->ev, p->p};
        double *src[5] = {S.es_dot, S.es, S.ev_dot, S.ev, S.p};
        for (int k = 0; k < 5; ++k)
            if (dst[k] && n)
                CUDA_TRY(h, cudaMemcpyAsync(dst[k], src[k], sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(h, cudaStreamSynchronize(s));
    }
    if (b && nb) {
        std::vector<uint2> pairs(nb);
        std::vector<double4> dl(nb), om(nb);
        CUDA_TRY(h, d2h(pairs.data(), S.bonds, sizeof(uint2) * nb));
        CUDA_TRY(h, d2h(dl.data(), S.bdelta, sizeof(double4) * nb));
        CUDA_TRY(h, d2h(om.data(), S.bomega, sizeof(double4) * nb));
        for (uint64_t q = 0; q < nb; ++q) {
            if (b->pairs) { b->pairs[2 * q] = pairs[q].x; b->pairs[2 * q + 1] = pairs[q].y; }
            if (b->delta_n) b->delta_n[q] = dl[q].w;
            if (b->delta_t) { b->delta_t[3 * q] = dl[q].x; b->delta_t[3 * q + 1] = dl[q].y; b->delta_t[3 * q + 2] = dl[q].z; }
            if (b->omega_n) b->omega_n[q] = om[q].w;
            if (b->omega_t) { b->omega_t[3 * q] = om[q].x; b->omega_t[3 * q + 1] = om[q].y; b->omega_t[3 * q + 2] = om[q].z; }
        }
    }
    return SPH_OK;
}

// The boxes as created, with the fields the step changes taken from the
// device box table image d.
static void boxes_from(SphHandle *h, const std::vector<DevBox> &d, SphBox *boxes)
{
    for (uint32_t k = 0; k < h->nbox; ++k) {
        SphBox b = h->boxes[k];
        for (int c = 0; c < 2; ++c) b.grid.L[c] = d[k].L[c];
        b.grid.L[2] = d[k].L2_out;
        for (uint32_t w = 0; w < SPH_MAXWALLS; ++w)
            for (int c = 0; c < 4; ++c) {
                b.walls.nx[w][c] = d[k].wnx[w][c];
                b.walls.mvfd[w][c] = d[k].wmvfd[w][c];
            }
        b.t_current = d[k].t_current;
        boxes[k] = b;
    }
}

extern "C" {

int sph_download(SphHandle *h, SphParticles *p, SphBonds *b)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    int st = sync_public(h);
    if (st != SPH_OK) return st;
    return download_from(h, h->A, nullptr, p, b);
}

int sph_get_boxes(SphHandle *h, SphBox *boxes)
{
    if (!h || !boxes) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    std::vector<DevBox> d(h->nbox);
    CUDA_TRY(h, cudaMemcpy(d.data(), h->A.boxes, sizeof(DevBox) * h->nbox, cudaMemcpyDeviceToHost));
    boxes_from(h, d, boxes);
    return SPH_OK;
}

int sph_box_state_bytes(const SphHandle *h, uint64_t *bytes)
{
    if (!h || !bytes) return SPH_ERR_INPUT;
    *bytes = sizeof(DevBox) * (uint64_t)h->nbox;
    return SPH_OK;
}

int sph_get_boxes_async(SphHandle *h, void *staging, uint64_t staging_bytes)
{
    if (!h || !staging) return SPH_ERR_INPUT;
    if (staging_bytes < sizeof(DevBox) * (uint64_t)h->nbox)
        return fail(h, SPH_ERR_INPUT, "staging buffer smaller than sph_box_state_bytes");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaMemcpyAsync(staging, h->A.boxes, sizeof(DevBox) * h->nbox,
                                cudaMemcpyDeviceToHost, h->stream));
    return SPH_OK;
}

int sph_boxes_from_staging(SphHandle *h, const void *staging, uint64_t nstates, SphBox *boxes)
{
    if (!h || (nstates && (!staging || !boxes))) return SPH_ERR_INPUT;
    std::vector<DevBox> d(h->nbox);
    const uint8_t *src = static_cast<const uint8_t *>(staging);
    for (uint64_t s = 0; s < nstates; ++s) {
        memcpy(d.data(), src + s * sizeof(DevBox) * h->nbox, sizeof(DevBox) * h->nbox);
        boxes_from(h, d, boxes + s * h->nbox);
    }
    return SPH_OK;
}

int sph_snapshot(SphHandle *h)
{
    if (!h) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_snapshot before sph_upload");
    cudaSetDevice(h->device);
    const uint64_t n = h->ntot, nb = h->nbonds;
    StepArgs &S = h->snap;
    if (!h->snap_alloc) {
        int st;
        if ((st = dalloc(h, &S.x, n)) || (st = dalloc(h, &S.vel, n)) ||
            (st = dalloc(h, &S.angvel, n)) || (st = dalloc(h, &S.angpos, n)) ||
            (st = dalloc(h, &S.xyzsum, n)) || (st = dalloc(h, &S.force, n)) ||
            (st = dalloc(h, &S.torque, n)) || (st = dalloc(h, &S.es_dot, n)) ||
            (st = dalloc(h, &S.es, n)) || (st = dalloc(h, &S.ev_dot, n)) ||
            (st = dalloc(h, &S.ev, n)) || (st = dalloc(h, &S.p, n)) ||
            (st = dalloc(h, &S.bonds, nb)) || (st = dalloc(h, &S.bdelta, nb)) ||
            (st = dalloc(h, &S.bomega, nb)) || (st = dalloc(h, &S.boxes, h->nbox)) ||
            (st = dalloc(h, &S.err, 1)))
            return st;
        CUDA_TRY(h, cudaEventCreateWithFlags(&h->snap_ev, cudaEventDisableTiming));
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
        h->snap_alloc = true;
    }
    if (h->pair_ahead) {
        // the compact state into the FP64 arrays, on the stream, before the copies
        int st = sph::pair_flush(h->A, h->P, h->stream);
        if (st != SPH_OK) return fail(h, st, "list-step state flush failed");
        h->pair_ahead = false;
    }
    const StepArgs &A = h->A;
    auto d2d = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream);
    };
    const size_t n4 = sizeof(double4) * (n ? n : 1), n1 = sizeof(double) * (n ? n : 1);
    CUDA_TRY(h, d2d(S.x, A.x, n4));
    CUDA_TRY(h, d2d(S.vel, A.vel, n4));
    CUDA_TRY(h, d2d(S.angvel, A.angvel, n4));
    CUDA_TRY(h, d2d(S.angpos, A.angpos, n4));
    CUDA_TRY(h, d2d(S.xyzsum, A.xyzsum, n4));
    CUDA_TRY(h, d2d(S.force, A.force, n4));
    CUDA_TRY(h, d2d(S.torque, A.torque, n4));
    CUDA_TRY(h, d2d(S.es_dot, A.es_dot, n1));
    CUDA_TRY(h, d2d(S.es, A.es, n1));
    CUDA_TRY(h, d2d(S.ev_dot, A.ev_dot, n1));
    CUDA_TRY(h, d2d(S.ev, A.ev, n1));
    CUDA_TRY(h, d2d(S.p, A.p, n1));
    if (nb) {
        CUDA_TRY(h, d2d(S.bonds, A.bonds, sizeof(uint2) * nb));
        CUDA_TRY(h, d2d(S.bdelta, A.bdelta, sizeof(double4) * nb));
        CUDA_TRY(h, d2d(S.bomega, A.bomega, sizeof(double4) * nb));
    }
    CUDA_TRY(h, d2d(S.boxes, A.boxes, sizeof(DevBox) * h->nbox));
    CUDA_TRY(h, d2d(S.err, A.err, sizeof(uint32_t)));
    // errors are reported once: by the snapshot that saw them
    CUDA_TRY(h, cudaMemsetAsync(A.err, 0, sizeof(uint32_t), h->stream));
    CUDA_TRY(h, cudaEventRecord(h->snap_ev, h->stream));
    h->snap_pending = true;
    return SPH_OK;
}

int sph_snapshot_read(SphHandle *h, SphParticles *p, SphBonds *b, SphBox *boxes)
{
    if (!h) return SPH_ERR_INPUT;
    if (!h->snap_pending) return fail(h, SPH_ERR_STATE, "no snapshot to read");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaEventSynchronize(h->snap_ev));
    h->snap_pending = false;
    int st = download_from(h, h->snap, h->snap_stream, p, b);
    if (st != SPH_OK) return st;
    uint32_t bits = 0;
    std::vector<DevBox> d(h->nbox);
    CUDA_TRY(h, cudaMemcpyAsync(d.data(), h->snap.boxes, sizeof(DevBox) * h->nbox,
                                cudaMemcpyDeviceToHost, h->snap_stream));
    CUDA_TRY(h, cudaMemcpyAsync(&bits, h->snap.err, sizeof bits, cudaMemcpyDeviceToHost,
                                h->snap_stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->snap_stream));
    if (boxes) boxes_from(h, d, boxes);
    if (!bits) return SPH_OK;
    static const int order[] = {SPH_ERR_TIMEOUT, SPH_ERR_NAN, SPH_ERR_OUT_OF_GRID, SPH_ERR_INPUT,
                                SPH_ERR_NC_OVERFLOW};
    for (int code : order)
        if (bits & (1u << code)) return fail(h, code, sph_status_string(code));
    return SPH_OK;
}

int sph_get_contacts(SphHandle *h, uint32_t *contacts, double *delta_t, double *distmod)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st = sync_public(h);
        if (st != SPH_OK) return st;
    }
    const uint64_t n = h->ntot, ns = n * sph::NC;
    if (n == 0) return SPH_OK;
    std::vector<uint32_t> w(ns);
    std::vector<double4> x(n);
    CUDA_TRY(h, cudaMemcpy(w.data(), h->A.slots, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(x.data(), h->A.x, sizeof(double4) * n, cudaMemcpyDeviceToHost));
    if (delta_t)
        CUDA_TRY(h, cudaMemcpy(delta_t, h->A.hist, sizeof(double4) * ns, cudaMemcpyDeviceToHost));
    for (uint32_t k = 0; k < h->nbox; ++k) {
        const DevBox &d = h->dbox[k];
        for (uint64_t i = d.p_base; i < (uint64_t)d.p_base + d.np; ++i)
            for (int s = 0; s < sph::NC; ++s) {
                const uint64_t q = i * sph::NC + s;
                const uint32_t v = w[q];
                double dm[4] = {0.0, 0.0, 0.0, 0.0};
                uint32_t partner = d.np;
                if (v != sph::EMPTY) {
                    const uint32_t g = v & sph::ID_MASK;
                    partner = g - d.p_base;
                    int sx = (int)((v >> sph::CODE_SHIFT) & 3u), sy = (int)((v >> (sph::CODE_SHIFT + 2)) & 3u);
                    if (sx == 3) sx = -1;
                    if (sy == 3) sy = -1;
                    dm[0] = sx == 0 ? 0.0 : (sx > 0 ? d.L[0] : -d.L[0]);
                    dm[1] = sy == 0 ? 0.0 : (sy > 0 ? d.L[1] : -d.L[1]);
                    dm[3] = x[g].w;
                }
                if (contacts) contacts[q] = partner;
                if (distmod)
                    for (int c = 0; c < 4; ++c) distmod[4 * q + c] = dm[c];
            }
    }
    return SPH_OK;
}

int sph_set_contacts(SphHandle *h, const uint32_t *contacts, const double *delta_t)
{
    if (!h || !contacts) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_set_contacts before sph_upload");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const uint64_t n = h->ntot, ns = n * sph::NC;
    if (n == 0) return SPH_OK;
    std::vector<uint32_t> w(ns, sph::EMPTY);
    for (uint32_t k = 0; k < h->nbox; ++k) {
        const DevBox &d = h->dbox[k];
        for (uint64_t i = d.p_base; i < (uint64_t)d.p_base + d.np; ++i)
            for (int s = 0; s < sph::NC; ++s) {
                const uint64_t q = i * sph::NC + s;
                const uint32_t b = contacts[q];
                if (b == d.np) continue;
                if (b > d.np || (uint64_t)d.p_base + b == i) {
                    char buf[160];
                    snprintf(buf, sizeof buf, "box %u sphere %llu slot %d: partner %u is not "
                             "another sphere of the box", k, (unsigned long long)(i - d.p_base), s, b);
                    return fail(h, SPH_ERR_INPUT, buf);
                }
                w[q] = d.p_base + b;   // image code set on the device
            }
    }
    std::vector<double4> hist(ns);
    for (uint64_t q = 0; q < ns; ++q)
        hist[q] = delta_t && w[q] != sph::EMPTY
                      ? make_double4(delta_t[4 * q], delta_t[4 * q + 1], delta_t[4 * q + 2], 0.0)
                      : make_double4(0.0, 0.0, 0.0, 0.0);
    CUDA_TRY(h, cudaMemcpy(h->A.slots, w.data(), sizeof(uint32_t) * ns, cudaMemcpyHostToDevice));
    CUDA_TRY(h, cudaMemcpy(h->A.hist, hist.data(), sizeof(double4) * ns, cudaMemcpyHostToDevice));
    k_image_codes<<<(unsigned)((ns + 255) / 256), 256, 0, h->stream>>>(h->A, ns);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    invalidate_pair(h);
    return SPH_OK;
}

int sph_barrier_check(uint32_t blocks, uint32_t expected, uint32_t rounds, double limit_s)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return SPH_ERR_CUDA;
    if (blocks == 0 || (int)blocks > sms || !(limit_s > 0.0) || limit_s > 10.0 || expected == 0)
        return SPH_ERR_INPUT;
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, 3 * sizeof(uint32_t)) != cudaSuccess) return SPH_ERR_NOMEM;
    int st = sph::barrier_check(blocks, expected, rounds, (unsigned long long)(limit_s * 1e9), d,
                                d + 2, nullptr);
    uint32_t err = 0;
    if (st == SPH_OK && cudaMemcpy(&err, d + 2, sizeof err, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = SPH_ERR_CUDA;
    cudaFree(d);
    if (st != SPH_OK) return st;
    return err & (1u << SPH_ERR_TIMEOUT) ? SPH_ERR_TIMEOUT : SPH_OK;
}

uint64_t sph_total_cells(const SphHandle *h) { return h ? h->ncells : 0; }

int sph_get_sort(SphHandle *h, uint32_t *cell_id, uint32_t *perm, uint32_t *cell_start,
                 uint32_t *cell_end)
{
    if (!h) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const uint64_t n = h->ntot, nc = h->ncells;
    if (cell_id && n) CUDA_TRY(h, cudaMemcpy(cell_id, h->A.cell_id, 4 * n, cudaMemcpyDeviceToHost));
    if (perm && n) CUDA_TRY(h, cudaMemcpy(perm, h->A.perm, 4 * n, cudaMemcpyDeviceToHost));
    if (cell_start || cell_end) {
        std::vector<uint32_t> off(nc + 1);
        CUDA_TRY(h, cudaMemcpy(off.data(), h->A.cell_off, 4 * (nc + 1), cudaMemcpyDeviceToHost));
        for (uint64_t c = 0; c < nc; ++c) {
            const bool empty = off[c + 1] == off[c];
            if (cell_start) cell_start[c] = empty ? 0xffffffffu : off[c];
            if (cell_end) cell_end[c] = empty ? 0xffffffffu : off[c + 1];
        }
    }
    return SPH_OK;
}

int sph_count_contacts(SphHandle *h, uint64_t *ncontacts)
{
    if (!h || !ncontacts) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    uint64_t nl = 0;
    int st;
    if (pair_active(h) && h->pair_valid) {
        st = sph::pair_count_live(h->A, h->P, h->stream, h->d_count);
        nl = 1;
    } else {
        st = sync_public(h);
        if (st == SPH_OK) st = sph::count_live_slots(h->A, h->stream, h->d_count, &nl);
    }
    h->launches += nl;
    if (st != SPH_OK) return fail(h, st, "count_live_slots failed");
    unsigned long long c = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&c, h->d_count, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    *ncontacts = c;
    return SPH_OK;
}

int sph_neighbor_stats(SphHandle *h, uint64_t *stats)
{
    if (!h || !stats) return SPH_ERR_INPUT;
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    const uint64_t n = h->ntot;
    std::vector<uint32_t> vc(n ? n : 1);
    uint32_t flag[2] = {0, 0};
    const uint32_t *counts = h->A.vcount;
    if (pair_active(h) && h->pair_valid) {
        // the list step's lists in use
        uint32_t ls = 0;
        CUDA_TRY(h, cudaMemcpy(&ls, h->P.lsel, sizeof ls, cudaMemcpyDeviceToHost));
        counts = h->P.cnt[ls & 1u];
    }
    if (n) CUDA_TRY(h, cudaMemcpy(vc.data(), counts, 4 * n, cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(flag, h->A.vflag, sizeof flag, cudaMemcpyDeviceToHost));
    uint64_t with = 0, over = 0, sum = 0, mx = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (vc[i] > (uint32_t)sph::VL_MAX) {
            ++over;
        } else {
            ++with;
            sum += vc[i];
            mx = vc[i] > mx ? vc[i] : mx;
        }
    }
    stats[0] = with;
    stats[1] = over;
    stats[2] = sum;
    stats[3] = mx;
    stats[4] = flag[1];
    return SPH_OK;
}

uint64_t sph_kernel_launches(const SphHandle *h) { return h ? h->launches : 0; }

// ------------------------------------------------------------- adjoint

namespace {

struct StateRef {
    void *ptr;
    size_t bytes;
};

// Every device array a step mutates; a checkpoint is a copy of all of them.
std::vector<StateRef> mutable_state(SphHandle *h)
{
    const size_t n = h->ntot ? h->ntot : 1;
    const StepArgs &A = h->A;
    return {{A.x, 32 * n},       {A.vel, 32 * n},      {A.angvel, 32 * n},   {A.angpos, 32 * n},
            {A.xyzsum, 32 * n},  {A.acc, 32 * n},      {A.angacc, 32 * n},   {A.force, 32 * n},
            {A.torque, 32 * n},  {A.es_dot, 8 * n},    {A.es, 8 * n},        {A.ev_dot, 8 * n},
            {A.ev, 8 * n},       {A.p, 8 * n},         {A.slots, 4 * n * sph::NC},
            {A.hist, 32 * n * sph::NC},                {A.boxes, sizeof(DevBox) * h->nbox}};
}

size_t state_bytes(SphHandle *h)
{
    size_t b = 0;
    for (const auto &p : mutable_state(h)) b += p.bytes;
    return b;
}

void copy_state(SphHandle *h, char *snaps, uint64_t k, bool save)
{
    const size_t sb = state_bytes(h);
    char *c = snaps + sb * k;
    for (const auto &p : mutable_state(h)) {
        if (save) cudaMemcpyAsync(c, p.ptr, p.bytes, cudaMemcpyDeviceToDevice, h->stream);
        else cudaMemcpyAsync(p.ptr, c, p.bytes, cudaMemcpyDeviceToDevice, h->stream);
        c += p.bytes;
    }
    // restored positions may lie outside the current neighbour lists
    if (!save) cudaMemsetAsync(h->A.vflag, 1, 1, h->stream);
}

void free_adjoint(SphHandle *h)
{
    if (h->adj_snaps) cudaFree(h->adj_snaps);
    h->adj_snaps = nullptr;
    h->adj_nsteps = 0;
}

}  // namespace

int sph_adjoint_forward(SphHandle *h, uint64_t nsteps, uint32_t ckpt, double *forward_ms)
{
    if (!h || nsteps == 0 || ckpt == 0) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_adjoint_forward before sph_upload");
    if (h->darcy_on) return fail(h, SPH_ERR_UNSUPPORTED, "the adjoint of the Darcy coupling");
    const SphBox &b0 = h->boxes[0];
    if (h->nbox != 1 || h->precision != SPH_PREC_FP64 || h->lenmode != SPH_LEN_FP64 ||
        b0.params.contactmodel != 2 || b0.params.E > 0.001 || b0.params.kappa != 0.0 ||
        b0.nb0 != 0 || b0.walls.nw != 0 || b0.grid.adaptive != 0 || b0.params.gamma_wt != 0.0)
        return fail(h, SPH_ERR_UNSUPPORTED,
                    "the adjoint covers one box, FP64 with FP64 lengths, contact model 2, E = 0, "
                    "kappa = 0, no bonds, no dynamic walls, fixed grid, gamma_wt = 0");
    cudaSetDevice(h->device);
    int st;
    if ((st = build_graph(h)) != SPH_OK) return st;
    free_adjoint(h);
    const uint64_t nseg = (nsteps + ckpt - 1) / ckpt;
    const size_t sb = state_bytes(h);
    void *q = nullptr;
    if (cudaMalloc(&q, sb * (nseg + 1)) != cudaSuccess)
        return fail(h, SPH_ERR_NOMEM, "adjoint checkpoints do not fit in device memory");
    h->adj_snaps = (char *)q;
    DevBox box0;
    CUDA_TRY(h, cudaMemcpy(&box0, h->A.boxes, sizeof box0, cudaMemcpyDeviceToHost));
    h->adj_iter0 = box0.iter;
    h->adj_nsteps = nsteps;
    h->adj_ckpt = ckpt;
    cudaEvent_t ev[2];
    for (auto &e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], h->stream);
    for (uint64_t sgm = 0; sgm < nseg; ++sgm) {
        copy_state(h, h->adj_snaps, sgm, true);
        const uint64_t ns = std::min<uint64_t>(ckpt, nsteps - sgm * ckpt);
        for (uint64_t k = 0; k < ns; ++k)
            if ((st = launch_one(h)) != SPH_OK) break;
        if (st != SPH_OK) break;
    }
    copy_state(h, h->adj_snaps, nseg, true);
    cudaEventRecord(ev[1], h->stream);
    h->launches += nsteps * h->launches_per_step;
    st = st == SPH_OK ? collect_errors(h) : st;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    for (auto &e : ev) cudaEventDestroy(e);
    if (forward_ms) *forward_ms = ms;
    if (st != SPH_OK) free_adjoint(h);
    return st;
}

int sph_adjoint_backward(SphHandle *h, const double *dx_final, double *grad_params,
                         double *grad_v0, double *adjoint_ms)
{
    if (!h || !dx_final) return SPH_ERR_INPUT;
    if (!h->adj_snaps) return fail(h, SPH_ERR_STATE, "sph_adjoint_backward without a forward");
    cudaSetDevice(h->device);
    const uint32_t n = (uint32_t)h->ntot;
    const uint64_t nsteps = h->adj_nsteps, ckpt = h->adj_ckpt;
    const uint64_t nseg = (nsteps + ckpt - 1) / ckpt;
    const size_t n4 = sizeof(double4) * (n ? n : 1);
    const size_t step_tape = 3 * n4 + 2 * sizeof(uint32_t) * n * sph::NC + n4 * sph::NC;
    std::vector<void *> mine;
    auto get = [&](size_t bytes) -> void * {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
        mine.push_back(q);
        return q;
    };
    auto release = [&]() {
        for (void *q : mine) cudaFree(q);
        mine.clear();
    };
    char *tape = (char *)get(step_tape * ckpt);
    double4 *lbuf = (double4 *)get(10 * n4);
    double4 *lH = (double4 *)get(n4 * sph::NC);
    double *dscal = (double *)get(sizeof(double) * 3);
    if (!tape || !lbuf || !lH || !dscal) {
        release();
        return fail(h, SPH_ERR_NOMEM, "adjoint buffers do not fit in device memory");
    }
    double4 *lnext[5], *lnext0[5], *lcur0[5];
    for (int k = 0; k < 5; ++k) {
        lnext0[k] = lnext[k] = lbuf + (size_t)k * n;
        lcur0[k] = lbuf + (size_t)(5 + k) * n;
    }
    std::vector<double4> seed(n ? n : 1);
    for (uint32_t i = 0; i < n; ++i)
        seed[i] = make_double4(dx_final[3 * i], dx_final[3 * i + 1], dx_final[3 * i + 2], 0.0);
    cudaEvent_t ev[2];
    for (auto &e : ev) cudaEventCreate(&e);
    int st = SPH_OK;
    cudaError_t e = cudaMemsetAsync(lbuf, 0, 10 * n4, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(lH, 0, n4 * sph::NC, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dscal, 0, sizeof(double) * 3, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(lnext[0], seed.data(), n4, cudaMemcpyHostToDevice, h->stream);
    // Each segment's recompute (the steps from its checkpoint, each step's
    // start state and contact rows copied to the tape) and its reverse (the
    // steps' adjoint kernels, last step first) are captured once as CUDA
    // graphs and launched for every segment of that shape: the tape
    // offsets are the same in every segment, the reverse differs only in
    // the segment's length, in whether it holds the run's first step (whose
    // previous accelerations are zero) and in which of the two adjoint
    // buffers it starts from.
    struct SegGraph {
        uint64_t ns;
        int kind;   // recompute: -1; reverse: first * 2 + parity
        cudaGraph_t g;
        cudaGraphExec_t ge;
    };
    std::vector<SegGraph> graphs;
    auto seg_graph = [&](uint64_t ns, int kind, cudaGraphExec_t *out) -> int {
        for (const SegGraph &q : graphs)
            if (q.ns == ns && q.kind == kind) {
                *out = q.ge;
                return SPH_OK;
            }
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SPH_ERR_CUDA;
        (void)cudaGetLastError();
        if (cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return SPH_ERR_CUDA;
        int rst = SPH_OK;
        if (kind < 0) {
            for (uint64_t k = 0; k < ns && rst == SPH_OK; ++k) {
                char *t = tape + step_tape * k;
                cudaMemcpyAsync(t, h->A.x, n4, cudaMemcpyDeviceToDevice, h->own);
                cudaMemcpyAsync(t + n4, h->A.vel, n4, cudaMemcpyDeviceToDevice, h->own);
                cudaMemcpyAsync(t + 2 * n4, h->A.angvel, n4, cudaMemcpyDeviceToDevice, h->own);
                StepArgs Ar = h->A;
                Ar.tape_rows_pre = (uint32_t *)(t + 3 * n4);
                Ar.tape_rows_post = Ar.tape_rows_pre + (size_t)n * sph::NC;
                Ar.tape_hist = (double4 *)(Ar.tape_rows_post + (size_t)n * sph::NC);
                uint64_t nl = 0;
                rst = sph::launch_step(Ar, h->cfg, h->own, &nl);
            }
        } else {
            const bool first = (kind >> 1) != 0;
            double4 *ln[5], *lc[5];
            for (int q = 0; q < 5; ++q) {
                ln[q] = (kind & 1) ? lcur0[q] : lnext0[q];
                lc[q] = (kind & 1) ? lnext0[q] : lcur0[q];
            }
            for (uint64_t k = ns; k-- > 0 && rst == SPH_OK;) {
                const char *t = tape + step_tape * k;
                const double4 *tx = (const double4 *)t, *tv = tx + n, *tw = tv + n;
                const uint32_t *rpre = (const uint32_t *)(t + 3 * n4);
                const uint32_t *rpost = rpre + (size_t)n * sph::NC;
                const double4 *th = (const double4 *)(rpost + (size_t)n * sph::NC);
                // the iteration index matters only as "the run's first step or not"
                const uint64_t it = first && k == 0 ? 0 : 1;
                rst = sph::adjoint_step(h->A.boxes, n, it, tx, tv, tw, rpre, rpost, th, ln, lc,
                                        lH, dscal, h->own);
                for (int q = 0; q < 5; ++q) std::swap(ln[q], lc[q]);
            }
        }
        SegGraph q{ns, kind, nullptr, nullptr};
        const cudaError_t ec = cudaStreamEndCapture(h->own, &q.g);
        if (rst != SPH_OK || ec != cudaSuccess) {
            if (q.g) cudaGraphDestroy(q.g);
            return rst != SPH_OK ? rst : SPH_ERR_CUDA;
        }
        if (cudaGraphInstantiate(&q.ge, q.g, 0) != cudaSuccess) {
            cudaGraphDestroy(q.g);
            return SPH_ERR_CUDA;
        }
        graphs.push_back(q);
        *out = q.ge;
        return SPH_OK;
    };
    // every segment shape's graphs captured first: a one-time set-up, kept
    // out of the timed backward pass as the forward's step graph is built
    // before the forward's time is taken
    {
        int par = 0;
        for (uint64_t sgm = nseg; e == cudaSuccess && st == SPH_OK && sgm-- > 0;) {
            const uint64_t ns = std::min<uint64_t>(ckpt, nsteps - sgm * ckpt);
            const bool first = sgm == 0 && h->adj_iter0 == 0;
            cudaGraphExec_t g0 = nullptr, g1 = nullptr;
            if ((st = seg_graph(ns, -1, &g0)) == SPH_OK) st = seg_graph(ns, (first ? 2 : 0) + par, &g1);
            if (ns & 1) par ^= 1;
        }
    }
    cudaEventRecord(ev[0], h->stream);
    int parity = 0;   // 1: the step after the last reversed one is in lcur0
    for (uint64_t sgm = nseg; e == cudaSuccess && st == SPH_OK && sgm-- > 0;) {
        copy_state(h, h->adj_snaps, sgm, false);
        const uint64_t ns = std::min<uint64_t>(ckpt, nsteps - sgm * ckpt);
        cudaGraphExec_t gr = nullptr, gb = nullptr;
        const bool first = sgm == 0 && h->adj_iter0 == 0;
        if ((st = seg_graph(ns, -1, &gr)) != SPH_OK ||
            (st = seg_graph(ns, (first ? 2 : 0) + parity, &gb)) != SPH_OK)
            break;
        if (cudaGraphLaunch(gr, h->stream) != cudaSuccess || cudaGraphLaunch(gb, h->stream) != cudaSuccess) {
            st = SPH_ERR_CUDA;
            break;
        }
        h->launches += ns * (h->launches_per_step + 2);
        if (ns & 1) parity ^= 1;
    }
    // the adjoints of the run's initial state
    for (int q = 0; q < 5; ++q) lnext[q] = parity ? lcur0[q] : lnext0[q];
    cudaEventRecord(ev[1], h->stream);
    cudaStreamSynchronize(h->stream);
    for (const SegGraph &q : graphs) {
        cudaGraphExecDestroy(q.ge);
        cudaGraphDestroy(q.g);
    }
    // leave the handle at the forward's final state
    copy_state(h, h->adj_snaps, nseg, false);
    double scal[3] = {0, 0, 0};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scal, dscal, sizeof scal, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && grad_v0)
        e = cudaMemcpyAsync(seed.data(), lnext[1], n4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    for (auto &x : ev) cudaEventDestroy(x);
    release();
    free_adjoint(h);
    if (st != SPH_OK) return fail(h, st, "adjoint launch failed");
    if (e != cudaSuccess)
        return fail(h, SPH_ERR_CUDA, std::string("adjoint: ") + cudaGetErrorString(e));
    if (grad_params)
        for (int k = 0; k < 3; ++k) grad_params[k] = scal[k];
    if (grad_v0)
        for (uint32_t i = 0; i < n; ++i) {
            grad_v0[3 * i] = seed[i].x;
            grad_v0[3 * i + 1] = seed[i].y;
            grad_v0[3 * i + 2] = seed[i].z;
        }
    if (adjoint_ms) *adjoint_ms = ms;
    return collect_errors(h);
}

// Drop the captured step graphs (they hold the kernel arguments and launch
// shapes); the next step captures them again.
static int drop_graphs(SphHandle *h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
    for (int k = 1; k < 4; ++k) {
        if (h->pexec_ph[k]) cudaGraphExecDestroy(h->pexec_ph[k]);
        if (h->pgraph_ph[k]) cudaGraphDestroy(h->pgraph_ph[k]);
        h->pexec_ph[k] = nullptr;
        h->pgraph_ph[k] = nullptr;
    }
    for (int r = 0; r < SphHandle::PR; ++r) {
        if (h->pexec[r]) cudaGraphExecDestroy(h->pexec[r]);
        if (h->pgraph[r]) cudaGraphDestroy(h->pgraph[r]);
        h->pexec[r] = nullptr;
        h->pgraph[r] = nullptr;
    }
    if (h->prof_on) return build_prof_graphs(h);
    return SPH_OK;
}

// Buffers of the split step, allocated when that variant is first chosen.
static int ensure_split(SphHandle *h)
{
    if (h->A.csum) return SPH_OK;
    const uint64_t n = h->ntot;
    // a live entry holds the sphere index in 27 bits
    if (n > (uint64_t)sph::SPLIT_ID_MASK + 1u)
        return fail(h, SPH_ERR_UNSUPPORTED, "split step: more than 2^27 spheres");
    uint2 *lent = nullptr;
    uint32_t *nlive = nullptr;
    sph::Acc *csum = nullptr;
    int st;
    if ((st = dalloc(h, &lent, n * sph::NC)) || (st = dalloc(h, &nlive, n)) ||
        (st = dalloc(h, &csum, n)))
        return st;
    h->A.lent = lent;
    h->A.nlive = nlive;
    h->A.csum = csum;
    return SPH_OK;
}

int sph_set_variant(SphHandle *h, int variant)
{
    if (!h) return SPH_ERR_INPUT;
    if (variant < 0 || variant >= sph::INTERACT_VARIANTS)
        return fail(h, SPH_ERR_INPUT, "variant out of range");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st = sync_public(h);
        if (st != SPH_OK) return st;
    }
    if (variant == sph::SPLIT_VARIANT) {
        int st = ensure_split(h);
        if (st != SPH_OK) return st;
    }
    if (variant == sph::PAIR_VARIANT && pair_eligible(h)) {
        int st = ensure_pair(h);
        if (st != SPH_OK) return st;
    }
    h->cfg.variant = variant;
    return drop_graphs(h);
}

int sph_set_launch_shape(SphHandle *h, int shape)
{
    if (!h) return SPH_ERR_INPUT;
    if (shape < 0 || shape >= sph::PAIR_SHAPES) return fail(h, SPH_ERR_INPUT, "shape out of range");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->cfg.pair_shape = shape;
    return drop_graphs(h);
}

int sph_get_tuning(const SphHandle *h, int *variant, int *shape)
{
    if (!h) return SPH_ERR_INPUT;
    if (variant) *variant = h->cfg.variant;
    if (shape) *shape = h->cfg.pair_shape;
    return SPH_OK;
}

int sph_get_shape_times(const SphHandle *h, double *ms, int n)
{
    if (!h || !ms || n < 0) return SPH_ERR_INPUT;
    for (int k = 0; k < n; ++k) ms[k] = k < sph::PAIR_SHAPES ? h->shape_ms[k] : -1.0;
    return SPH_OK;
}

int sph_autotune(SphHandle *h, uint32_t steps, double *ms_per_step, int *chosen)
{
    if (!h || steps == 0) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_autotune before sph_upload");
    if (h->darcy_on)
        return fail(h, SPH_ERR_UNSUPPORTED, "sph_autotune with the Darcy coupling (its timed "
                                            "steps would advance the fluid)");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st0 = sync_public(h);
        if (st0 != SPH_OK) return st0;
    }
    const size_t sb = state_bytes(h);
    char *snap = nullptr;
    if (cudaMalloc((void **)&snap, sb) != cudaSuccess)
        return fail(h, SPH_ERR_NOMEM, "no device memory for the autotune snapshot");
    const std::vector<double> t_saved = h->t_host;
    const uint64_t launches_saved = h->launches;
    copy_state(h, snap, 0, true);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = h->cfg.variant, best_shape = h->cfg.pair_shape, st = SPH_OK;
    double best_ms = 1e300;
    constexpr int NCAND = sph::INTERACT_VARIANTS - 1 + sph::PAIR_SHAPES;
    double cand_ms[NCAND];
    for (int t = 0; t < NCAND; ++t) cand_ms[t] = -1.0;
    // the variants, and the list step at each of its launch shapes; two
    // rounds over all of them, each candidate keeping its better time, so
    // that no candidate is picked or dropped on one run alone
    for (int u = 0; u < 2 * NCAND && st == SPH_OK; ++u) {
        const int t = u % NCAND;
        const int v = t < sph::INTERACT_VARIANTS ? t : sph::PAIR_VARIANT;
        const int shape = t < sph::PAIR_VARIANT ? 0 : t - sph::PAIR_VARIANT;
        // the split step needs contact models 2/3, fused integration,
        // neighbour lists and its buffers; otherwise it is not a candidate
        if (v == sph::SPLIT_VARIANT &&
            (!h->cfg.all_cm23 || h->cfg.unfused || !h->A.vlist || ensure_split(h) != SPH_OK))
            continue;
        // the list step: the FP32-mixed form's cases it covers
        if (v == sph::PAIR_VARIANT && (!pair_eligible(h) || ensure_pair(h) != SPH_OK)) continue;
        h->cfg.variant = v;
        h->cfg.pair_shape = shape;
        if ((st = drop_graphs(h)) != SPH_OK || (st = build_graph(h)) != SPH_OK) break;
        copy_state(h, snap, 0, false);
        invalidate_pair(h);
        if ((st = prepare_steps(h)) != SPH_OK) break;
        // one untimed step (graph upload, list build), then the timed ones
        if ((st = launch_one(h)) != SPH_OK) break;
        cudaEventRecord(e0, h->stream);
        for (uint32_t k = 0; k < steps && st == SPH_OK; ++k) st = launch_one(h);
        cudaEventRecord(e1, h->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = SPH_ERR_CUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double per = (double)ms / steps;
        if (cand_ms[t] < 0.0 || per < cand_ms[t]) cand_ms[t] = per;
    }
    if (ms_per_step)
        for (int v = 0; v < sph::INTERACT_VARIANTS; ++v) ms_per_step[v] = -1.0;
    for (int k = 0; k < sph::PAIR_SHAPES; ++k) h->shape_ms[k] = -1.0;
    for (int t = 0; t < NCAND; ++t) {
        if (cand_ms[t] < 0.0) continue;
        const int v = t < sph::INTERACT_VARIANTS ? t : sph::PAIR_VARIANT;
        const int shape = t < sph::PAIR_VARIANT ? 0 : t - sph::PAIR_VARIANT;
        const double per = cand_ms[t];
        if (v == sph::PAIR_VARIANT) h->shape_ms[shape] = per;
        if (ms_per_step && (ms_per_step[v] < 0.0 || per < ms_per_step[v])) ms_per_step[v] = per;
        if (per < best_ms) {
            best_ms = per;
            best = v;
            best_shape = shape;
        }
    }
    copy_state(h, snap, 0, false);
    invalidate_pair(h);
    cudaStreamSynchronize(h->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(snap);
    h->t_host = t_saved;
    h->launches = launches_saved;
    cudaMemset(h->A.err, 0, sizeof(uint32_t));
    h->cfg.variant = best;
    h->cfg.pair_shape = best_shape;
    const int st2 = drop_graphs(h);
    if (st != SPH_OK) return fail(h, st, "autotune step failed");
    if (chosen) *chosen = best;
    return st2;
}

int sph_porosity(SphHandle *h, uint32_t box, uint32_t z_slices, double *z_pos, double *porosity)
{
    if (!h || !z_pos || !porosity || z_slices == 0) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_porosity before sph_upload");
    if (box >= h->nbox) return fail(h, SPH_ERR_INPUT, "no such box");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st0 = sync_public(h);
        if (st0 != SPH_OK) return st0;
    }
    DevBox d;
    CUDA_TRY(h, cudaMemcpy(&d, h->A.boxes + box, sizeof d, cudaMemcpyDeviceToHost));
    // src/sphere.cpp:492-515: the top is wall 0 when there are walls
    const double top = d.nw > 0 ? d.wnx[0][3] : d.L[2];
    const double h_slice = (top - d.origo[2]) / (double)z_slices;
    if (h_slice <= h->rmax_box[box] * 2.0)
        return fail(h, SPH_ERR_INPUT, "the number of z-slices is too high (slab <= 2 r_max)");
    const double V_slice = h_slice * d.L[0] * d.L[1];
    double *dz = nullptr, *dp = nullptr;
    if (cudaMalloc((void **)&dz, sizeof(double) * z_slices) != cudaSuccess ||
        cudaMalloc((void **)&dp, sizeof(double) * z_slices) != cudaSuccess) {
        cudaFree(dz);
        return fail(h, SPH_ERR_NOMEM, "porosity buffers");
    }
    int st = sph::porosity_profile(h->A.x, d.p_base, d.np, h_slice, V_slice, z_slices, dz, dp,
                                   h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (st == SPH_OK && e == cudaSuccess) {
        e = cudaMemcpy(z_pos, dz, sizeof(double) * z_slices, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(porosity, dp, sizeof(double) * z_slices, cudaMemcpyDeviceToHost);
    }
    cudaFree(dz);
    cudaFree(dp);
    if (st != SPH_OK) return fail(h, st, "porosity kernel launch failed");
    if (e != cudaSuccess) return fail(h, SPH_ERR_CUDA, cudaGetErrorString(e));
    return SPH_OK;
}

int sph_overlaps(SphHandle *h, uint32_t box, uint64_t max_pairs, uint32_t *pairs, double *delta_n,
                 uint64_t *npairs)
{
    if (!h || !npairs) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_overlaps before sph_upload");
    if (box >= h->nbox) return fail(h, SPH_ERR_INPUT, "no such box");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st0 = sync_public(h);
        if (st0 != SPH_OK) return st0;
    }
    DevBox d;
    CUDA_TRY(h, cudaMemcpy(&d, h->A.boxes + box, sizeof d, cudaMemcpyDeviceToHost));
    sph::OverlapArgs O{};
    O.x = h->A.x;
    O.vel = h->A.vel;
    O.p0 = d.p_base;
    O.np = d.np;
    double cmin = 1e300;
    for (int c = 0; c < 3; ++c) {
        O.origo[c] = d.origo[c];
        O.cw[c] = d.L[c] / d.num[c];
        O.num[c] = (int)d.num[c];
        cmin = fmin(cmin, O.cw[c]);
    }
    O.R = (int)ceil(2.0 * h->rmax_box[box] / cmin);
    if (O.R < 1) O.R = 1;
    const uint64_t ncells = (uint64_t)d.num[0] * d.num[1] * d.num[2];
    const uint64_t n = d.np ? d.np : 1;
    if (n > 4096ull * 4096ull) return fail(h, SPH_ERR_UNSUPPORTED, "box too large for sph_overlaps");
    std::vector<void *> mine;
    auto get = [&](size_t bytes) -> void * {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) return nullptr;
        mine.push_back(q);
        return q;
    };
    auto release = [&]() {
        for (void *q : mine) cudaFree(q);
    };
    O.cell_of = (uint32_t *)get(4 * n);
    O.slot = (uint32_t *)get(4 * n);
    O.count = (uint32_t *)get(4 * (ncells + 1));
    O.coff = (uint32_t *)get(4 * (ncells + 1));
    O.items = (uint32_t *)get(4 * n);
    O.npair = (uint32_t *)get(4 * (n + 1));
    O.poff = (uint32_t *)get(4 * (n + 1));
    uint32_t *scan_tmp = (uint32_t *)get(4 * (ncells / 4096 + n / 4096 + 2));
    if (!O.cell_of || !O.slot || !O.count || !O.coff || !O.items || !O.npair || !O.poff ||
        !scan_tmp) {
        release();
        return fail(h, SPH_ERR_NOMEM, "overlap-search buffers");
    }
    int st = sph::find_overlaps(O, (uint32_t)ncells, scan_tmp, h->stream, 0);
    uint32_t total = 0;
    cudaError_t e = cudaSuccess;
    if (st == SPH_OK) {
        e = cudaMemcpyAsync(&total, O.poff + d.np, sizeof total, cudaMemcpyDeviceToHost,
                            h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    if (st == SPH_OK && e == cudaSuccess && total > 0 && max_pairs > 0 && (pairs || delta_n)) {
        O.pairs = (uint32_t *)get(8 * (size_t)total);
        O.delta = (double *)get(8 * (size_t)total);
        if (!O.pairs || !O.delta) {
            release();
            return fail(h, SPH_ERR_NOMEM, "overlap list buffers");
        }
        st = sph::find_overlaps(O, (uint32_t)ncells, scan_tmp, h->stream, 1);
        const uint64_t m = total < max_pairs ? total : max_pairs;
        if (st == SPH_OK && pairs)
            e = cudaMemcpyAsync(pairs, O.pairs, 8 * m, cudaMemcpyDeviceToHost, h->stream);
        if (st == SPH_OK && e == cudaSuccess && delta_n)
            e = cudaMemcpyAsync(delta_n, O.delta, 8 * m, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    release();
    if (st != SPH_OK) return fail(h, st, "overlap-search launch failed");
    if (e != cudaSuccess) return fail(h, SPH_ERR_CUDA, cudaGetErrorString(e));
    *npairs = total;
    return SPH_OK;
}

int sph_render(SphHandle *h, uint32_t box, int method, float maxval, float lower_cutoff,
               float focal_length, uint32_t width, uint32_t height, uint8_t *rgb)
{
    (void)focal_length;   // src/raytracer.cuh:313: the focal distance is 0.8 |eye - lookat|
    if (!h || !rgb) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_render before sph_upload");
    if (box >= h->nbox) return fail(h, SPH_ERR_INPUT, "no such box");
    if (method < 0 || method > 5)
        return fail(h, SPH_ERR_INPUT, "render method must be 0 (normal) to 5 (angpos)");
    if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 31))
        return fail(h, SPH_ERR_INPUT, "image size out of range");
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st0 = sync_public(h);
        if (st0 != SPH_OK) return st0;
    }
    DevBox d;
    CUDA_TRY(h, cudaMemcpy(&d, h->A.boxes + box, sizeof d, cudaMemcpyDeviceToHost));
    const double *d_L = reinterpret_cast<const double *>(
        reinterpret_cast<const char *>(h->A.boxes + box) + offsetof(DevBox, L));
    const size_t bytes = (size_t)width * height * 3;
    uint8_t *img = nullptr;
    if (cudaMalloc((void **)&img, bytes) != cudaSuccess)
        return fail(h, SPH_ERR_NOMEM, "image buffer");
    sph::RenderStats rs;
    int st = sph::render_image(h->A, d.p_base, d.np, d_L, method, maxval, lower_cutoff, width,
                               height, img, h->stream, &rs);
    h->launches += (uint64_t)rs.launches;
    cudaError_t e = cudaSuccess;
    if (st == SPH_OK) e = cudaMemcpy(rgb, img, bytes, cudaMemcpyDeviceToHost);
    cudaFree(img);
    if (st != SPH_OK) return fail(h, st, "ray-tracing kernels failed");
    if (e != cudaSuccess) return fail(h, SPH_ERR_CUDA, cudaGetErrorString(e));
    return SPH_OK;
}

int sph_set_neighbor_lists(SphHandle *h, uint32_t capacity)
{
    if (!h) return SPH_ERR_INPUT;
    if (capacity > (uint32_t)sph::VL_MAX)
        return fail(h, SPH_ERR_INPUT, "neighbour-list capacity above " + std::to_string(sph::VL_MAX));
    cudaSetDevice(h->device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    {
        int st = sync_public(h);
        if (st != SPH_OK) return st;
    }
    h->A.vlist = capacity ? h->vlist_mem : nullptr;
    h->A.vcap = capacity;
    CUDA_TRY(h, cudaMemset(h->A.vflag, 1, 1));
    return drop_graphs(h);
}

int sph_relax(SphHandle *h, uint32_t sweeps, double alpha, double z_top, double *max_overlap)
{
    if (!h || !(alpha > 0.0) || !(alpha <= 1.0)) return SPH_ERR_INPUT;
    if (!h->uploaded) return fail(h, SPH_ERR_STATE, "sph_relax before sph_upload");
    cudaSetDevice(h->device);
    {
        int st0 = sync_public(h);
        if (st0 != SPH_OK) return st0;
        invalidate_pair(h);   // the sweeps move the spheres in the FP64 arrays
    }
    uint64_t nl = 0;
    for (uint32_t k = 0; k < sweeps; ++k) {
        int st = sph::relax_sweep(h->A, h->stream, alpha, z_top, h->d_count, &nl);
        if (st != SPH_OK) return fail(h, st, "relax sweep launch failed");
    }
    h->launches += nl;
    unsigned long long bits = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&bits, h->d_count, sizeof bits, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    if (max_overlap) memcpy(max_overlap, &bits, sizeof(double));
    CUDA_TRY(h, cudaMemset(h->A.force, 0, sizeof(double4) * (h->ntot ? h->ntot : 1)));
    CUDA_TRY(h, cudaMemset(h->A.vflag, 1, 1));
    return collect_errors(h);
}

}  // extern "C"
