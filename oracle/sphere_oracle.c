/*
 * sphere_oracle.c -- TEST INFRASTRUCTURE ONLY (parity checker, never shipped).
 *
 * A plain-C FP64 restatement of the reference's DEM time step for
 * fluid == 0, used by tests/ and by bench.py's cpu_baseline leg to check and
 * time the CUDA path.  It follows, function by function:
 *   src/sorting.cuh:7-132          cell hash, sort, reorder
 *   src/contactsearch.cuh:12-726   periodic shift, topology, interact, walls
 *   src/contactmodels.cuh:10-600   contact laws
 *   src/cohesion.cuh:8-277         bonds, capillary cohesion
 *   src/integration.cuh:14-484     integrate, summation, integrateWalls
 *   src/device.cu:1031-2538        step order
 * Expressions keep the reference's operand order and its vector helpers
 * (src/vector_arithmetic.h) so that, compiled without FP contraction, the
 * results equal the reference's bit for bit.  Parity is pinned by running
 * the reference's own kernels on the CPU (oracle/ref_emu, libsphere_ref.so)
 * on the same inputs.
 *
 * Deliberate deviations from the reference (identical results otherwise):
 *  - contactmodels.cuh:500-559: contactHertz raises a negative overlap to
 *    fractional powers (NaN).  Here delta^(3/2) = delta*sqrt(|delta|) and
 *    delta^(1/4), delta^(1/2) act on |delta| (the evident intent).
 *  - contactmodels.cuh:320/487: the new tangential displacement is left
 *    uninitialised when both the old displacement and the sliding velocity
 *    have zero length; it is zero here.
 *  - contactsearch.cuh:267-299: when a row has no free slot the reference may
 *    write past the end of the particle's row; here such a write is dropped
 *    and SPH_ERR_NC_OVERFLOW is raised.
 *  - cohesion.cuh:30/205: a broken bond is marked with index nb0 and is
 *    active again when nb0 < np; here a bond broken during a run stays broken.
 *  - integration.cuh:57-62: wall0mode is uninitialised when nw == 0; here 0.
 *  - sorting.cuh:7-18: positions outside the grid give out-of-range cell ids;
 *    here they are clamped and SPH_ERR_OUT_OF_GRID is raised.
 *  - the bond scatter-add (cohesion.cuh:220-226) races between bonds that
 *    share a particle; here bonds are applied in ascending bond index.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "sphere_oracle.h"

#define NC SPH_NC
static const double PI = 3.14159265358979; /* src/constants.h:15 */
/* M_PI of the C library, which src/darcy.cuh uses */
static const double OR_DARCY_PI = 3.14159265358979323846;

typedef struct { double x, y, z; } v3;
static inline v3 mk(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vadds(v3 a, double b) { return mk(a.x + b, a.y + b, a.z + b); }
static inline v3 smul(double s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline v3 muls(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 divs(v3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline v3 vneg(v3 a) { return mk(-a.x, -a.y, -a.z); }
/* vector_arithmetic.h:304-307 */
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* vector_arithmetic.h:414-416 */
static inline v3 cross(v3 a, v3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 ld3(const double *p) { return mk(p[0], p[1], p[2]); }

typedef struct {
    const OrState *s;
    const SphParams *P;
    double origo[3], L[3];
    unsigned num[3];
    int periodic;
    unsigned np, nw;
    double dt;
    int lenmode;
} Ctx;

/* vector_arithmetic.h:317-320: length() is sqrtf() of the FP64 dot product */
static inline double vlen(const Ctx *c, v3 v)
{
    double d = dot(v, v);
    return c->lenmode ? sqrt(d) : (double)sqrtf((float)d);
}
static inline double fsqrtf(double d) { return (double)sqrtf((float)d); }

#define FLAG(s, code) __atomic_fetch_or(&(s)->error_flags, (int32_t)(1 << (code)), __ATOMIC_RELAXED)

/* ---------------------------------------------------------------- sorting */

/* sorting.cuh:7-20 calcCellID */
static unsigned calc_cell_id(const Ctx *c, OrState *s, const double *x)
{
    unsigned i[3];
    for (int d = 0; d < 3; ++d) {
        double f = floor((x[d] - c->origo[d]) / (c->L[d] / c->num[d]));
        if (!(f >= 0.0)) { FLAG(s, f != f ? SPH_ERR_NAN : SPH_ERR_OUT_OF_GRID); f = 0.0; }
        if (f >= (double)c->num[d]) { FLAG(s, SPH_ERR_OUT_OF_GRID); f = (double)(c->num[d] - 1); }
        i[d] = (unsigned)f;
    }
    return (i[2] * c->num[1]) * c->num[0] + i[1] * c->num[0] + i[0];
}

/* ---------------------------------------------------------- contact search */

/* contactsearch.cuh:12-83 findDistMod */
static int find_dist_mod(const Ctx *c, int t[3], v3 *dm)
{
    if (c->periodic == 1) {
        if (t[0] < 0) { t[0] += c->num[0]; *dm = vadd(*dm, mk(c->L[0], 0.0, 0.0)); }
        if (t[0] >= (int)c->num[0]) { t[0] -= c->num[0]; *dm = vsub(*dm, mk(c->L[0], 0.0, 0.0)); }
        if (t[1] < 0) { t[1] += c->num[1]; *dm = vadd(*dm, mk(0.0, c->L[1], 0.0)); }
        if (t[1] >= (int)c->num[1]) { t[1] -= c->num[1]; *dm = vsub(*dm, mk(0.0, c->L[1], 0.0)); }
    }
    if (c->periodic == 2) {
        if (t[0] < 0) { t[0] += c->num[0]; *dm = vadd(*dm, mk(c->L[0], 0.0, 0.0)); }
        if (t[0] >= (int)c->num[0]) { t[0] -= c->num[0]; *dm = vsub(*dm, mk(c->L[0], 0.0, 0.0)); }
        if (t[1] < 0 || t[1] >= (int)c->num[1]) return -1;
    }
    if (c->periodic > 2 || c->periodic < 1) {
        if (t[0] < 0 || t[0] >= (int)c->num[0]) return -1;
        if (t[1] < 0 || t[1] >= (int)c->num[1]) return -1;
    }
    if (t[2] < 0 || t[2] >= (int)c->num[2]) return -1;
    /* a particle far outside the grid can still be outside after one wrap */
    if (t[0] < 0 || t[0] >= (int)c->num[0] || t[1] < 0 || t[1] >= (int)c->num[1]) return -1;
    return 0;
}

static void grid_pos(const Ctx *c, const double *x, int g[3])
{
    for (int d = 0; d < 3; ++d)
        g[d] = (int)floor((x[d] - c->origo[d]) / (c->L[d] / c->num[d]));
}

/* contactsearch.cuh:194-322 findContactsInCell (slot insertion rule) */
static void find_contacts_in_cell(const Ctx *c, OrState *s, int t[3], unsigned idx_a,
                                  const double *x_a, double radius_a, int *nc)
{
    v3 distmod = mk(0.0, 0.0, 0.0);
    if (find_dist_mod(c, t, &distmod) == -1) return;
    unsigned cell = t[0] + t[1] * c->num[0] + (c->num[0] * c->num[1]) * t[2];
    unsigned start = s->cell_start[cell];
    if (start == 0xffffffffu) return;
    unsigned end = s->cell_end[cell];
    unsigned a_orig = s->perm[idx_a];
    for (unsigned idx_b = start; idx_b < end; ++idx_b) {
        if (idx_b == idx_a) continue;
        const double *x_b = s->x_sorted + 4 * (size_t)idx_b;
        double radius_b = x_b[3];
        unsigned b_orig = s->perm[idx_b];
        v3 x_ab = mk(x_a[0] - x_b[0], x_a[1] - x_b[1], x_a[2] - x_b[2]);
        x_ab = vadd(x_ab, distmod);
        double len = vlen(c, x_ab);
        double delta = len - (radius_a + radius_b);
        if (delta < 0.0) {
            int cpos = *nc;
            uint32_t *row = s->contacts + (size_t)a_orig * NC;
            for (int i = 0; i < NC; ++i) {
                uint32_t cidx = row[i];
                if (cidx == c->np) cpos = i;
                else if (cidx == b_orig) { cpos = i; break; }
            }
            if (cpos < NC) {
                row[cpos] = b_orig;
                double *dm = s->distmod + 4 * ((size_t)a_orig * NC + cpos);
                dm[0] = distmod.x; dm[1] = distmod.y; dm[2] = distmod.z; dm[3] = radius_b;
            } else {
                FLAG(s, SPH_ERR_NC_OVERFLOW);
            }
            ++*nc;
            if (*nc > NC) { FLAG(s, SPH_ERR_NC_OVERFLOW); return; }
        }
    }
}

/* contactsearch.cuh:329-371 topology */
static void topology(const Ctx *c, OrState *s)
{
    long n = (long)c->np;
#pragma omp parallel for schedule(dynamic, 256)
    for (long ia = 0; ia < n; ++ia) {
        unsigned idx_a = (unsigned)ia;
        const double *x_a = s->x_sorted + 4 * (size_t)idx_a;
        double radius_a = x_a[3];
        int nc = 0;
        int g[3];
        grid_pos(c, x_a, g);
        for (int dz = -1; dz < 2; ++dz)
            for (int dy = -1; dy < 2; ++dy)
                for (int dx = -1; dx < 2; ++dx) {
                    int t[3] = {g[0] + dx, g[1] + dy, g[2] + dz};
                    find_contacts_in_cell(c, s, t, idx_a, x_a, radius_a, &nc);
                }
    }
}

/* ----------------------------------------------------------- contact laws */

typedef struct { v3 F, T; double es_dot, ev_dot, p; } Acc;

/* contactmodels.cuh:10-117 contactLinear_wall */
static double contact_linear_wall(const Ctx *c, Acc *a, v3 vel_linear, v3 angvel,
                                  double radius_a, v3 n, double delta, double wvel)
{
    const SphParams *P = c->P;
    v3 vel = vadds(vadd(vel_linear, smul(radius_a + delta / 2.0, cross(n, angvel))), wvel);
    double vel_n = dot(vel_linear, n);
    v3 vel_t = vsub(vel, muls(n, dot(n, vel)));
    double vel_t_length = vlen(c, vel_t);
    double k_n = P->k_n;
    if (P->E > .001) k_n = 3.141592654 / 2.0 * P->E * radius_a;
    v3 f_n = smul(fmax(0.0, -k_n * delta - P->gamma_wn * vel_n), n);
    double f_n_length = vlen(c, f_n);
    a->ev_dot += P->gamma_wn * vel_n * vel_n;
    v3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_length > 0.0 && P->gamma_wt > 0.0) {
        v3 f_t_visc = smul(P->gamma_wt, vel_t);
        double f_t_visc_length = vlen(c, f_t_visc);
        double f_t_limit;
        if (vel_t_length > 0.0) f_t_limit = P->mu_wd * f_n_length;
        else f_t_limit = P->mu_ws * f_n_length;
        if (f_t_visc_length < f_t_limit) {
            f_t = smul(-1.0, f_t_visc);
        } else {
            f_t = divs(smul(-f_t_limit, vel_t), vel_t_length);
            a->es_dot += vlen(c, muls(smul(vlen(c, f_t), vel_t), c->dt)) / c->dt;
        }
    }
    a->F = vadd(a->F, vadd(f_n, f_t));
    a->T = vadd(a->T, cross(smul(-(radius_a + delta * 0.5), n), f_t));
    a->p += f_n_length / (4.0f * PI * radius_a * radius_a);
    return dot(f_n, n);
}

/* contactmodels.cuh:122-240 contactLinearViscous */
static void contact_linear_viscous(const Ctx *c, Acc *a, v3 vel_a, v3 vel_b, v3 angvel_a,
                                   v3 angvel_b, double radius_a, double radius_b, v3 x_ab,
                                   double x_ab_length, double delta_ab, double kappa)
{
    const SphParams *P = c->P;
    v3 n_ab = divs(x_ab, x_ab_length);
    v3 vel_ab_linear = vsub(vel_a, vel_b);
    v3 vel_ab = vadd(vadd(vel_ab_linear, smul(radius_a + delta_ab / 2.0f, cross(n_ab, angvel_a))),
                     smul(radius_b + delta_ab / 2.0f, cross(n_ab, angvel_b)));
    double vel_n_ab = dot(vel_ab_linear, n_ab);
    v3 vel_t_ab = vsub(vel_ab, muls(n_ab, dot(vel_ab, n_ab)));
    double vel_t_ab_length = vlen(c, vel_t_ab);
    double k_n = P->k_n;
    if (P->E > .001) k_n = 3.141592654 / 2.0 * P->E * (radius_a + radius_b) / 2.;
    v3 f_n = smul(fmax(0.0, -k_n * delta_ab - P->gamma_n * vel_n_ab), n_ab);
    if (dot(f_n, n_ab) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(c, f_n);
    v3 f_c = smul(-kappa * fsqrtf(radius_a * radius_b), n_ab);
    v3 f_t = mk(0.0, 0.0, 0.0);
    if (vel_t_ab_length > 0.0) {
        double f_t_visc = P->gamma_t * vel_t_ab_length;
        double f_t_limit;
        if (vel_t_ab_length > (double)0.001f) f_t_limit = P->mu_d * vlen(c, vsub(f_n, f_c));
        else f_t_limit = P->mu_s * vlen(c, vsub(f_n, f_c));
        if (f_t_visc < f_t_limit) f_t = divs(smul(-f_t_visc, vel_t_ab), vel_t_ab_length);
        else f_t = divs(smul(-f_t_limit, vel_t_ab), vel_t_ab_length);
    }
    a->F = vadd(a->F, vadd(vadd(f_n, f_t), f_c));
    a->T = vadd(a->T, smul(-(radius_a + delta_ab / 2.0f), cross(n_ab, f_t)));
    a->p += f_n_length / (4.0f * PI * radius_a * radius_a);
}

/* contactmodels.cuh:244-411 contactLinear; returns the new tangential
 * displacement through dt_out */
static void contact_linear(const Ctx *c, Acc *a, v3 vel_a, v3 vel_b, v3 angvel_a, v3 angvel_b,
                           double radius_a, double radius_b, v3 x, double x_length, double delta,
                           v3 delta_t0_uncor, v3 *dt_out)
{
    const SphParams *P = c->P;
    v3 n = divs(x, x_length);
    v3 vel_linear = vsub(vel_a, vel_b);
    v3 vel = vadd(vadd(vel_linear, smul(radius_a + delta / 2.0, cross(n, angvel_a))),
                  smul(radius_b + delta / 2.0, cross(n, angvel_b)));
    double vel_n = -dot(vel_linear, n);
    v3 vel_t = vsub(vel, muls(n, dot(n, vel)));
    double vel_t_length = vlen(c, vel_t);
    v3 delta_t0 = vsub(delta_t0_uncor, muls(n, dot(n, delta_t0_uncor)));
    double delta_t0_length = vlen(c, delta_t0);
    v3 delta_t = mk(0.0, 0.0, 0.0);
    double k_n = P->k_n, k_t = P->k_t;
    if (P->E > .001) {
        k_n = 3.141592654 / 2.0 * P->E * (radius_a + radius_b) / 2.;
        k_t = k_n;
    }
    v3 f_n = smul(fmax(0.0, -k_n * delta + P->gamma_n * vel_n), n);
    double f_n_length = vlen(c, f_n);
    a->ev_dot += 0.5 * P->gamma_n * vel_n * vel_n;
    v3 f_c = smul(-P->kappa * fsqrtf(radius_a * radius_b), n);
    v3 f_t = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.0 || vel_t_length > 0.0) {
        delta_t = vadd(delta_t0, muls(vel_t, c->dt));
        v3 f_t_elast = smul(-k_t, delta_t);
        v3 f_t_visc = smul(-P->gamma_t, vel_t);
        f_t = vadd(f_t_elast, f_t_visc);
        double f_t_length = vlen(c, f_t);
        double f_t_limit = P->mu_s * vlen(c, vsub(f_n, f_c));
        a->ev_dot += 0.5 * P->gamma_t * vel_t_length * vel_t_length;
        if (f_t_length > f_t_limit) {
            v3 t = divs(f_t, vlen(c, f_t));
            f_t = smul(f_t_limit, t);
            delta_t = smul(-1.0 / k_t, vadd(smul(P->mu_d * vlen(c, vsub(f_n, f_c)), t),
                                            smul(P->gamma_t, vel_t)));
            a->es_dot += 0.5 * vlen(c, muls(smul(vlen(c, f_t), vel_t), c->dt)) / c->dt;
        }
    }
    a->F = vadd(a->F, vadd(vadd(f_n, f_t), f_c));
    a->T = vadd(a->T, cross(smul(-(radius_a + delta * 0.5), n), f_t));
    a->p += f_n_length / (4.0f * PI * radius_a * radius_a);
    *dt_out = delta_t;
}

/* contactmodels.cuh:417-600 contactHertz, with the fractional powers taken of
 * the overlap magnitude (see header) */
static void contact_hertz(const Ctx *c, Acc *a, v3 vel_a, v3 vel_b, v3 angvel_a, v3 angvel_b,
                          double radius_a, double radius_b, v3 x_ab, double x_ab_length,
                          double delta_ab, v3 delta_t0_uncor, v3 *dt_out)
{
    const SphParams *P = c->P;
    double ad = fabs(delta_ab);
    double d12 = sqrt(ad);         /* |delta|^(1/2) */
    double d14 = sqrt(d12);        /* |delta|^(1/4) */
    double d32 = delta_ab * d12;   /* delta^(3/2), sign kept */
    v3 n_ab = divs(x_ab, x_ab_length);
    v3 vel_ab_linear = vsub(vel_a, vel_b);
    v3 vel_ab = vadd(vadd(vel_ab_linear, smul(radius_a + delta_ab / 2.0f, cross(n_ab, angvel_a))),
                     smul(radius_b + delta_ab / 2.0f, cross(n_ab, angvel_b)));
    v3 angvel_ab = vsub(angvel_a, angvel_b);
    double angvel_ab_length = vlen(c, angvel_ab);
    double vel_n_ab = dot(vel_ab_linear, n_ab);
    v3 vel_t_ab = vsub(vel_ab, muls(n_ab, dot(vel_ab, n_ab)));
    double vel_t_ab_length = vlen(c, vel_t_ab);
    v3 delta_t0 = vsub(delta_t0_uncor, muls(n_ab, dot(delta_t0_uncor, n_ab)));
    double delta_t0_length = vlen(c, delta_t0);
    v3 delta_t = mk(0.0, 0.0, 0.0);
    double k_n = P->k_n, k_t = P->k_t;
    if (P->E > .001) {
        k_n = 3.141592654 / 2.0 * P->E * (radius_a + radius_b) / 2.;
        k_t = k_n;
    }
    v3 f_n = smul(-k_n * d32 - P->gamma_n * d14 * vel_n_ab, n_ab);
    a->ev_dot += P->gamma_n * vel_n_ab * vel_n_ab;
    if (dot(f_n, n_ab) < 0.0f) f_n = mk(0.0, 0.0, 0.0);
    double f_n_length = vlen(c, f_n);
    v3 f_c = smul(-P->kappa * fsqrtf(radius_a * radius_b), n_ab);
    v3 f_t = mk(0.0, 0.0, 0.0);
    v3 T_res = mk(0.0, 0.0, 0.0);
    if (delta_t0_length > 0.f || vel_t_ab_length > 0.f) {
        v3 f_t_elast = smul(-k_t * d12, delta_t0);
        v3 f_t_visc = smul(-P->gamma_t * d14, vel_t_ab);
        double f_t_limit;
        if (vel_t_ab_length > (double)0.001f) f_t_limit = P->mu_d * vlen(c, vsub(f_n, f_c));
        else f_t_limit = P->mu_s * vlen(c, vsub(f_n, f_c));
        f_t = vadd(f_t_elast, f_t_visc);
        double f_t_length = vlen(c, f_t);
        if (f_t_length > f_t_limit) {
            f_t = muls(f_t, f_t_limit / f_t_length);
            delta_t = divs(vadd(f_t, smul(P->gamma_t * d14, vel_t_ab)), -k_t * d12);
            a->es_dot += vlen(c, vsub(delta_t0, delta_t)) * k_t / c->dt;
        } else {
            delta_t = vadd(delta_t0, muls(vel_t_ab, c->dt));
        }
    }
    if (angvel_ab_length > 0.f) {
        T_res = divs(smul(-1.0f * fmin(P->gamma_r * radius_a * angvel_ab_length,
                                       P->mu_r * radius_a * f_n_length), angvel_ab),
                     angvel_ab_length);
    }
    a->F = vadd(a->F, vadd(vadd(f_n, f_t), f_c));
    a->T = vadd(a->T, vadd(smul(-(radius_a + delta_ab / 2.0f), cross(n_ab, f_t)), T_res));
    a->p += f_n_length / (4.0f * PI * radius_a * radius_a);
    *dt_out = delta_t;
}

/* cohesion.cuh:237-277 capillaryCohesion_exp */
static void capillary_cohesion_exp(const Ctx *c, Acc *a, double radius_a, double radius_b,
                                   double delta_ab, v3 x_ab, double x_ab_length, double kappa)
{
    v3 n_ab = divs(x_ab, x_ab_length);
    double r;
    if ((radius_a / radius_b) > (radius_b / radius_a)) r = radius_a / radius_b;
    else r = radius_b / radius_a;
    double h = -fsqrtf(r);
    double R_har = (2.0f * radius_a * radius_b) / (radius_a + radius_b);
    double R_geo = fsqrtf(radius_a * radius_b);
    double lambda = (double)0.9f * h * fsqrtf(c->P->V_b / R_har);
    v3 f_c = smul(-kappa * R_geo * (double)expf((float)(-delta_ab / lambda)), n_ab);
    a->F = vadd(a->F, f_c);
}

/* contactsearch.cuh:91-186 findAndProcessContactsInCell (contact model 1) */
static void find_and_process_in_cell(const Ctx *c, OrState *s, int t[3], unsigned idx_a,
                                     const double *x_a, double radius_a, Acc *a)
{
    v3 distmod = mk(0.0, 0.0, 0.0);
    if (find_dist_mod(c, t, &distmod) == -1) return;
    unsigned cell = t[0] + t[1] * c->num[0] + (c->num[0] * c->num[1]) * t[2];
    unsigned start = s->cell_start[cell];
    if (start == 0xffffffffu) return;
    unsigned end = s->cell_end[cell];
    for (unsigned idx_b = start; idx_b < end; ++idx_b) {
        if (idx_b == idx_a) continue;
        const double *x_b = s->x_sorted + 4 * (size_t)idx_b;
        double radius_b = x_b[3];
        double kappa = c->P->kappa;
        v3 x_ab = mk(x_a[0] - x_b[0], x_a[1] - x_b[1], x_a[2] - x_b[2]);
        x_ab = vadd(x_ab, distmod);
        double x_ab_length = vlen(c, x_ab);
        double delta_ab = x_ab_length - (radius_a + radius_b);
        if (delta_ab < 0.0f) {
            contact_linear_viscous(c, a, ld3(s->vel_sorted + 4 * (size_t)idx_a),
                                   ld3(s->vel_sorted + 4 * (size_t)idx_b),
                                   ld3(s->angvel_sorted + 4 * (size_t)idx_a),
                                   ld3(s->angvel_sorted + 4 * (size_t)idx_b), radius_a, radius_b,
                                   x_ab, x_ab_length, delta_ab, kappa);
        } else if (delta_ab < c->P->db) {
            capillary_cohesion_exp(c, a, radius_a, radius_b, delta_ab, x_ab, x_ab_length, kappa);
        }
    }
}

/* contactsearch.cuh:385-726 interact */
static void interact(const Ctx *c, OrState *s)
{
    const SphParams *P = c->P;
    const SphWalls *W = &s->box.walls;
    long n = (long)c->np;
    /* default wall normals and positions, contactsearch.cuh:431-443 */
    double wnx[5][4] = {{0.0, 0.0, -1.0, c->L[2]}, {-1.0, 0.0, 0.0, c->L[0]},
                        {1.0, 0.0, 0.0, 0.0},      {0.0, -1.0, 0.0, c->L[1]},
                        {0.0, 1.0, 0.0, 0.0}};
    double wmvfd[5][4] = {{0}};
    for (unsigned w = 0; w < 5 && w < c->nw; ++w)
        for (int k = 0; k < 4; ++k) { wnx[w][k] = W->nx[w][k]; wmvfd[w][k] = W->mvfd[w][k]; }

#pragma omp parallel for schedule(dynamic, 256)
    for (long ia = 0; ia < n; ++ia) {
        unsigned idx_a = (unsigned)ia;
        unsigned a_orig = s->perm[idx_a];
        const double *x_a = s->x_sorted + 4 * (size_t)idx_a;
        double radius_a = x_a[3];
        Acc a;
        a.F = mk(0.0, 0.0, 0.0); a.T = mk(0.0, 0.0, 0.0);
        a.es_dot = 0.0; a.ev_dot = 0.0; a.p = 0.0;
        v3 vel_a = ld3(s->vel_sorted + 4 * (size_t)idx_a);
        v3 angvel_a = ld3(s->angvel_sorted + 4 * (size_t)idx_a);

        if (P->contactmodel == 2 || P->contactmodel == 3) {
            for (int i = 0; i < NC; ++i) {
                size_t mempos = (size_t)a_orig * NC + i;
                uint32_t b_orig = s->contacts[mempos];
                double *dt4 = s->delta_t + 4 * mempos;
                if (b_orig != c->np) {
                    const double *dm = s->distmod + 4 * mempos;
                    const double *x_b = s->x + 4 * (size_t)b_orig;
                    double radius_b = x_b[3];
                    v3 x_ab = mk(x_a[0] - x_b[0] + dm[0], x_a[1] - x_b[1] + dm[1],
                                 x_a[2] - x_b[2] + dm[2]);
                    double x_ab_length = vlen(c, x_ab);
                    double delta_n = x_ab_length - (radius_a + radius_b);
                    if (delta_n < 0.0) {
                        v3 nd;
                        v3 vel_b = ld3(s->vel + 4 * (size_t)b_orig);
                        v3 angvel_b = ld3(s->angvel + 4 * (size_t)b_orig);
                        if (P->contactmodel == 2)
                            contact_linear(c, &a, vel_a, vel_b, angvel_a, angvel_b, radius_a,
                                           radius_b, x_ab, x_ab_length, delta_n, ld3(dt4), &nd);
                        else
                            contact_hertz(c, &a, vel_a, vel_b, angvel_a, angvel_b, radius_a,
                                          radius_b, x_ab, x_ab_length, delta_n, ld3(dt4), &nd);
                        dt4[0] = nd.x; dt4[1] = nd.y; dt4[2] = nd.z; dt4[3] = 0.0;
                    } else {
                        s->contacts[mempos] = c->np;
                        dt4[0] = dt4[1] = dt4[2] = dt4[3] = 0.0;
                    }
                } else {
                    dt4[0] = dt4[1] = dt4[2] = dt4[3] = 0.0;
                }
            }
        } else if (P->contactmodel == 1) {
            int g[3];
            grid_pos(c, x_a, g);
            for (int dz = -1; dz < 2; ++dz)
                for (int dy = -1; dy < 2; ++dy)
                    for (int dx = -1; dx < 2; ++dx) {
                        int t[3] = {g[0] + dx, g[1] + dy, g[2] + dz};
                        find_and_process_in_cell(c, s, t, idx_a, x_a, radius_a, &a);
                    }
        }

        /* walls, contactsearch.cuh:602-701 */
        double wf[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        double delta_w;
        v3 w_n;
        delta_w = wnx[0][3] - (x_a[2] + radius_a);
        w_n = mk(wnx[0][0], wnx[0][1], wnx[0][2]);
        if (delta_w < 0.0f)
            wf[0] = contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, wmvfd[0][1]);
        delta_w = x_a[2] - radius_a - c->origo[2];
        w_n = mk(0.0f, 0.0f, 1.0f);
        if (delta_w < 0.0f)
            (void)contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, 0.0);
        if (c->periodic == 0) {
            delta_w = wnx[1][3] - (x_a[0] + radius_a);
            w_n = mk(wnx[1][0], wnx[1][1], wnx[1][2]);
            if (delta_w < 0.0f)
                wf[1] = contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, wmvfd[1][1]);
            delta_w = x_a[0] - radius_a - wnx[2][3];
            w_n = mk(wnx[2][0], wnx[2][1], wnx[2][2]);
            if (delta_w < 0.0f)
                wf[2] = contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, wmvfd[2][1]);
        }
        if (c->periodic == 0 || c->periodic == 2) {
            delta_w = wnx[3][3] - (x_a[1] + radius_a);
            w_n = mk(wnx[3][0], wnx[3][1], wnx[3][2]);
            if (delta_w < 0.0f)
                wf[3] = contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, wmvfd[3][1]);
            delta_w = x_a[1] - radius_a - wnx[4][3];
            w_n = mk(wnx[4][0], wnx[4][1], wnx[4][2]);
            if (delta_w < 0.0f)
                wf[4] = contact_linear_wall(c, &a, vel_a, angvel_a, radius_a, w_n, delta_w, wmvfd[4][1]);
        }

        /* contactsearch.cuh:707-724 */
        double *f = s->force + 4 * (size_t)a_orig;
        double *tq = s->torque + 4 * (size_t)a_orig;
        f[0] = a.F.x; f[1] = a.F.y; f[2] = a.F.z; f[3] = 0.0;
        tq[0] = a.T.x; tq[1] = a.T.y; tq[2] = a.T.z; tq[3] = 0.0;
        s->es_dot[a_orig] = a.es_dot;
        s->ev_dot[a_orig] = a.ev_dot;
        s->es[a_orig] += a.es_dot * c->dt;
        s->ev[a_orig] += a.ev_dot * c->dt;
        s->p[a_orig] = a.p;
        for (unsigned w = 0; w < 5 && w < c->nw; ++w)
            s->walls_force_pp[a_orig + (size_t)w * c->np] = wf[w];
    }
}

/* ------------------------------------------------------------------ bonds */

/* cohesion.cuh:8-233 bondsLinear, applied in ascending bond order */
static void bonds_linear(const Ctx *c, OrState *s, uint8_t *broken)
{
    const SphParams *P = c->P;
    const double dt = c->dt;
    for (uint32_t k = 0; k < s->box.nb0; ++k) {
        uint32_t bx = s->bonds[2 * k], by = s->bonds[2 * k + 1];
        if (!(bx < c->np) || broken[k]) continue;
        double *d4 = s->bonds_delta + 4 * (size_t)k;
        double *o4 = s->bonds_omega + 4 * (size_t)k;
        v3 delta0_t = ld3(d4);
        double delta0_n = d4[3];
        v3 omega0_t = ld3(o4);
        double omega0_n = o4[3];
        const double *x_i = s->x + 4 * (size_t)bx, *x_j = s->x + 4 * (size_t)by;
        v3 vel_i = ld3(s->vel + 4 * (size_t)bx), vel_j = ld3(s->vel + 4 * (size_t)by);
        v3 angvel_i = ld3(s->angvel + 4 * (size_t)bx), angvel_j = ld3(s->angvel + 4 * (size_t)by);
        double R_bar = P->lambda_bar * fmin(x_i[3], x_j[3]);
        double A = PI * R_bar * R_bar;
        double I = 0.25 * PI * R_bar * R_bar * R_bar * R_bar;
        double J = I * 2.0;
        v3 x = mk(x_i[0] - x_j[0], x_i[1] - x_j[1], x_i[2] - x_j[2]);
        double x_length = vlen(c, x);
        double overlap = fmin(0.0, x_length - (x_i[3] + x_j[3]));
        v3 n = divs(x, x_length);
        delta0_t = vsub(delta0_t, muls(n, dot(n, delta0_t)));
        v3 ddelta = muls(vadd(vadd(vsub(vel_i, vel_j), smul(x_i[3] + overlap / 2.0, cross(n, angvel_i))),
                              smul(x_j[3] + overlap / 2.0, cross(n, angvel_j))),
                         dt);
        double ddelta_n = -dot(ddelta, n);
        double delta_n = delta0_n + ddelta_n;
        v3 ddelta_t = vsub(ddelta, muls(n, dot(n, ddelta)));
        v3 delta_t = vadd(delta0_t, ddelta_t);
        v3 f_n = smul(P->k_n * A * delta_n + P->gamma_n * ddelta_n / dt, n);
        v3 f_t = vsub(smul(-P->k_t * A, delta_t), divs(smul(P->gamma_t, ddelta_t), dt));
        v3 f = vadd(f_n, f_t);
        v3 nn = vneg(n);
        omega0_t = vsub(omega0_t, muls(nn, dot(omega0_t, nn)));
        v3 domega = muls(vsub(angvel_j, angvel_i), dt);
        double domega_n = dot(domega, nn);
        double omega_n = omega0_n + domega_n;
        v3 domega_t = vsub(domega, smul(domega_n, nn));
        v3 omega_t = vadd(omega0_t, domega_t);
        v3 t_n = smul(-P->k_t * J * omega_n, nn);
        v3 t_t = smul(-P->k_n * I, omega_t);
        v3 t_j = vadd(t_n, t_t);
        double sigma_max = vlen(c, f_n) / A + vlen(c, t_t) * R_bar / I;
        double tau_max = vlen(c, f_t) / A + vlen(c, t_n) * R_bar / J;
        if (sigma_max >= P->sigma_b || tau_max >= P->tau_b) {
            s->bonds[2 * k] = s->box.nb0;
            broken[k] = 1;
            continue;
        }
        d4[0] = delta_t.x; d4[1] = delta_t.y; d4[2] = delta_t.z; d4[3] = delta_n;
        o4[0] = omega_t.x; o4[1] = omega_t.y; o4[2] = omega_t.z; o4[3] = omega_n;
        double *fi = s->force + 4 * (size_t)bx, *fj = s->force + 4 * (size_t)by;
        double *ti = s->torque + 4 * (size_t)bx, *tj = s->torque + 4 * (size_t)by;
        fi[0] += f.x; fi[1] += f.y; fi[2] += f.z; fi[3] += 0.0;
        fj[0] -= f.x; fj[1] -= f.y; fj[2] -= f.z; fj[3] -= 0.0;
        ti[0] -= t_j.x; ti[1] -= t_j.y; ti[2] -= t_j.z; ti[3] -= 0.0;
        tj[0] += t_j.x; tj[1] += t_j.y; tj[2] += t_j.z; tj[3] += 0.0;
    }
}

/* ------------------------------------------------------------ integration */

/* integration.cuh:309-341 summation: per-block tree reduction of in[0:np] */
static void summation(unsigned np, const double *in, double *out)
{
    unsigned blocks = (np + 255) / 256;
    for (unsigned b = 0; b < blocks; ++b) {
        double cache[256];
        for (unsigned t = 0; t < 256; ++t) {
            double temp = 0.0f;
            unsigned idx = b * 256 + t;
            if (idx < np) temp += in[idx];
            cache[t] = temp;
        }
        for (unsigned i = 128; i != 0; i /= 2)
            for (unsigned t = 0; t < i; ++t) cache[t] += cache[t + i];
        out[b] = cache[0];
    }
}

/* integration.cuh:457-484 findShearStressOnFixedMovingParticles */
static void find_shear_stress(const Ctx *c, OrState *s)
{
    for (unsigned i = 0; i < c->np; ++i) {
        double z = s->x[4 * (size_t)i + 2];
        double fixvel = s->vel[4 * (size_t)i + 3];
        double force_x = s->force[4 * (size_t)i];
        double f_x = 0.0;
        if (fixvel > 0.0 && z > c->L[2] * 0.5) f_x = force_x;
        s->tau_eff_x_pp[i] = f_x / (c->L[0] * c->L[1]);
    }
}

/* integration.cuh:14-305 integrate (TY3) */
static void integrate(const Ctx *c, OrState *s, int change_velocity_state)
{
    const SphParams *P = c->P;
    const SphWalls *W = &s->box.walls;
    const double dt = c->dt;
    const double velocity_factor = 10.0; /* device.cu:996 */
    unsigned blocks = (c->np + 255) / 256;
    int wall0mode = 0;
    double wall0mass = 0.0;
    if (c->nw > 0) { wall0mode = W->wmode[0]; wall0mass = W->mvfd[0][0]; }
    double tau_eff_x = 0.0;
    if (c->nw > 0 && wall0mode == 3)
        for (unsigned i = 0; i < blocks; ++i) tau_eff_x += s->tau_eff_x_partial[i];
    const double tau_x = W->tau_x;
    long n = (long)c->np;
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < n; ++ii) {
        unsigned idx = (unsigned)ii;
        unsigned o = s->perm[idx];
        const double *force = s->force + 4 * (size_t)o;
        const double *torque = s->torque + 4 * (size_t)o;
        const double *angpos = s->angpos + 4 * (size_t)o;
        const double *x = s->x_sorted + 4 * (size_t)idx;
        const double *vel = s->vel_sorted + 4 * (size_t)idx;
        const double *angvel = s->angvel_sorted + 4 * (size_t)idx;
        double xyzsum[4];
        memcpy(xyzsum, s->xyzsum + 4 * (size_t)o, sizeof(xyzsum));
        double acc0[4] = {0.0, 0.0, 0.0, 0.0}, angacc0[4] = {0.0, 0.0, 0.0, 0.0};
        if (s->iter != 0) {
            memcpy(acc0, s->acc + 4 * (size_t)o, sizeof(acc0));
            memcpy(angacc0, s->angacc + 4 * (size_t)o, sizeof(angacc0));
        }
        const double radius = x[3];
        double m = 4.0 / 3.0 * PI * radius * radius * radius * P->rho;
        double acc[4] = {0.0, 0.0, 0.0, 0.0}, angacc[4] = {0.0, 0.0, 0.0, 0.0};
        acc[0] = force[0] / m + P->g[0];
        acc[1] = force[1] / m + P->g[1];
        acc[2] = force[2] / m + P->g[2];
        angacc[0] = torque[0] * 1.0 / (2.0 / 5.0 * m * radius * radius);
        angacc[1] = torque[1] * 1.0 / (2.0 / 5.0 * m * radius * radius);
        angacc[2] = torque[2] * 1.0 / (2.0 / 5.0 * m * radius * radius);
        if (wall0mode == 3 && vel[3] > 0.0001 && x[2] > c->L[2] * 0.5) {
            const double f_tau_x = (tau_x + tau_eff_x) * c->L[0] * c->L[1];
            acc[0] = f_tau_x / wall0mass;
            acc[1] = 0.0;
            acc[2] -= P->g[2];
            angacc[0] = angacc[1] = angacc[2] = angacc[3] = 0.0;
        } else if (vel[3] > 0.0001 && vel[3] < 10.0) {
            acc[0] = 0.0;
            acc[1] = 0.0;
            acc[2] -= P->g[2];
            angacc[0] = angacc[1] = angacc[2] = angacc[3] = 0.0;
        }
        if (vel[3] >= 10.0) { acc[1] = 0.0; angacc[0] = 0.0; angacc[2] = 0.0; }
        if (vel[3] < -0.0001) {
            acc[0] = acc[1] = acc[2] = 0.0;
            angacc[0] = angacc[1] = angacc[2] = angacc[3] = 0.0;
        }
        double x_new[4], vel_new[4], angpos_new[4], angvel_new[4];
        for (int d = 0; d < 3; ++d) {
            const double dacc = (acc[d] - acc0[d]) / dt;
            const double dangacc = (angacc[d] - angacc0[d]) / dt;
            x_new[d] = x[d] + vel[d] * dt + 0.5 * acc[d] * dt * dt + 1.0 / 6.0 * dacc * dt * dt * dt;
            vel_new[d] = vel[d] + acc[d] * dt + 0.5 * dacc * dt * dt;
            angpos_new[d] = angpos[d] + angvel[d] * dt + 0.5 * angacc[d] * dt * dt +
                            1.0 / 6.0 * dangacc * dt * dt * dt;
            angvel_new[d] = angvel[d] + angacc[d] * dt + 0.5 * dangacc * dt * dt;
            xyzsum[d] += vel[d] * dt + 0.5 * acc[d] * dt * dt + 1.0 / 6.0 * dacc * dt * dt * dt;
        }
        x_new[3] = x[3];
        vel_new[3] = vel[3];
        angpos_new[3] = angpos[3];
        angvel_new[3] = angvel[3];
        if (c->periodic == 1) {
            if (x_new[0] < c->origo[0]) x_new[0] += c->L[0];
            if (x_new[0] > c->L[0]) x_new[0] -= c->L[0];
            if (x_new[1] < c->origo[1]) x_new[1] += c->L[1];
            if (x_new[1] > c->L[1]) x_new[1] -= c->L[1];
        } else if (c->periodic == 2) {
            if (x_new[0] < c->origo[0]) x_new[0] += c->L[0];
            if (x_new[0] > c->L[0]) x_new[0] -= c->L[0];
        }
        if (vel[3] > 5.0 && vel[3] < 10.0) {
            if (change_velocity_state == 1) vel_new[0] *= velocity_factor;
            else if (change_velocity_state == -1) vel_new[0] /= velocity_factor;
        }
        memcpy(s->xyzsum + 4 * (size_t)o, xyzsum, sizeof(xyzsum));
        memcpy(s->acc + 4 * (size_t)o, acc, sizeof(acc));
        memcpy(s->angacc + 4 * (size_t)o, angacc, sizeof(angacc));
        memcpy(s->angvel + 4 * (size_t)o, angvel_new, sizeof(angvel_new));
        memcpy(s->vel + 4 * (size_t)o, vel_new, sizeof(vel_new));
        memcpy(s->angpos + 4 * (size_t)o, angpos_new, sizeof(angpos_new));
        memcpy(s->x + 4 * (size_t)o, x_new, sizeof(x_new));
    }
}

/* integration.cuh:344-450 integrateWalls (TY3) */
static void integrate_walls(const Ctx *c, OrState *s, double t_current)
{
    const SphParams *P = c->P;
    SphWalls *W = &s->box.walls;
    unsigned blocks = (c->np + 255) / 256;
    const double dt = c->dt;
    for (unsigned idx = 0; idx < c->nw; ++idx) {
        double *w_nx = W->nx[idx];
        double *w_mvfd = W->mvfd[idx];
        int wmode = W->wmode[idx];
        if (wmode == 0) continue;
        double acc0 = (s->iter == 0) ? 0.0 : s->walls_acc[idx];
        w_mvfd[2] = 0.0;
        for (unsigned i = 0; i < blocks; ++i) w_mvfd[2] += s->walls_force_partial[i];
        const double sigma_0 = w_mvfd[3] + P->sigma0_A * sin(2.0 * PI * P->sigma0_f * t_current);
        const double N = -sigma_0 * c->L[0] * c->L[1];
        double acc = (w_mvfd[2] + N) / w_mvfd[0];
        if (wmode == 2) acc = 0.0;
        const double dacc_dt = (acc - acc0) / dt;
        w_nx[3] += w_mvfd[1] * dt + 0.5 * acc * dt * dt + 1.0 / 6.0 * dacc_dt * dt * dt * dt;
        w_mvfd[1] += acc * dt + 0.5 * dacc_dt * dt * dt;
        s->walls_acc[idx] = acc;
    }
}

/* ------------------------------------------------------------------ Darcy */

/* The Darcy coupling (fluid == 1, cfd_solver == 1), src/darcy.cuh and the
 * Darcy part of the step loop, src/device.cu:1891-2419.  Each function is
 * one kernel, run over the cells (or spheres) in launch order; none reads a
 * value that another thread of the same launch writes, except where
 * noted, so the order of the threads does not matter. */

typedef struct {
    OrDarcy *d;
    const SphDarcy *P;
    int nx, ny, nz;
    double dx, dy, dz;
} Dc;

static void ctx_init(Ctx *c, OrState *s);

/* darcy.cuh:146-157 d_idx (navierstokes.cuh:231-240 idx is the same) */
static inline uint32_t d_idx(const Dc *c, int x, int y, int z)
{
    return (uint32_t)(x + 1) + (uint32_t)(c->nx + 2) * (uint32_t)(y + 1) +
           (uint32_t)(c->nx + 2) * (uint32_t)(c->ny + 2) * (uint32_t)(z + 1);
}

/* darcy.cuh:346-349 sphereVolume: 4/3 pi r^3 with the C library's M_PI */
static inline double sphere_volume(double r) { return 4.0 / 3.0 * OR_DARCY_PI * pow(r, 3); }

/* darcy.cuh:356-385 weight / weightDist of the vector between the points */
static inline double weight_dist(v3 x, double dx, double dy, double dz)
{
    const v3 dist = mk(fabs(x.x), fabs(x.y), fabs(x.z));
    if (dist.x < dx && dist.y < dy && dist.z < dz)
        return (1.0 - dist.x / dx) * (1.0 - dist.y / dy) * (1.0 - dist.z / dz);
    return 0.0;
}

/* darcy.cuh:212-285 setDarcyGhostNodes (m doubles per cell) */
static void darcy_ghost(const Dc *c, double *f, int m)
{
    const SphDarcy *P = c->P;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double val[3];
                memcpy(val, f + (size_t)m * d_idx(c, x, y, z), sizeof(double) * m);
#define PUT(X, Y, Z) memcpy(f + (size_t)m * d_idx(c, X, Y, Z), val, sizeof(double) * m)
                if (x == 0 && P->bc_xn == 0) PUT(-1, y, z);
                if (x == 1 && P->bc_xn == 1) PUT(-1, y, z);
                if (x == 0 && P->bc_xn == 2) PUT(nx, y, z);
                if (x == nx - 1 && P->bc_xp == 0) PUT(nx, y, z);
                if (x == nx - 2 && P->bc_xp == 1) PUT(nx, y, z);
                if (x == nx - 1 && P->bc_xp == 2) PUT(-1, y, z);
                if (y == 0 && P->bc_yn == 0) PUT(x, -1, z);
                if (y == 1 && P->bc_yn == 1) PUT(x, -1, z);
                if (y == 0 && P->bc_yn == 2) PUT(x, ny, z);
                if (y == ny - 1 && P->bc_yp == 0) PUT(x, ny, z);
                if (y == ny - 2 && P->bc_yp == 1) PUT(x, ny, z);
                if (y == ny - 1 && P->bc_yp == 2) PUT(x, -1, z);
                if (z == 0 && P->bc_bot == 0) PUT(x, y, -1);
                if (z == 1 && P->bc_bot == 1) PUT(x, y, -1);
                if (z == 0 && P->bc_bot == 2) PUT(x, y, nz);
                if (z == nz - 1 && P->bc_top == 0) PUT(x, y, nz);
                if (z == nz - 2 && P->bc_top == 1) PUT(x, y, nz);
                if (z == nz - 1 && P->bc_top == 2) PUT(x, y, -1);
#undef PUT
            }
}

/* darcy.cuh:288-329 setDarcyGhostNodesFlux */
static void darcy_ghost_flux(const Dc *c, double *f, const double *k, double L2)
{
    const SphDarcy *P = c->P;
    if (!(P->bc_bot == 4 || P->bc_top == 4)) return;
    const int nx = c->nx, ny = c->ny, nz = c->nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const double p = f[d_idx(c, x, y, z)];
                const double kk = k[d_idx(c, x, y, z)];
                const double dz = L2 / nz;
                double q_z = 0.;
                if (z == 0) q_z = P->bc_bot_flux;
                else if (z == nz - 1) q_z = P->bc_top_flux;
                const double p_ghost = -P->mu / kk * q_z * dz + p;
                if (z == 0 && P->bc_bot == 4) f[d_idx(c, x, y, -1)] = p_ghost;
                if (z == nz - 1 && P->bc_top == 4) f[d_idx(c, x, y, nz)] = p_ghost;
            }
}

/* darcy.cuh:1101-1157 findDarcyPressureGradient (also
 * findDarcyPermeabilityGradients, :1535-1593: the same central difference) */
static void darcy_gradient(const Dc *c, const double *f, double *g)
{
    for (int z = 0; z < c->nz; ++z)
        for (int y = 0; y < c->ny; ++y)
            for (int x = 0; x < c->nx; ++x) {
                const double xn = f[d_idx(c, x - 1, y, z)], xp = f[d_idx(c, x + 1, y, z)];
                const double yn = f[d_idx(c, x, y - 1, z)], yp = f[d_idx(c, x, y + 1, z)];
                const double zn = f[d_idx(c, x, y, z - 1)], zp = f[d_idx(c, x, y, z + 1)];
                double *o = g + 3 * (size_t)d_idx(c, x, y, z);
                o[0] = (xp - xn) / (c->dx + c->dx);
                o[1] = (yp - yn) / (c->dy + c->dy);
                o[2] = (zp - zn) / (c->dz + c->dz);
            }
}

/* darcy.cuh:1160-1318 findDarcyPressureForceLinear, per sphere (original
 * order): the pressure gradient interpolated from the 27 cells around the
 * sphere's cell, times the sphere volume, plus buoyancy; added to the
 * sphere's force.  The index sums are unsigned as in the reference (a
 * sphere in the bottom layer compares 0xffffffff with wall0_iz - 1). */
static void darcy_force(const Ctx *c, const Dc *dc, OrState *s)
{
    const OrDarcy *D = dc->d;
    const SphDarcy *P = dc->P;
    const uint32_t nx = c->num[0], ny = c->num[1], nz = c->num[2];
    for (unsigned i = 0; i < c->np; ++i) {
        const double *x = s->x + 4 * (size_t)i;
        const v3 x3 = mk(x[0], x[1], x[2]);
        const uint32_t i_x = (uint32_t)floor((x[0] - c->origo[0]) / (c->L[0] / c->num[0]));
        const uint32_t i_y = (uint32_t)floor((x[1] - c->origo[1]) / (c->L[1] / c->num[1]));
        const uint32_t i_z = (uint32_t)floor((x[2] - c->origo[2]) / (c->L[2] / c->num[2]));
        if (!(x[0] >= c->origo[0] && x[1] >= c->origo[1] && x[2] >= c->origo[2]) || i_x >= nx ||
            i_y >= ny || i_z >= nz) {
            /* outside the grid (the reference reads past its arrays): no
             * pressure force */
            FLAG(s, SPH_ERR_OUT_OF_GRID);
            memset(D->f_p + 4 * (size_t)i, 0, 32);
            continue;
        }
        const double dx = c->L[0] / nx, dy = c->L[1] / ny, dz = c->L[2] / nz;
        const v3 X = mk(i_x * dx + 0.5 * dx, i_y * dy + 0.5 * dy, i_z * dz + 0.5 * dz);
        v3 grad_p = mk(0., 0., 0.);
        for (int d_iz = -1; d_iz < 2; d_iz++)
            for (int d_iy = -1; d_iy < 2; d_iy++)
                for (int d_ix = -1; d_ix < 2; d_ix++) {
                    const int ix_n = (int)(i_x + (uint32_t)d_ix);
                    const int iy_n = (int)(i_y + (uint32_t)d_iy);
                    const int iz_n = (int)(i_z + (uint32_t)d_iz);
                    v3 gpi = ld3(D->grad_p + 3 * (size_t)d_idx(dc, ix_n, iy_n, iz_n));
                    if ((ix_n == -1 && iy_n == -1) || (ix_n == -1 && iz_n == -1) ||
                        (iy_n == -1 && iz_n == -1) || (ix_n == (int)nx && iy_n == (int)ny) ||
                        (ix_n == (int)nx && iz_n == (int)nz) ||
                        (iy_n == (int)ny && iz_n == (int)nz) ||
                        (ix_n == (int)nx && iy_n == -1) || (ix_n == (int)nx && iz_n == -1) ||
                        (iy_n == (int)ny && ix_n == -1) || (iy_n == (int)ny && iz_n == -1) ||
                        (iz_n == (int)nz && ix_n == -1) || (iz_n == (int)nz && iy_n == -1))
                        gpi = mk(0., 0., 0.);
                    if (P->bc_top == 0 && i_z + (uint32_t)d_iz >= D->wall0_iz - 1u) gpi.z = 0.0;
                    const v3 n = mk(dx * d_ix, dy * d_iy, dz * d_iz);
                    const double w = weight_dist(vsub(x3, vadd(X, n)), dx, dy, dz);
                    grad_p = vadd(grad_p, smul(w, gpi));
                }
        const double v = sphere_volume(x[3]);
        const SphParams *Pm = c->P;
        v3 f_p = vsub(muls(smul(-1.0, grad_p), v),
                      smul(P->rho_f * v, mk(Pm->g[0], Pm->g[1], Pm->g[2])));
        if (P->bc_top == 0 && i_z >= D->wall0_iz) f_p.z = 0.0;
        double *F = s->force + 4 * (size_t)i;
        F[0] += f_p.x;
        F[1] += f_p.y;
        F[2] += f_p.z;
        F[3] += 0.0;
        double *o = D->f_p + 4 * (size_t)i;
        o[0] = f_p.x;
        o[1] = f_p.y;
        o[2] = f_p.z;
        o[3] = 0.0;
    }
}

/* darcy.cuh:392-730 findDarcyPorositiesLinear: per cell, the solid volume
 * of the spheres in the 27 cells around it weighted by the trilinear hat
 * centred on the cell, now and after an Euler step of the positions; the
 * sphere-weighted mean sphere velocity.  Spheres in sorted order. */
static void darcy_porosities(const Ctx *c, const Dc *dc, OrState *s, uint64_t iteration)
{
    OrDarcy *D = dc->d;
    const double c_phi = dc->P->c_phi;
    const int nx = dc->nx, ny = dc->ny, nz = dc->nz;
    const double dx = dc->dx, dy = dc->dy, dz = dc->dz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const uint32_t cellidx = d_idx(dc, x, y, z);
                if (c->np == 0) {
                    D->phi[cellidx] = 0.9;
                    D->dphi[cellidx] = 0.0;
                    continue;
                }
                double solid_volume = 0.0, solid_volume_new = 0.0;
                const v3 X = mk(x * dx + 0.5 * dx, y * dy + 0.5 * dy, z * dz + 0.5 * dz);
                v3 vp_avg_num = mk(0.0, 0.0, 0.0);
                double vp_avg_denum = 0.0;
                const double phi_0 = D->phi[cellidx];
                for (int z_dim = -1; z_dim < 2; ++z_dim)
                    for (int y_dim = -1; y_dim < 2; ++y_dim)
                        for (int x_dim = -1; x_dim < 2; ++x_dim) {
                            int t[3] = {x + x_dim, y + y_dim, z + z_dim};
                            if (t[2] == -1) t[2] = 1;
                            if (c->periodic == 2) {
                                if (t[1] == -1) t[1] = 1;
                                if (t[1] == (int)c->num[1]) t[1] = (int)c->num[1] - 2;
                            }
                            v3 distmod = mk(0.0, 0.0, 0.0);
                            if (find_dist_mod(c, t, &distmod) == -1) continue;
                            const uint32_t cellID = (uint32_t)t[0] + (uint32_t)t[1] * c->num[0] +
                                                    (c->num[0] * c->num[1]) * (uint32_t)t[2];
                            const uint32_t start = s->cell_start[cellID];
                            if (start == 0xffffffffu) continue;
                            const uint32_t end = s->cell_end[cellID];
                            for (uint32_t i = start; i < end; ++i) {
                                double xr[4], vv[4];
                                memcpy(xr, s->x_sorted + 4 * (size_t)i, 32);
                                memcpy(vv, s->vel_sorted + 4 * (size_t)i, 32);
                                v3 dist = mk(X.x - xr[0], X.y - xr[1], X.z - xr[2]);
                                dist = vadd(dist, distmod);
                                const double sw = weight_dist(dist, dx, dy, dz);
                                const double vol_p = sphere_volume(xr[3]);
                                solid_volume += sw * vol_p;
                                vp_avg_num = vadd(vp_avg_num, smul(sw * vol_p, mk(vv[0], vv[1], vv[2])));
                                vp_avg_denum += sw * vol_p;
                                for (int q = 0; q < 4; ++q) xr[q] += vv[q] * c->dt;
                                dist = vadd(mk(X.x - xr[0], X.y - xr[1], X.z - xr[2]), distmod);
                                solid_volume_new += weight_dist(dist, dx, dy, dz) * vol_p;
                            }
                        }
                double cell_volume = dx * dy * dz;
                if (z == nz - 1) cell_volume *= 0.875;
                const double phi = fmin(0.9, fmax(0.1, 1.0 - solid_volume / cell_volume));
                const double phi_new = fmin(0.9, fmax(0.1, 1.0 - solid_volume_new / cell_volume));
                double dphi;
                v3 vp_avg;
                if (iteration == 0) {
                    dphi = 0.0;
                    vp_avg = mk(0.0, 0.0, 0.0);
                } else {
                    dphi = 0.5 * (phi_new - phi_0);
                    vp_avg = divs(vp_avg_num, fmax(1.0e-16, vp_avg_denum));
                }
                D->phi[cellidx] = phi * c_phi;
                D->dphi[cellidx] = dphi * c_phi;
                D->vp_avg[3 * (size_t)cellidx] = vp_avg.x;
                D->vp_avg[3 * (size_t)cellidx + 1] = vp_avg.y;
                D->vp_avg[3 * (size_t)cellidx + 2] = vp_avg.z;
            }
}

/* darcy.cuh:733-807 copyDarcyPorositiesToEdges / ToBottom (periodic == 2):
 * phi, dphi, div_v_p and vp_avg of the y edge layers from the layer inside
 * them, then of the bottom layer from the layer above it */
static void darcy_copy_cell(const Dc *dc, uint32_t w, uint32_t r)
{
    OrDarcy *D = dc->d;
    D->phi[w] = D->phi[r];
    D->dphi[w] = D->dphi[r];
    D->div_v_p[w] = D->div_v_p[r];
    memcpy(D->vp_avg + 3 * (size_t)w, D->vp_avg + 3 * (size_t)r, 24);
}

static void darcy_copy_edges(const Dc *dc)
{
    for (int z = 0; z < dc->nz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x) {
                if (!(y == 0 || y == dc->ny - 1)) continue;
                int y_read = 0;
                if (y == 0) y_read = 1;
                if (y == dc->ny - 1) y_read = dc->ny - 2;
                darcy_copy_cell(dc, d_idx(dc, x, y, z), d_idx(dc, x, y_read, z));
            }
}

static void darcy_copy_bottom(const Dc *dc)
{
    for (int y = 0; y < dc->ny; ++y)
        for (int x = 0; x < dc->nx; ++x) darcy_copy_cell(dc, d_idx(dc, x, y, 0), d_idx(dc, x, y, 1));
}

/* darcy.cuh:1414-1435 setDarcyTopPressure: the condition reads
 * (x < nx && y < ny && z == nz - 1) || z == wall0_iz, so at z == wall0_iz
 * every thread of the launch grid (8 x 8 x 8 blocks covering the cells,
 * src/device.cu:865-869) writes, also those past nx or ny (their index
 * lands in other cells of the padded array); then :1438-1459
 * setDarcyTopWallPressure at z == wall0_iz */
static void darcy_top_pressure(const Dc *dc, double new_pressure)
{
    OrDarcy *D = dc->d;
    const int gx = (dc->nx + 7) / 8 * 8, gy = (dc->ny + 7) / 8 * 8, gz = (dc->nz + 7) / 8 * 8;
    const uint64_t ncell = (uint64_t)(dc->nx + 2) * (dc->ny + 2) * (dc->nz + 2);
    for (int z = 0; z < gz; ++z)
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) {
                if ((x < dc->nx && y < dc->ny && z == dc->nz - 1) || (uint32_t)z == D->wall0_iz) {
                    const uint32_t k = d_idx(dc, x, y, z);
                    if (k < ncell) D->p[k] = new_pressure;
                }
            }
    for (int z = 0; z < gz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x)
                if ((uint32_t)z == D->wall0_iz) D->p[d_idx(dc, x, y, z)] = new_pressure;
}

/* darcy.cuh:1462-1482 setDarcyTopWallFixedFlow: p at z = wall0_iz + 1 from
 * z = wall0_iz - 1 */
static void darcy_top_fixed_flow(const Dc *dc)
{
    OrDarcy *D = dc->d;
    const int gz = (dc->nz + 7) / 8 * 8;
    const uint64_t ncell = (uint64_t)(dc->nx + 2) * (dc->ny + 2) * (dc->nz + 2);
    for (int z = 0; z < gz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x)
                if ((uint32_t)z == D->wall0_iz + 1u) {
                    /* cells past the padded array (a wall at or above the
                     * top of the grid) are skipped */
                    const uint32_t w = d_idx(dc, x, y, z), r = d_idx(dc, x, y, z - 2);
                    if (w < ncell && r < ncell) D->p[w] = D->p[r];
                }
}

/* darcy.cuh:1485-1532 findDarcyPermeabilities (Kozeny-Carman, capped) */
static void darcy_permeabilities(const Dc *dc)
{
    OrDarcy *D = dc->d;
    for (int z = 0; z < dc->nz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x) {
                const uint32_t ci = d_idx(dc, x, y, z);
                double phi = D->phi[ci];
                if (phi > 0.9999) phi = 0.9999;
                double k = dc->P->k_c * pow(phi, 3) / pow(1.0 - phi, 2);
                k = fmin(2.7e-10, k);
                D->k[ci] = k;
            }
}

/* darcy.cuh:1644-1923 firstDarcySolution (explicit) and :1926-2226
 * updateDarcySolution (the Jacobi update): the pressure change of the
 * diffusion term (harmonic means of k across faces) and of the porosity
 * forcing, zero at Dirichlet boundaries (the +y test compares y with
 * nx - 1, as written) and in cells of constant pressure */
static double darcy_dp(const Dc *dc, const Ctx *c, int x, int y, int z, const double *pf)
{
    const OrDarcy *D = dc->d;
    const SphDarcy *P = dc->P;
    const int nx = dc->nx, ny = dc->ny, nz = dc->nz;
    const double dx = dc->dx, dy = dc->dy, dz = dc->dz;
    const uint32_t ci = d_idx(dc, x, y, z);
    const double phi_xn = D->phi[d_idx(dc, x - 1, y, z)], phi = D->phi[ci];
    const double phi_xp = D->phi[d_idx(dc, x + 1, y, z)];
    const double phi_yn = D->phi[d_idx(dc, x, y - 1, z)], phi_yp = D->phi[d_idx(dc, x, y + 1, z)];
    const double phi_zn = D->phi[d_idx(dc, x, y, z - 1)], phi_zp = D->phi[d_idx(dc, x, y, z + 1)];
    const double dphi = D->dphi[ci];
    const v3 vp_avg = ld3(D->vp_avg + 3 * (size_t)ci);
    const int p_constant = D->p_constant[ci];
    double p_xn = pf[d_idx(dc, x - 1, y, z)];
    const double p = pf[ci];
    double p_xp = pf[d_idx(dc, x + 1, y, z)];
    double p_yn = pf[d_idx(dc, x, y - 1, z)], p_yp = pf[d_idx(dc, x, y + 1, z)];
    double p_zn = pf[d_idx(dc, x, y, z - 1)], p_zp = pf[d_idx(dc, x, y, z + 1)];
    const double k_xn = D->k[d_idx(dc, x - 1, y, z)], k = D->k[ci];
    const double k_xp = D->k[d_idx(dc, x + 1, y, z)];
    const double k_yn = D->k[d_idx(dc, x, y - 1, z)], k_yp = D->k[d_idx(dc, x, y + 1, z)];
    const double k_zn = D->k[d_idx(dc, x, y, z - 1)], k_zp = D->k[d_idx(dc, x, y, z + 1)];
    if (x == 0 && P->bc_xn == 1) p_xn = p;
    if (x == nx - 1 && P->bc_xp == 1) p_xp = p;
    if (y == 0 && P->bc_yn == 1) p_yn = p;
    if (y == ny - 1 && P->bc_yp == 1) p_yp = p;
    if (z == 0 && P->bc_bot == 1) p_zn = p;
    if (z == nz - 1 && P->bc_top == 1) p_zp = p;
    const v3 grad_phi = mk((phi_xp - phi_xn) / (dx + dx), (phi_yp - phi_yn) / (dy + dy),
                           (phi_zp - phi_zn) / (dz + dz));
    const double div_k_grad_p =
        (2. * k_xp * k / (k_xp + k) * (p_xp - p) / dx - 2. * k_xn * k / (k_xn + k) * (p - p_xn) / dx) / dx +
        (2. * k_yp * k / (k_yp + k) * (p_yp - p) / dy - 2. * k_yn * k / (k_yn + k) * (p - p_yn) / dy) / dy +
        (2. * k_zp * k / (k_zp + k) * (p_zp - p) / dz - 2. * k_zn * k / (k_zn + k) * (p - p_zn) / dz) / dz;
    const double ndt = P->ndem * c->dt;
    double dp = ndt / (P->beta_f * phi * P->mu) * div_k_grad_p -
                (ndt / (P->beta_f * phi * (1.0 - phi))) * (dphi / ndt + dot(vp_avg, grad_phi));
    if ((P->bc_bot == 0 && z == 0) || (P->bc_top == 0 && z == nz - 1) ||
        ((uint32_t)z >= D->wall0_iz && P->bc_top == 0) || (P->bc_xn == 0 && x == 0) ||
        (P->bc_xp == 0 && x == nx - 1) || (P->bc_yn == 0 && y == 0) ||
        (P->bc_yp == 0 && y == nx - 1) || p_constant == 1)
        dp = 0.0;
    return dp;
}

/* darcy.cuh:2267-2325 findDarcyVelocities */
static void darcy_velocities(const Dc *dc)
{
    OrDarcy *D = dc->d;
    const double mu = dc->P->mu;
    for (int z = 0; z < dc->nz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x) {
                const uint32_t ci = d_idx(dc, x, y, z);
                const double xn = D->p[d_idx(dc, x - 1, y, z)], xp = D->p[d_idx(dc, x + 1, y, z)];
                const double yn = D->p[d_idx(dc, x, y - 1, z)], yp = D->p[d_idx(dc, x, y + 1, z)];
                const double zn = D->p[d_idx(dc, x, y, z - 1)], zp = D->p[d_idx(dc, x, y, z + 1)];
                const double k = D->k[ci], phi = D->phi[ci];
                const v3 grad_p = mk((xp - xn) / (dc->dx + dc->dx), (yp - yn) / (dc->dy + dc->dy),
                                     (zp - zn) / (dc->dz + dc->dz));
                const v3 v = divs(smul(-k / mu, grad_p), phi);
                D->v[3 * (size_t)ci] = v.x;
                D->v[3 * (size_t)ci + 1] = v.y;
                D->v[3 * (size_t)ci + 2] = v.z;
            }
}

static void darcy_interior_copy(const Dc *dc, const double *src, double *dst)
{
    for (int z = 0; z < dc->nz; ++z)
        for (int y = 0; y < dc->ny; ++y)
            for (int x = 0; x < dc->nx; ++x) dst[d_idx(dc, x, y, z)] = src[d_idx(dc, x, y, z)];
}

static void dc_init(Dc *dc, const Ctx *c, OrDarcy *D)
{
    dc->d = D;
    dc->P = &D->prm;
    dc->nx = (int)c->num[0];
    dc->ny = (int)c->num[1];
    dc->nz = (int)c->num[2];
    dc->dx = c->L[0] / c->num[0];
    dc->dy = c->L[1] / c->num[1];
    dc->dz = c->L[2] / c->num[2];
}

void or_darcy_start(OrState *s)
{
    OrDarcy *D = s->darcy;
    if (!D) return;
    Ctx c;
    ctx_init(&c, s);
    Dc dc;
    dc_init(&dc, &c, D);
    /* device.cu:1009-1015 */
    D->p_top_orig = D->p[d_idx(&dc, 0, 0, dc.nz - 1)] -
                    D->prm.p_mod_A * sin(2.0 * OR_DARCY_PI * D->prm.p_mod_f * s->box.t_current +
                                         D->prm.p_mod_phi);
    D->filetimeclock = 0.0;
    D->wall_w_host = s->box.walls.nw > 0 ? s->box.walls.nx[0][3] : 0.0;
    D->wall0_iz = 10000000u;
    D->log_n = 0;
}

static void darcy_log(OrDarcy *D, uint64_t step, uint32_t iters, uint32_t ok)
{
    if (D->log_n < D->log_cap) {
        D->log_step[D->log_n] = step;
        D->log_iters[D->log_n] = iters;
        D->log_ok[D->log_n] = ok;
        D->log_n++;
    }
}

/* device.cu:1891-2419: the Darcy part of one step, after interact and
 * bonds, before the shear-stress sums and integrate.  The Jacobi loop's
 * residual check (every nijacnorm = 10 iterations, src/debug.h:16) takes
 * the largest |norm| over the cells (darcy.cpp:266-293); a NaN raises
 * SPH_ERR_NAN and ends the solve (the reference exits). */
static void darcy_step(const Ctx *c, OrState *s)
{
    OrDarcy *D = s->darcy;
    const SphDarcy *P = &D->prm;
    Dc dc;
    dc_init(&dc, c, D);
    const uint64_t iter = s->iter;
    /* device.cu:1901-1904 wall0_iz from the host's copy of wall 0 */
    if (c->nw > 0 && (s->box.walls.wmode[0] == 1 || s->box.walls.wmode[0] == 3))
        D->wall0_iz = (uint32_t)(D->wall_w_host / (c->L[2] / c->num[2]));
    if (c->np > 0) {
        darcy_ghost(&dc, D->p, 1);
        darcy_gradient(&dc, D->p, D->grad_p);
        darcy_ghost(&dc, D->grad_p, 3);
        darcy_force(c, &dc, s);
    }
    if (iter % P->ndem != 0) return;
    darcy_porosities(c, &dc, s, iter);
    if (c->periodic == 2) {
        darcy_copy_edges(&dc);
        darcy_copy_bottom(&dc);
    }
    if ((P->p_mod_A > 1.0e-5 || P->p_mod_A < -1.0e-5) && P->p_mod_f > 1.0e-7) {
        const double new_pressure =
            D->p_top_orig + P->p_mod_A * sin(2.0 * OR_DARCY_PI * P->p_mod_f * s->box.t_current +
                                              P->p_mod_phi);
        darcy_top_pressure(&dc, new_pressure);
    }
    darcy_permeabilities(&dc);
    darcy_ghost(&dc, D->phi, 1);
    darcy_ghost(&dc, D->k, 1);
    darcy_gradient(&dc, D->k, D->grad_k);
    if (iter == 0) {
        for (int z = 0; z < dc.nz; ++z)
            for (int y = 0; y < dc.ny; ++y)
                for (int x = 0; x < dc.nx; ++x) D->norm[d_idx(&dc, x, y, z)] = 0.0;
        darcy_interior_copy(&dc, D->p, D->p_old);
    }
    darcy_ghost_flux(&dc, D->p, D->k, c->L[2]);
    uint32_t nijac = 0, ok = 0;
    for (nijac = 0; nijac < P->maxiter; ++nijac) {
        if (nijac == 0) darcy_interior_copy(&dc, D->p, D->p_old);
        darcy_ghost(&dc, D->p, 1);
        if (nijac == 0)
            for (int z = 0; z < dc.nz; ++z)
                for (int y = 0; y < dc.ny; ++y)
                    for (int x = 0; x < dc.nx; ++x)
                        D->dp_expl[d_idx(&dc, x, y, z)] = darcy_dp(&dc, c, x, y, z, D->p);
        for (int z = 0; z < dc.nz; ++z)
            for (int y = 0; y < dc.ny; ++y)
                for (int x = 0; x < dc.nx; ++x) {
                    const uint32_t ci = d_idx(&dc, x, y, z);
                    const double dp_impl = darcy_dp(&dc, c, x, y, z, D->p);
                    const double epsilon = 0.5;
                    const double p = D->p[ci];
                    double p_new = D->p_old[ci] + (1.0 - epsilon) * D->dp_expl[ci] + epsilon * dp_impl;
                    const double theta = 0.05;
                    p_new = p * (1.0 - theta) + p_new * theta;
                    D->p_new[ci] = p_new;
                    D->norm[ci] = (p_new - p) / (p + 1.0e-16);
                }
        if (P->bc_top == 1) darcy_top_fixed_flow(&dc);
        darcy_ghost_flux(&dc, D->p, D->k, c->L[2]);
        darcy_interior_copy(&dc, D->p_new, D->p);
        if (nijac % 10 == 0) {
            double max_norm_res = -1.0e9;
            int nan = 0;
            for (int z = 0; z < dc.nz && !nan; ++z)
                for (int y = 0; y < dc.ny && !nan; ++y)
                    for (int x = 0; x < dc.nx; ++x) {
                        const double r = fabs(D->norm[d_idx(&dc, x, y, z)]);
                        if (r != r) { nan = 1; break; }
                        if (r > max_norm_res) max_norm_res = r;
                    }
            if (nan) {
                FLAG(s, SPH_ERR_NAN);
                break;
            }
            if (max_norm_res <= P->tolerance) {
                ok = 1;
                break;
            }
        }
        if (nijac == P->maxiter - 1) break;
    }
    darcy_log(D, iter + 1, nijac, ok);
    if (D->filetimeclock + c->dt < P->file_dt)
        for (int z = 0; z < dc.nz; ++z)
            for (int y = 0; y < dc.ny; ++y)
                for (int x = 0; x < dc.nx; ++x) D->dphi[d_idx(&dc, x, y, z)] = 0.0;
    darcy_ghost(&dc, D->p, 1);
    darcy_velocities(&dc);
}

/* device.cu:2537 and 2569-2672: the host's file clock, and the host copy of
 * the walls refreshed by the output's transfer from the device */
static void darcy_clock(const Ctx *c, OrState *s)
{
    OrDarcy *D = s->darcy;
    D->filetimeclock += c->dt;
    if (D->filetimeclock >= D->prm.file_dt) {
        D->filetimeclock = 0.0;
        if (c->nw > 0) D->wall_w_host = s->box.walls.nx[0][3];
    }
}

/* --------------------------------------------------------------- step loop */

static void ctx_init(Ctx *c, OrState *s)
{
    c->s = s;
    c->P = &s->box.params;
    for (int d = 0; d < 3; ++d) {
        c->origo[d] = s->box.grid.origo[d];
        c->L[d] = s->box.grid.L[d];
        c->num[d] = s->box.grid.num[d];
    }
    c->periodic = s->box.grid.periodic;
    c->np = s->box.np;
    c->nw = s->box.walls.nw;
    c->dt = s->box.dt;
    c->lenmode = s->length_mode;
}

/* device.cu:241-276 checkParticlePositions, as error flags */
static void check_positions(const Ctx *c, OrState *s)
{
    for (unsigned i = 0; i < c->np; ++i) {
        const double *x = s->x + 4 * (size_t)i;
        if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2])) FLAG(s, SPH_ERR_NAN);
        else if (x[0] < c->origo[0] || x[1] < c->origo[1] || x[2] < c->origo[2] ||
                 x[0] > c->L[0] || x[1] > c->L[1] || x[2] > c->L[2])
            FLAG(s, SPH_ERR_OUT_OF_GRID);
    }
}

int or_step(OrState *s, uint64_t nsteps)
{
#ifdef _OPENMP
    if (s->nthreads > 0) omp_set_num_threads(s->nthreads);
#endif
    const unsigned np = s->box.np;
    for (uint64_t step = 0; step < nsteps; ++step) {
        /* device.cu:1050-1052 adaptive grid */
        if (s->box.grid.adaptive == 1 && s->box.walls.nw > 0) s->box.grid.L[2] = s->box.walls.nx[0][3];
        Ctx c;
        ctx_init(&c, s);
        const uint64_t ncells = (uint64_t)c.num[0] * c.num[1] * c.num[2];
        if (np > 0) {
            check_positions(&c, s);
            /* sorting.cuh:25-51 + stable sort by key (device.cu:1075) as a
             * counting sort, which is stable */
            uint32_t *count = (uint32_t *)calloc(ncells + 1, sizeof(uint32_t));
            for (unsigned i = 0; i < np; ++i) {
                s->cell_id[i] = calc_cell_id(&c, s, s->x + 4 * (size_t)i);
                count[s->cell_id[i] + 1]++;
            }
            for (uint64_t k = 0; k < ncells; ++k) count[k + 1] += count[k];
            for (unsigned i = 0; i < np; ++i) s->perm[count[s->cell_id[i]]++] = i;
            free(count);
            /* device.cu:1089 and sorting.cuh:56-132 reorderArrays */
            memset(s->cell_start, 0xff, ncells * sizeof(uint32_t));
            for (unsigned i = 0; i < np; ++i) {
                uint32_t cell = s->cell_id[s->perm[i]];
                uint32_t prev = i > 0 ? s->cell_id[s->perm[i - 1]] : 0;
                if (i == 0 || cell != prev) {
                    s->cell_start[cell] = i;
                    if (i > 0) s->cell_end[prev] = i;
                }
                if (i == np - 1) s->cell_end[cell] = i + 1;
                memcpy(s->x_sorted + 4 * (size_t)i, s->x + 4 * (size_t)s->perm[i], 32);
                memcpy(s->vel_sorted + 4 * (size_t)i, s->vel + 4 * (size_t)s->perm[i], 32);
                memcpy(s->angvel_sorted + 4 * (size_t)i, s->angvel + 4 * (size_t)s->perm[i], 32);
            }
            /* cell ids were sorted keys in the reference: keep the sorted copy */
            if (s->box.params.contactmodel == 2 || s->box.params.contactmodel == 3)
                topology(&c, s);
            interact(&c, s);
            if (s->box.nb0 > 0) bonds_linear(&c, s, s->bonds_broken);
        }
        if (s->darcy) darcy_step(&c, s);
        if (np > 0) {
            if (c.nw > 0 && s->box.walls.wmode[0] == 3) {
                find_shear_stress(&c, s);
                summation(np, s->tau_eff_x_pp, s->tau_eff_x_partial);
            }
            /* device.cu:2455-2462 stepwise velocity change */
            int change = 0;
            double tc = s->box.t_current;
            if (tc >= 10.0 && tc < 15.0 && s->velocity_state == 1) { change = 1; s->velocity_state = 2; }
            else if (tc >= 15.0 && s->velocity_state == 2) { change = -1; s->velocity_state = 1; }
            integrate(&c, s, change);
            if (c.nw > 0) summation(np, s->walls_force_pp, s->walls_force_partial);
            if (c.nw > 0) integrate_walls(&c, s, s->box.t_current);
        }
        s->box.t_current += s->box.dt;
        if (s->darcy) darcy_clock(&c, s);
        s->iter++;
    }
    return s->error_flags;
}

/* ----------------------------------------------------------- analysis */

/* M_PI of the C library, which src/sphere.cpp uses (not the 3.14159265358979
 * of the step kernels) */
static const double OR_M_PI = 3.14159265358979323846;

/* src/sphere.cpp:468-471 sphericalCap */
static double or_cap(double h, double r) { return OR_M_PI * h * h / 3.0 * (3.0 * r - h); }

/* src/sphere.cpp:487-606 DEM::porosity: per slab, the slab volume less
 * every sphere's volume inside it, with the reference's cap terms (a sphere
 * cut by a slab face subtracts the sphere volume plus the cap, as the
 * reference writes it), spheres in index order. */
int or_porosity(const double *x, uint32_t np, double top, double origo_z, double L0, double L1,
                uint32_t z_slices, double *z_pos, double *porosity)
{
    double r_max = 0.0;
    for (uint32_t i = 0; i < np; ++i)
        if (x[4 * (size_t)i + 3] > r_max) r_max = x[4 * (size_t)i + 3];
    const double h_slice = (top - origo_z) / (double)z_slices;
    if (h_slice <= r_max * 2.0) return -1;
    const double V_slice = h_slice * L0 * L1;
    for (uint32_t iz = 0; iz < z_slices; ++iz) {
        double V_void = V_slice;
        const double z_low = iz * h_slice;
        const double z_high = z_low + h_slice;
        for (uint32_t i = 0; i < np; ++i) {
            const double zc = x[4 * (size_t)i + 2], r = x[4 * (size_t)i + 3];
            const double zl = zc - r, zh = zc + r;
            const double V_s = 4.0 / 3.0 * OR_M_PI * r * r * r;
            if (z_low <= zl && zh <= z_high) {
                V_void -= V_s;
            } else {
                if (z_low >= zc && z_low <= zh) V_void -= or_cap(zh - z_low, r);
                else if (z_low < zc && z_low > zl) V_void -= V_s + or_cap(z_low - zl, r);
                if (z_high <= zc && z_high >= zl) V_void -= or_cap(z_high - zl, r);
                else if (z_high > zc && z_high < zh) V_void -= V_s + or_cap(zh - z_high, r);
            }
        }
        z_pos[iz] = z_low + 0.5 * h_slice;
        porosity[iz] = V_void / V_slice;
    }
    return 0;
}

/* src/sphere.cpp:677-725 DEM::findOverlaps: all pairs i < j (no periodic
 * images) with |x_j - x_i| - (r_i + r_j) < 0 and both fixvel == 0. */
uint64_t or_overlaps(const double *x, const double *vel, uint32_t np, uint64_t max_pairs,
                     uint32_t *pairs, double *delta_n)
{
    uint64_t n = 0;
    for (uint32_t i = 0; i < np; ++i)
        for (uint32_t j = i + 1; j < np; ++j) {
            const double *xi = x + 4 * (size_t)i, *xj = x + 4 * (size_t)j;
            const double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
            const double len = sqrt(dx * dx + dy * dy + dz * dz);
            const double d = len - (xi[3] + xj[3]);
            if (d < 0.0 && vel[4 * (size_t)i + 3] == 0.0 && vel[4 * (size_t)j + 3] == 0.0) {
                if (n < max_pairs) {
                    if (pairs) {
                        pairs[2 * n] = i;
                        pairs[2 * n + 1] = j;
                    }
                    if (delta_n) delta_n[n] = d;
                }
                ++n;
            }
        }
    return n;
}

/* ---- ray tracer (src/raytracer.cuh), FP32 as the reference computes it.
 * One ray per pixel, every sphere in index order, the first strictly
 * smallest |t| kept; normalisation by 1 / sqrtf, IEEE division and square
 * root, no contraction (the build's -ffp-contract=off). */
typedef struct {
    float x, y, z;
} of3;

static of3 o3(float x, float y, float z)
{
    of3 r = {x, y, z};
    return r;
}
static of3 o_add(of3 a, of3 b) { return o3(a.x + b.x, a.y + b.y, a.z + b.z); }
static of3 o_sub(of3 a, of3 b) { return o3(a.x - b.x, a.y - b.y, a.z - b.z); }
static of3 o_mul(float s, of3 a) { return o3(s * a.x, s * a.y, s * a.z); }
static of3 o_div(of3 a, float s) { return o3(a.x / s, a.y / s, a.z / s); }
static of3 o_neg(of3 a) { return o3(-a.x, -a.y, -a.z); }
static float o_dot(of3 a, of3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static of3 o_cross(of3 a, of3 b)
{
    return o3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static float o_len(of3 a) { return sqrtf(o_dot(a, a)); }
static of3 o_unit(of3 a) { return o_mul(1.0f / sqrtf(o_dot(a, a)), a); }

/* src/colorbar.h:7-20 */
static float o_red(float r) { return fminf(1.0f, 0.209f * r * r * r - 2.49f * r * r + 3.0f * r + 0.0109f); }
static float o_green(float r) { return fminf(1.0f, -2.44f * r * r + 2.15f * r + 0.369f); }
static float o_blue(float r) { return fminf(1.0f, -2.21f * r * r + 1.61f * r + 0.573f); }

/* |(v.x, v.y, v.z)| in double, as render() fills its linear array */
static double o_mag(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

void or_render(const double *x, const double *vel, const double *angvel, const double *angpos,
               const double *xyzsum, const double *p, uint32_t np, const double *L, int method,
               float maxval, float lower_cutoff, uint32_t width, uint32_t height, uint8_t *rgb)
{
    /* src/sphere.cpp:641-670 maxPos: componentwise max of the positions and 0 */
    double mx[3] = {0.0, 0.0, 0.0};
    for (uint32_t i = 0; i < np; ++i)
        for (int a = 0; a < 3; ++a)
            if (mx[a] < x[4 * (size_t)i + a]) mx[a] = x[4 * (size_t)i + a];
    /* src/raytracer.cuh:379-400 render, :291-333 cameraInit */
    const float imgw = (float)(L[0] * 1.35f);
    const of3 lookat = o_div(o3((float)mx[0], (float)mx[1], (float)mx[2]), 2.0f);
    const of3 eye = o3((float)(L[0] * 2.3f), (float)(L[1] * -5.0f), (float)(L[2] * 1.3f));
    const float hw_ratio = (float)(height / width);
    const float pl = -0.5f * imgw, pr = 0.5f * imgw;
    const float pb = -0.5f * imgw * hw_ratio, pt = 0.5f * imgw * hw_ratio;
    const of3 view = o_sub(eye, lookat);
    const of3 up = o3(0.0f, 0.0f, 1.0f);
    const of3 w = o_div(o_neg(view), o_len(view));
    const of3 u = o_div(o_cross(up, w), o_len(o_cross(up, w)));
    const of3 v = o_cross(w, u);
    const float dfoc = o_len(view) * 0.8f;
    const of3 le = o_mul(-1.0f, eye);
    const of3 light = o_unit(o3(le.x * 1.0f, le.y * 0.2f, le.z * 0.6f));
    const int64_t pixels = (int64_t)width * height;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t m = 0; m < pixels; ++m) {
        const unsigned int mempos = (unsigned int)m;
        /* :29-56 rayInitPerspective */
        const unsigned int i = mempos % width;
        const unsigned int j = (unsigned int)(int)floorf((float)mempos / width) % width;
        const float p_u = pl + (pr - pl) * (i + 0.5f) / width;
        const float p_v = pb + (pt - pb) * (j + 0.5f) / height;
        const of3 e = eye;
        const of3 d = o_add(o_add(o_mul(-dfoc, w), o_mul(p_u, u)), o_mul(p_v, v));
        /* :59-144 rayIntersectSpheres, :146-288 rayIntersectSpheresColormap */
        float tdist = 1e10f;
        of3 n = o3(0.0f, 0.0f, 0.0f);
        uint32_t hitidx = 0;
        for (uint32_t k = 0; k < np; ++k) {
            const double *xk = x + 4 * (size_t)k;
            const of3 c = o3((float)xk[0], (float)xk[1], (float)xk[2]);
            const float R = (float)xk[3];
            const float Delta = (2.0f * o_dot(d, o_sub(e, c))) * (2.0f * o_dot(d, o_sub(e, c))) -
                                4.0f * o_dot(d, d) * (o_dot(o_sub(e, c), o_sub(e, c)) - R * R);
            int take = Delta > 0.0f;
            if (method != 0 && lower_cutoff > 0.0) {
                double val;
                switch (method) {
                case 1: val = p[k]; break;
                case 2: val = o_mag(vel + 4 * (size_t)k); break;
                case 3: val = o_mag(angvel + 4 * (size_t)k); break;
                case 4: val = xyzsum[4 * (size_t)k]; break;
                default: val = o_mag(angpos + 4 * (size_t)k); break;
                }
                const float fval = (float)val;
                const float fixvel = (float)vel[4 * (size_t)k + 3];
                take = take && fval > lower_cutoff && fixvel == 0.f;
            }
            if (!take) continue;
            const float t_minus =
                (o_dot(o_neg(d), o_sub(e, c)) -
                 sqrtf(o_dot(d, o_sub(e, c)) * o_dot(d, o_sub(e, c)) -
                       o_dot(d, d) * (o_dot(o_sub(e, c), o_sub(e, c)) - R * R))) /
                o_dot(d, d);
            if (fabsf(t_minus) < tdist) {
                const of3 pt3 = o_add(e, o_mul(t_minus, d));
                tdist = fabsf(t_minus);
                n = o_unit(o_mul(2.0f, o_sub(pt3, c)));
                hitidx = k;
            }
        }
        uint8_t *px = rgb + 3 * (size_t)mempos;
        if (!(tdist < 1e10f)) {
            px[0] = px[1] = px[2] = 255; /* :14-27 imageInit */
            continue;
        }
        const float dotprod = fmaxf(0.0f, o_dot(n, light));
        const float I_d = 40.0f, k_d = 5.0f, k_a = 10.0f, I_a = 5.0f;
        if (method == 0) {
            px[0] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.48f);
            px[1] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.41f);
            px[2] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * 0.27f);
            continue;
        }
        double val;
        switch (method) {
        case 1: val = p[hitidx]; break;
        case 2: val = o_mag(vel + 4 * (size_t)hitidx); break;
        case 3: val = o_mag(angvel + 4 * (size_t)hitidx); break;
        case 4: val = xyzsum[4 * (size_t)hitidx]; break;
        default: val = o_mag(angpos + 4 * (size_t)hitidx); break;
        }
        const float fixvel = (float)vel[4 * (size_t)hitidx + 3];
        float ratio = (float)(val / maxval);
        if (ratio < 0.01f) ratio = 0.01f;
        if (ratio > 0.99f) ratio = 0.99f;
        float redv = o_red(ratio), greenv = o_green(ratio), bluev = o_blue(ratio);
        if (fixvel > 0.f) {
            redv = 0.5f;
            greenv = 0.5f;
            bluev = 0.5f;
        }
        px[0] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * redv);
        px[1] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * greenv);
        px[2] = (uint8_t)((k_d * I_d * dotprod + k_a * I_a) * bluev);
    }
}

/* ------------------------------------------------------------ packing sweep */

/* The project's scene-preparation sweep (sphere_b200 sph_relax: kernels
 * k_hash, k_place, k_relax, k_relax_apply; no counterpart in the reference,
 * whose packs come from running the DEM itself), restated for one box as the
 * checker of that kernel chain and as a CPU packer for bench.py's reference
 * arm.  Per sweep: spheres binned into the grid's cells (cell ids clamped
 * into the grid), ordered by cell and, within a cell, by index; for each
 * sphere in that order, every overlapping sphere of the 27 cells around it
 * (periodic images by the rule of calc_cell_id / find_dist_mod, visited in
 * (z, y, x) order, a cell's spheres in index order) adds alpha * overlap / 2
 * along the centre line; the floor, the ceiling z_top and the side walls of
 * non-periodic axes push back; then every sphere moves (Jacobi), periodic
 * axes wrap, and positions are clamped into [origo, L (1 - 1e-12)].
 * x4: [np][4] (x, y, z, r), updated.  *max_ov: the largest overlap seen in
 * the last sweep.  Arithmetic in the operand order of the CUDA kernels,
 * without contraction, so the result is the GPU's bit for bit. */
void or_relax(double *x4, uint32_t np, const double origo[3], const double L[3],
              const uint32_t num[3], int periodic, uint32_t sweeps, double alpha, double z_top,
              int nthreads, double *max_ov)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    const size_t ncells = (size_t)num[0] * num[1] * num[2];
    uint32_t *cell = (uint32_t *)malloc(sizeof(uint32_t) * (np ? np : 1));
    uint32_t *off = (uint32_t *)calloc(ncells + 1, sizeof(uint32_t));
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (np ? np : 1));
    double *xs = (double *)malloc(sizeof(double) * 4 * (np ? np : 1));
    double *disp = (double *)malloc(sizeof(double) * 3 * (np ? np : 1));
    double worst_all = 0.0;
    for (uint32_t sw = 0; sw < sweeps; ++sw) {
        memset(off, 0, sizeof(uint32_t) * (ncells + 1));
        for (uint32_t i = 0; i < np; ++i) {
            unsigned c[3];
            for (int d = 0; d < 3; ++d) {
                double f = floor((x4[4 * (size_t)i + d] - origo[d]) / (L[d] / num[d]));
                if (!(f >= 0.0)) f = 0.0;
                if (f >= (double)num[d]) f = (double)(num[d] - 1);
                c[d] = (unsigned)f;
            }
            cell[i] = (c[2] * num[1]) * num[0] + c[1] * num[0] + c[0];
            off[cell[i] + 1]++;
        }
        for (size_t k = 0; k < ncells; ++k) off[k + 1] += off[k];
        {
            uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * (ncells ? ncells : 1));
            memcpy(fill, off, sizeof(uint32_t) * ncells);
            for (uint32_t i = 0; i < np; ++i) {   /* ascending index within a cell */
                const uint32_t a = fill[cell[i]]++;
                perm[a] = i;
                memcpy(xs + 4 * (size_t)a, x4 + 4 * (size_t)i, 4 * sizeof(double));
            }
            free(fill);
        }
        double worst = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(max : worst)
        for (long long aa = 0; aa < (long long)np; ++aa) {
            const uint32_t a = (uint32_t)aa;
            const double *xa = xs + 4 * (size_t)a;
            int g[3];
            for (int d = 0; d < 3; ++d) g[d] = (int)floor((xa[d] - origo[d]) / (L[d] / num[d]));
            double dx = 0.0, dy = 0.0, dz = 0.0, w = 0.0;
            for (int oz = -1; oz < 2; ++oz)
                for (int oy = -1; oy < 2; ++oy)
                    for (int ox = -1; ox < 2; ++ox) {
                        int tx = g[0] + ox, ty = g[1] + oy;
                        const int tz = g[2] + oz;
                        int sx = 0, sy = 0;
                        const int nx = (int)num[0], ny = (int)num[1], nz = (int)num[2];
                        if (periodic == 1) {
                            if (tx < 0) { tx += nx; sx = 1; }
                            if (tx >= nx) { tx -= nx; sx = -1; }
                            if (ty < 0) { ty += ny; sy = 1; }
                            if (ty >= ny) { ty -= ny; sy = -1; }
                        } else if (periodic == 2) {
                            if (tx < 0) { tx += nx; sx = 1; }
                            if (tx >= nx) { tx -= nx; sx = -1; }
                            if (ty < 0 || ty >= ny) continue;
                        } else {
                            if (tx < 0 || tx >= nx || ty < 0 || ty >= ny) continue;
                        }
                        if (tz < 0 || tz >= nz) continue;
                        if (tx < 0 || tx >= nx || ty < 0 || ty >= ny) continue;
                        const double dmx = sx == 0 ? 0.0 : (sx > 0 ? L[0] : -L[0]);
                        const double dmy = sy == 0 ? 0.0 : (sy > 0 ? L[1] : -L[1]);
                        const double dmz = 0.0;
                        const uint32_t c = (uint32_t)(tx + ty * nx + (nx * ny) * tz);
                        for (uint32_t b = off[c]; b < off[c + 1]; ++b) {
                            if (b == a) continue;
                            const double *xb = xs + 4 * (size_t)b;
                            const double rx = xa[0] - xb[0] + dmx, ry = xa[1] - xb[1] + dmy,
                                         rz = xa[2] - xb[2] + dmz;
                            const double len = sqrt(rx * rx + ry * ry + rz * rz);
                            const double ov = xa[3] + xb[3] - len;
                            if (ov > 0.0 && len > 0.0) {
                                const double s = 0.5 * alpha * ov / len;
                                dx += s * rx;
                                dy += s * ry;
                                dz += s * rz;
                                w = fmax(w, ov);
                            }
                        }
                    }
            const double below = (origo[2] + xa[3]) - xa[2];
            if (below > 0.0) { dz += below; w = fmax(w, below); }
            const double above = xa[2] + xa[3] - z_top;
            if (above > 0.0) { dz -= above; w = fmax(w, above); }
            if (periodic == 0) {
                const double lo = (origo[0] + xa[3]) - xa[0], hi = xa[0] + xa[3] - L[0];
                if (lo > 0.0) { dx += lo; w = fmax(w, lo); }
                if (hi > 0.0) { dx -= hi; w = fmax(w, hi); }
            }
            if (periodic != 1) {
                const double lo = (origo[1] + xa[3]) - xa[1], hi = xa[1] + xa[3] - L[1];
                if (lo > 0.0) { dy += lo; w = fmax(w, lo); }
                if (hi > 0.0) { dy -= hi; w = fmax(w, hi); }
            }
            double *d = disp + 3 * (size_t)perm[a];
            d[0] = dx;
            d[1] = dy;
            d[2] = dz;
            if (w > worst) worst = w;
        }
#pragma omp parallel for schedule(static)
        for (long long ii = 0; ii < (long long)np; ++ii) {
            double *x = x4 + 4 * (size_t)ii;
            const double *d = disp + 3 * (size_t)ii;
            x[0] += d[0];
            x[1] += d[1];
            x[2] += d[2];
            if (periodic == 1 || periodic == 2) {
                if (x[0] < origo[0]) x[0] += L[0] - origo[0];
                if (x[0] >= L[0]) x[0] -= L[0] - origo[0];
            }
            if (periodic == 1) {
                if (x[1] < origo[1]) x[1] += L[1] - origo[1];
                if (x[1] >= L[1]) x[1] -= L[1] - origo[1];
            }
            x[0] = fmin(fmax(x[0], origo[0]), L[0] * (1.0 - 1e-12));
            x[1] = fmin(fmax(x[1], origo[1]), L[1] * (1.0 - 1e-12));
            x[2] = fmin(fmax(x[2], origo[2]), L[2] * (1.0 - 1e-12));
        }
        worst_all = worst;
    }
    if (max_ov) *max_ov = worst_all;
    free(cell);
    free(off);
    free(perm);
    free(xs);
    free(disp);
}
