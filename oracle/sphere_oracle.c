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
