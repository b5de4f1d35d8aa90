// sph_adjoint.cu -- reverse-mode (adjoint) step of the FP64 DEM step.
//
// Differentiates one step of interact + TY3 integrate (src/contactmodels.cuh
// :244-411 contactLinear, :10-117 contactLinear_wall, src/integration.cuh
// :14-305) with the contact set frozen: the slots the forward contact
// search produced at that step (recorded on the tape) define which pairs
// interact; each pair's law is differentiated on the branch it took
// (normal force active or not, no tangential force / stick / slip).
// Scope: contact model 2, E == 0, kappa == 0, no bonds, no dynamic walls,
// gamma_wt == 0, FP64 lengths (SPH_LEN_FP64), one box.
//
// State of step s: y_s = (x, v, w, A, O, H): positions, velocities, angular
// velocities, previous accelerations A (TY3's acc0), previous angular
// accelerations O, tangential histories H.  The step computes
// acc = F(y_s)/m + g, alpha = T(y_s)/I and
//   x' = x + v dt + (2/3) acc dt^2 - (1/6) A dt^2
//   v' = v + (3/2) acc dt - (1/2) A dt
//   w' = w + (3/2) alpha dt - (1/2) O dt,   A' = acc, O' = alpha.
// Given the adjoints of y_{s+1} the kernels below produce those of y_s and
// accumulate the gradients of k_n, gamma_n and mu (= mu_s = mu_d).
#include <cstdint>

#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

__device__ __forceinline__ d3 d3z() { return mk(0.0, 0.0, 0.0); }
__device__ __forceinline__ void acc3(d3 &a, d3 b) { a = vadd(a, b); }

// VJP of contactLinear for one directed contact (a, b).  Inputs of the
// forward: xa, xb (+ periodic shift dm), va, vb, wa, wb, the stored
// history h0; outputs F, T (contributions to a) and the new history.  Fb, Tb,
// db are the adjoints of the outputs; the input adjoints are accumulated.
__device__ void linear_contact_vjp(const SphParams &P, double dt, d3 xa, d3 xb, d3 dm, d3 va,
                                   d3 vb, d3 wa, d3 wb, double ra, double rb, d3 h0, d3 Fb, d3 Tb,
                                   d3 db, d3 &xab, d3 &xbb, d3 &vab, d3 &vbb, d3 &wab, d3 &wbb,
                                   d3 &h0b, double &knb, double &gnb, double &mub)
{
    // ---- forward (same branches as contact_linear)
    const d3 X = vadd(vsub(xa, xb), dm);
    const double L = sqrt(dot(X, X));
    const double delta = L - (ra + rb);
    const d3 n = divs(X, L);
    const d3 vl = vsub(va, vb);
    const d3 ca = cross(n, wa), cb = cross(n, wb);
    const double sa = ra + delta * 0.5, sb = rb + delta * 0.5;
    const d3 vel = vadd(vadd(vl, smul(sa, ca)), smul(sb, cb));
    const double vn = -dot(n, vl);
    const double s1 = dot(n, vel);
    const d3 vt = vsub(vel, smul(s1, n));
    const double s2 = dot(n, h0);
    const d3 d0 = vsub(h0, smul(s2, n));
    const double kn = P.k_n, kt = P.k_t;
    const double fnm = -kn * delta + P.gamma_n * vn;
    const bool nact = fnm > 0.0;
    const d3 fn = nact ? smul(fnm, n) : d3z();
    const double c = -P.kappa * sqrt(ra * rb);
    const d3 fc = smul(c, n);
    const bool tang = sqrt(dot(d0, d0)) > 0.0 || sqrt(dot(vt, vt)) > 0.0;
    d3 ft = d3z(), t = d3z(), g = d3z();
    double ft0len = 0.0, glen = 0.0, lim = 0.0;
    bool slip = false;
    if (tang) {
        const d3 dtv = vadd(d0, muls(vt, dt));
        const d3 ft0 = vsub(smul(-kt, dtv), smul(P.gamma_t, vt));
        ft0len = sqrt(dot(ft0, ft0));
        g = vsub(fn, fc);
        glen = sqrt(dot(g, g));
        lim = P.mu_s * glen;
        slip = ft0len > lim;
        if (slip) {
            t = divs(ft0, ft0len);
            ft = smul(lim, t);
        } else {
            ft = ft0;
        }
    }
    // ---- reverse
    d3 nb = d3z(), ftb = d3z(), fnb = d3z(), fcb = d3z(), vtb = d3z(), velb = d3z(),
       vlb = d3z(), d0b = d3z(), cab = d3z(), cbb = d3z();
    double sab = 0.0, sbb = 0.0, deltab = 0.0, vnb = 0.0, Lb = 0.0;
    // T = -sa (n x ft)
    {
        const d3 u = cross(n, ft);
        const d3 ub = smul(-sa, Tb);
        sab += -dot(u, Tb);
        acc3(nb, cross(ft, ub));
        acc3(ftb, cross(ub, n));
    }
    // F = fn + ft + fc
    acc3(fnb, Fb);
    acc3(ftb, Fb);
    acc3(fcb, Fb);
    if (tang) {
        d3 ft0b;
        if (slip) {
            const double ik = -1.0 / kt;
            const d3 tb = vadd(smul(lim, ftb), smul(ik * P.mu_d * glen, db));
            const double limb = dot(t, ftb);
            const double glenb = P.mu_s * limb + ik * P.mu_d * dot(t, db);
            mub += glen * limb + ik * glen * dot(t, db);
            acc3(vtb, smul(ik * P.gamma_t, db));
            ft0b = divs(vsub(tb, smul(dot(t, tb), t)), ft0len);
            if (glen > 0.0) {
                const d3 gb = smul(glenb / glen, g);
                acc3(fnb, gb);
                fcb = vsub(fcb, gb);
            }
        } else {
            ft0b = ftb;
        }
        // ft0 = -kt dtv - gamma_t vt, dtv = d0 + vt dt (dtv is the new
        // history in the stick branch)
        d3 dtvb = smul(-kt, ft0b);
        if (!slip) acc3(dtvb, db);
        acc3(vtb, smul(-P.gamma_t, ft0b));
        acc3(d0b, dtvb);
        acc3(vtb, smul(dt, dtvb));
    }
    // fc = c n
    acc3(nb, smul(c, fcb));
    // fn = fnm n
    if (nact) {
        const double fnmb = dot(n, fnb);
        acc3(nb, smul(fnm, fnb));
        deltab += -kn * fnmb;
        vnb += P.gamma_n * fnmb;
        knb += -delta * fnmb;
        gnb += vn * fnmb;
    }
    // d0 = h0 - (n.h0) n
    {
        d3 hb = d0b;
        const double s2b = -dot(n, d0b);
        acc3(nb, smul(-s2, d0b));
        acc3(nb, smul(s2b, h0));
        acc3(hb, smul(s2b, n));
        acc3(h0b, hb);
    }
    // vt = vel - (n.vel) n
    {
        acc3(velb, vtb);
        const double s1b = -dot(n, vtb);
        acc3(nb, smul(-s1, vtb));
        acc3(nb, smul(s1b, vel));
        acc3(velb, smul(s1b, n));
    }
    // vn = -(n.vl)
    acc3(nb, smul(-vnb, vl));
    acc3(vlb, smul(-vnb, n));
    // vel = vl + sa ca + sb cb
    acc3(vlb, velb);
    sab += dot(ca, velb);
    acc3(cab, smul(sa, velb));
    sbb += dot(cb, velb);
    acc3(cbb, smul(sb, velb));
    deltab += 0.5 * sab + 0.5 * sbb;
    // ca = n x wa, cb = n x wb
    acc3(nb, cross(wa, cab));
    acc3(wab, cross(cab, n));
    acc3(nb, cross(wb, cbb));
    acc3(wbb, cross(cbb, n));
    // vl = va - vb
    acc3(vab, vlb);
    vbb = vsub(vbb, vlb);
    // n = X / L, delta = L - (ra + rb), L = |X|
    d3 Xb = divs(nb, L);
    Lb += -dot(nb, n) / L;
    Lb += deltab;
    acc3(Xb, smul(Lb, n));
    acc3(xab, Xb);
    xbb = vsub(xbb, Xb);
}

struct AdjArgs {
    const DevBox *box;
    uint32_t n;
    uint64_t iter;                 // index of the step being reversed
    // tape: state at the start of the step (original order)
    const double4 *x, *vel, *angvel;
    const uint32_t *rows_pre, *rows_post;
    const double4 *hist;
    // adjoints of the step's outputs (state s+1) and of its inputs (state s)
    const double4 *lx_n, *lv_n, *lw_n, *lA_n, *lO_n;
    double4 *lx, *lv, *lw, *lA, *lO;
    double4 *lH;                   // per slot; read as d(out history), written as d(in history)
    double *gparam;                // [3] d/dk_n, d/dgamma_n, d/dmu
};

__device__ __forceinline__ void atomic_add3(double4 *p, d3 v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}

// Identity part of the TY3 reverse, written before the contact pass adds
// its (atomic) contributions.
__global__ void k_adj_init(AdjArgs J)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.n) return;
    const double dt = J.box->dt;
    const double4 lx = J.lx_n[i], lv = J.lv_n[i], lw = J.lw_n[i];
    J.lx[i] = make_double4(lx.x, lx.y, lx.z, 0.0);
    J.lv[i] = make_double4(dt * lx.x + lv.x, dt * lx.y + lv.y, dt * lx.z + lv.z, 0.0);
    J.lw[i] = make_double4(lw.x, lw.y, lw.z, 0.0);
    if (J.iter > 0) {
        const double cx = -dt * dt / 6.0, cv = -0.5 * dt;
        J.lA[i] = make_double4(cx * lx.x + cv * lv.x, cx * lx.y + cv * lv.y, cx * lx.z + cv * lv.z, 0.0);
        J.lO[i] = make_double4(cv * lw.x, cv * lw.y, cv * lw.z, 0.0);
    } else {
        J.lA[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        J.lO[i] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

// Adjoint of the forces and torques of sphere i: the contacts of its row
// (frozen set) and the walls.
__global__ void __launch_bounds__(128) k_adj_contacts(AdjArgs J)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double knb = 0.0, gnb = 0.0, mub = 0.0;
    if (i < J.n) {
        const DevBox &B = *J.box;
        const SphParams &P = B.P;
        const double dt = B.dt;
        const double4 x4 = J.x[i], v4 = J.vel[i], w4 = J.angvel[i];
        const d3 xa = xyz(x4), va = xyz(v4), wa = xyz(w4);
        const double ra = x4.w;
        const double m = 4.0 / 3.0 * PI * ra * ra * ra * P.rho;
        const double I = 2.0 / 5.0 * m * ra * ra;
        const double4 lxn = J.lx_n[i], lvn = J.lv_n[i], lwn = J.lw_n[i], lAn = J.lA_n[i],
                      lOn = J.lO_n[i];
        const double cx = 2.0 / 3.0 * dt * dt, cv = 1.5 * dt;
        double lacc[3] = {cx * lxn.x + cv * lvn.x + lAn.x, cx * lxn.y + cv * lvn.y + lAn.y,
                          cx * lxn.z + cv * lvn.z + lAn.z};
        double lalp[3] = {cv * lwn.x + lOn.x, cv * lwn.y + lOn.y, cv * lwn.z + lOn.z};
        // fixed-velocity masks, integration.cuh:131-160
        const double fv = v4.w;
        if (fv > 0.0001 && fv < 10.0) {
            lacc[0] = lacc[1] = 0.0;
            lalp[0] = lalp[1] = lalp[2] = 0.0;
        }
        if (fv >= 10.0) {
            lacc[1] = 0.0;
            lalp[0] = lalp[2] = 0.0;
        }
        if (fv < -0.0001) {
            lacc[0] = lacc[1] = lacc[2] = 0.0;
            lalp[0] = lalp[1] = lalp[2] = 0.0;
        }
        const d3 Fb = mk(lacc[0] / m, lacc[1] / m, lacc[2] / m);
        const d3 Tb = mk(lalp[0] / I, lalp[1] / I, lalp[2] / I);
        d3 xab = d3z(), vab = d3z(), wab = d3z();
        // A slot that is empty after this step's contact search holds no
        // history adjoint: the step after wrote one only to slots that held
        // a contact at its start, i.e. at the end of this step, and those
        // were occupied after this step's search.  So only the occupied
        // slots are read and written.
        uint32_t occ = 0;
        {
            const uint4 *rp = reinterpret_cast<const uint4 *>(J.rows_post + (size_t)i * NC);
#pragma unroll
            for (int q4 = 0; q4 < NC / 4; ++q4) {
                const uint4 w4 = rp[q4];
                occ |= (w4.x != EMPTY ? 1u : 0u) << (4 * q4);
                occ |= (w4.y != EMPTY ? 1u : 0u) << (4 * q4 + 1);
                occ |= (w4.z != EMPTY ? 1u : 0u) << (4 * q4 + 2);
                occ |= (w4.w != EMPTY ? 1u : 0u) << (4 * q4 + 3);
            }
        }
        for (uint32_t m = occ; m; m &= m - 1u) {
            const int s = __ffs(m) - 1;
            const size_t q = (size_t)i * NC + s;
            const uint32_t w = J.rows_post[q];
            const double4 dbo = J.lH[q];
            double4 h0b_out = make_double4(0.0, 0.0, 0.0, 0.0);
            {
                const uint32_t b = w & ID_MASK;
                int sx, sy;
                decode_shift(w >> CODE_SHIFT, sx, sy);
                const d3 dm = shift_vec(B, sx, sy);
                const double4 xb4 = J.x[b];
                const d3 xb = xyz(xb4);
                const d3 X = vadd(vsub(xa, xb), dm);
                const double len = sqrt(dot(X, X));
                if (len - (ra + xb4.w) < 0.0) {
                    d3 xbb = d3z(), vbb = d3z(), wbb = d3z(), h0b = d3z();
                    linear_contact_vjp(P, dt, xa, xb, dm, va, xyz(J.vel[b]), wa, xyz(J.angvel[b]),
                                       ra, xb4.w, xyz(J.hist[q]), Fb, Tb, xyz(dbo), xab, xbb, vab,
                                       vbb, wab, wbb, h0b, knb, gnb, mub);
                    atomic_add3(J.lx + b, xbb);
                    atomic_add3(J.lv + b, vbb);
                    atomic_add3(J.lw + b, wbb);
                    // the history read at this step was written by the
                    // previous step only when the contact already existed
                    if (J.rows_pre[q] != EMPTY) h0b_out = make_double4(h0b.x, h0b.y, h0b.z, 0.0);
                }
            }
            J.lH[q] = h0b_out;
        }
        // walls, contactmodels.cuh:10-117 with gamma_wt = 0 (normal force only)
        double wpos[5] = {B.L[2], B.L[0], 0.0, B.L[1], 0.0};
        for (uint32_t k = 0; k < 5 && k < B.nw; ++k) wpos[k] = B.wnx[k][3];
        const double kn = P.k_n;
        auto wall = [&](double delta, d3 nrm, int axis, double sgn) {
            if (!(delta < 0.0)) return;
            const double vn = dot(va, nrm);
            const double fnm = -kn * delta - P.gamma_wn * vn;
            if (!(fnm > 0.0)) return;
            const double fnmb = dot(nrm, Fb);
            knb += -delta * fnmb;
            const double deltab = -kn * fnmb;
            acc3(vab, smul(-P.gamma_wn * fnmb, nrm));
            if (axis == 0) xab.x += sgn * deltab;
            else if (axis == 1) xab.y += sgn * deltab;
            else xab.z += sgn * deltab;
        };
        wall(wpos[0] - (xa.z + ra), mk(0.0, 0.0, -1.0), 2, -1.0);
        wall(xa.z - ra - B.origo[2], mk(0.0, 0.0, 1.0), 2, 1.0);
        if (B.periodic == 0) {
            wall(wpos[1] - (xa.x + ra), mk(-1.0, 0.0, 0.0), 0, -1.0);
            wall(xa.x - ra - wpos[2], mk(1.0, 0.0, 0.0), 0, 1.0);
        }
        if (B.periodic == 0 || B.periodic == 2) {
            wall(wpos[3] - (xa.y + ra), mk(0.0, -1.0, 0.0), 1, -1.0);
            wall(xa.y - ra - wpos[4], mk(0.0, 1.0, 0.0), 1, 1.0);
        }
        atomic_add3(J.lx + i, xab);
        atomic_add3(J.lv + i, vab);
        atomic_add3(J.lw + i, wab);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        knb += __shfl_down_sync(0xffffffffu, knb, o);
        gnb += __shfl_down_sync(0xffffffffu, gnb, o);
        mub += __shfl_down_sync(0xffffffffu, mub, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(J.gparam + 0, knb);
        atomicAdd(J.gparam + 1, gnb);
        atomicAdd(J.gparam + 2, mub);
    }
}

int adjoint_step(const DevBox *box, uint32_t n, uint64_t iter, const double4 *x,
                 const double4 *vel, const double4 *angvel, const uint32_t *rows_pre,
                 const uint32_t *rows_post, const double4 *hist, const double4 *const lnext[5],
                 double4 *const lcur[5], double4 *lH, double *gparam, cudaStream_t st)
{
    AdjArgs J;
    J.box = box;
    J.n = n;
    J.iter = iter;
    J.x = x;
    J.vel = vel;
    J.angvel = angvel;
    J.rows_pre = rows_pre;
    J.rows_post = rows_post;
    J.hist = hist;
    J.lx_n = lnext[0];
    J.lv_n = lnext[1];
    J.lw_n = lnext[2];
    J.lA_n = lnext[3];
    J.lO_n = lnext[4];
    J.lx = lcur[0];
    J.lv = lcur[1];
    J.lw = lcur[2];
    J.lA = lcur[3];
    J.lO = lcur[4];
    J.lH = lH;
    J.gparam = gparam;
    k_adj_init<<<(n + 255) / 256, 256, 0, st>>>(J);
    k_adj_contacts<<<(n + 127) / 128, 128, 0, st>>>(J);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}

}  // namespace sph
