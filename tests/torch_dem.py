"""Dense FP64 torch restatement of the linear-contact DEM step, for the
gradient checks of the adjoint (test infrastructure, not product code).

One step follows the reference's interact + integrate for contact model 2
with kappa = 0, E = 0, no bonds and the static walls of a box with nw = 0:
src/contactsearch.cuh:329-371 + :484-559 (contact set: every pair with
negative overlap; tangential history kept per directed pair while the pair
stays in contact, zero for a new pair), src/contactmodels.cuh:244-411
contactLinear (normal force max(0, -k_n delta + gamma_n v_n), Coulomb
tangential force with the stick/slip history update), :10-117
contactLinear_wall with gamma_wt = 0, src/integration.cuh:14-305 (TY3
integration, no acceleration history at the first step).

The contact set of each step is found without gradient tracking (all-pairs
distances), so torch autograd through this function differentiates each
step with its contact set frozen and each law on the branch it took -- the
same definition the hand-written adjoint implements.  Lengths are sqrt of
the FP64 dot product (the SPH_LEN_FP64 form).  Periodic boundaries are not
handled (periodic must be 0).
"""
import torch

PI = 3.14159265358979


def _safe_len(v):
    return torch.sqrt(torch.clamp((v * v).sum(-1), min=1e-300))


def rollout(s, k_n, gamma_n, mu, v0, nsteps, contact_log=None):
    """Final positions after nsteps steps of sim s (periodic 0, nw 0) with
    k_n, gamma_n, mu (0-d float64 tensors) and initial velocities v0
    [np, 3] (float64 tensor).  Differentiable in all four.  contact_log, a
    list, receives the number and a checksum of each step's contact set and
    of the spheres touching each wall."""
    assert int(s.periodic[0]) == 0 and int(s.nw[0]) == 0
    dev = v0.device
    f64 = dict(dtype=torch.float64, device=dev)
    n = int(s.np[0])
    x = torch.tensor(s.x, **f64)
    r = torch.tensor(s.radius, **f64)
    rho = float(s.rho[0])
    m = 4.0 / 3.0 * PI * r * r * r * rho
    inertia = 2.0 / 5.0 * m * r * r
    g = torch.tensor(s.g, **f64)
    dt = float(s.time_dt[0])
    k_t = float(s.k_t[0])
    gamma_t = float(s.gamma_t[0])
    gamma_wn = float(s.gamma_wn[0])
    origo = [float(v) for v in s.origo]
    L = [float(v) for v in s.L]
    v = v0
    w = torch.tensor(s.angvel, **f64)
    A = torch.zeros(n, 3, **f64)
    O = torch.zeros(n, 3, **f64)
    keys_prev = torch.zeros(0, dtype=torch.int64, device=dev)
    H_prev = torch.zeros(0, 3, **f64)
    eye = torch.eye(n, dtype=torch.bool, device=dev)
    for it in range(nsteps):
        with torch.no_grad():
            xd = x.detach()
            # candidates from cdist (inexact), then the exact test the step
            # makes: sqrt of the FP64 dot product of the componentwise
            # difference
            d = torch.cdist(xd, xd)
            near = (d - (r[:, None] + r[None, :]) < 1e-6 * float(r.max())) & ~eye
            ii, jj = torch.nonzero(near, as_tuple=True)
            Xe = xd[ii] - xd[jj]
            le = torch.sqrt(Xe[:, 0] * Xe[:, 0] + Xe[:, 1] * Xe[:, 1] + Xe[:, 2] * Xe[:, 2])
            keep = le - (r[ii] + r[jj]) < 0.0
            ii, jj = ii[keep], jj[keep]
            keys = ii * n + jj
            if contact_log is not None:
                contact_log.append((int(keys.numel()), int((keys * 2654435761 % 1000003).sum())))
            if keys_prev.numel():
                pos = torch.searchsorted(keys_prev, keys).clamp(max=keys_prev.numel() - 1)
                found = keys_prev[pos] == keys
            else:
                pos = torch.zeros_like(keys)
                found = torch.zeros_like(keys, dtype=torch.bool)
        ra, rb = r[ii], r[jj]
        X = x[ii] - x[jj]
        Ln = torch.sqrt(X[:, 0] * X[:, 0] + X[:, 1] * X[:, 1] + X[:, 2] * X[:, 2])
        delta = Ln - (ra + rb)
        nrm = X / Ln[:, None]
        vl = v[ii] - v[jj]
        sa = (ra + delta / 2.0)[:, None]
        sb = (rb + delta / 2.0)[:, None]
        vel = vl + sa * torch.cross(nrm, w[ii], dim=1) + sb * torch.cross(nrm, w[jj], dim=1)
        vn = -(vl * nrm).sum(1)
        vt = vel - nrm * (nrm * vel).sum(1, keepdim=True)
        if H_prev.numel():
            h0 = torch.where(found[:, None], H_prev[pos], torch.zeros_like(X))
        else:
            h0 = torch.zeros_like(X)
        d0 = h0 - nrm * (nrm * h0).sum(1, keepdim=True)
        fnm = -k_n * delta + gamma_n * vn
        fn = torch.clamp(fnm, min=0.0)[:, None] * nrm
        with torch.no_grad():
            tang = (torch.sqrt((d0 * d0).sum(1)) > 0.0) | (torch.sqrt((vt * vt).sum(1)) > 0.0)
        dtv = d0 + vt * dt
        ft0 = -k_t * dtv - gamma_t * vt
        ft0len = _safe_len(ft0)
        fnlen = _safe_len(fn)
        lim = mu * fnlen
        with torch.no_grad():
            slip = tang & (torch.sqrt((ft0 * ft0).sum(1)) > lim)
        tdir = ft0 / ft0len[:, None]
        ft_slip = lim[:, None] * tdir
        dn_slip = (-1.0 / k_t) * (mu * fnlen[:, None] * tdir + gamma_t * vt)
        ft = torch.where(slip[:, None], ft_slip, ft0)
        dnew = torch.where(slip[:, None], dn_slip, dtv)
        ft = torch.where(tang[:, None], ft, torch.zeros_like(ft))
        dnew = torch.where(tang[:, None], dnew, torch.zeros_like(dnew))
        F = torch.zeros(n, 3, **f64).index_add(0, ii, fn + ft)
        T = torch.zeros(n, 3, **f64).index_add(0, ii, -sa * torch.cross(nrm, ft, dim=1))
        # static walls: top at L[2], bottom at origo[2], x at L[0] and 0, y at L[1] and 0
        walls = ((2, L[2], -1.0), (2, origo[2], 1.0), (0, L[0], -1.0), (0, 0.0, 1.0),
                 (1, L[1], -1.0), (1, 0.0, 1.0))
        cols = []
        for axis, pos_w, sgn in walls:
            if sgn < 0.0:
                dw = pos_w - (x[:, axis] + r)
            else:
                dw = x[:, axis] - r - pos_w
            vnw = sgn * v[:, axis]
            if contact_log is not None:
                hit = torch.nonzero(dw.detach() < 0.0).flatten()
                contact_log.append((int(hit.numel()), int((hit * 2654435761 % 1000003).sum())))
            fw = torch.where(dw < 0.0, torch.clamp(-k_n * dw - gamma_wn * vnw, min=0.0),
                             torch.zeros_like(dw))
            cols.append((axis, sgn * fw))
        Fw = torch.stack([sum(f for a, f in cols if a == k) for k in range(3)], 1)
        F = F + Fw
        acc = F / m[:, None] + g
        alpha = T / inertia[:, None]
        if it == 0:
            A0 = torch.zeros_like(acc)
            O0 = torch.zeros_like(alpha)
        else:
            A0, O0 = A, O
        x = x + v * dt + 0.5 * acc * dt * dt + (1.0 / 6.0) * ((acc - A0) / dt) * dt * dt * dt
        v = v + acc * dt + 0.5 * ((acc - A0) / dt) * dt * dt
        w = w + alpha * dt + 0.5 * ((alpha - O0) / dt) * dt * dt
        A, O = acc, alpha
        keys_prev, H_prev = keys, dnew
    return x
