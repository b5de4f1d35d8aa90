"""The dense torch restatement used to check the adjoint (torch_dem.py)
against the oracle's forward step, and its autograd gradient against
central finite differences -- both on the CPU."""
import numpy
import torch

import oracle as O
import torch_dem
from sphere_b200 import scenes


def _t(v, grad=False):
    return torch.tensor(float(v), dtype=torch.float64, requires_grad=grad)


def test_torch_restatement_matches_oracle_trajectory():
    s = scenes.loose_pack(300, seed=1)
    steps = 60
    run = O.CpuRun(s, "oracle", length_mode=1)   # SPH_LEN_FP64
    run.step(steps)
    with torch.no_grad():
        xt = torch_dem.rollout(s, _t(s.k_n[0]), _t(s.gamma_n[0]), _t(s.mu_s[0]),
                               torch.tensor(s.vel), steps).numpy()
    moved = numpy.abs(run.x[:, :3] - s.x).max()
    assert moved > 1e-6
    # same arithmetic up to the order of the per-sphere force sums
    assert numpy.abs(xt - run.x[:, :3]).max() < 1e-9 * moved


def test_torch_autograd_matches_central_differences():
    """Central differences with relative step 1e-6 on k_n, gamma_n, mu and
    on the initial velocities along one random direction.  The scene is one
    in which no contact starts or ends inside any difference step (checked)
    and no stick/slip switch falls inside one (the loss is only piecewise
    smooth in the parameters: contact onset with damping is a jump, stick/
    slip and normal-force release are kinks)."""
    n, steps, seed = 120, 60, 5
    s = scenes.loose_pack(n, seed=seed)
    tgt = scenes.reparam(scenes.loose_pack(n, seed=seed), k_n=1e8, gamma_n=50.0, mu=0.4)
    with torch.no_grad():
        xt = torch_dem.rollout(tgt, _t(1e8), _t(50.0), _t(0.4), torch.tensor(tgt.vel), steps)

    def loss(kn, gn, mu, v0, log=None):
        x = torch_dem.rollout(s, kn, gn, mu, v0, steps, log)
        return ((x - xt) ** 2).sum(1).mean()

    p = [_t(1.5e8, True), _t(20.0, True), _t(0.5, True)]
    v0 = torch.tensor(s.vel, requires_grad=True)
    loss(*p, v0).backward()
    base = [1.5e8, 20.0, 0.5]
    vb = torch.tensor(s.vel)
    with torch.no_grad():
        for k in range(3):
            h = 1e-6 * base[k]
            a, b = list(base), list(base)
            a[k] += h
            b[k] -= h
            la, lb = [], []
            fd = (loss(*map(_t, a), vb, la).item() - loss(*map(_t, b), vb, lb).item()) / (2 * h)
            assert la == lb, "a contact starts or ends inside the difference step"
            assert abs(fd - p[k].grad.item()) <= 1e-4 * abs(fd), (k, fd, p[k].grad.item())
        u = torch.tensor(numpy.random.default_rng(5).normal(size=(n, 3)))
        u /= u.norm()
        h = 1e-6 * float(vb.norm())
        fd = (loss(*map(_t, base), vb + h * u).item() - loss(*map(_t, base), vb - h * u).item()) / (2 * h)
        ad = float((v0.grad * u).sum())
        assert abs(fd - ad) <= 1e-4 * abs(fd), (fd, ad)
