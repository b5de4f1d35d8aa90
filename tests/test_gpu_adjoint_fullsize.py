"""The adjoint at the size of the differentiable settling/impact workload:
50,000 spheres (radii U[0.009, 0.011] m, loose pack porosity 0.5, initial
velocities N(0, 0.1) m/s), linear contacts with k_n = 1.5e8, gamma_n = 20,
mu = 0.5, loss = mean squared distance of the final positions to a run with
k_n = 1e8, gamma_n = 50, mu = 0.4.

The adjoint is the derivative of the step with each step's contact set
frozen.  A central difference measures that derivative only while the two
perturbed runs keep the same contact history: where a contact begins, the
damped normal force jumps from zero to gamma_n v_n, so a perturbation that
moves a contact's first step makes the loss jump.  At this size a relative
step of 1e-6 already moves contacts (over 100 steps the per-step contact
counts of the two runs differ at 11 steps for k_n and 14 for v0; over 1,000
steps at 321 to 774), and the difference quotients then measure those
jumps; below a relative step of ~3e-8 the FP64 rounding of the positions
(differences of ~1e-14 m against an ulp of ~3e-17 m) limits the quotients
to ~1e-3.  Between the two, over 50 steps with a relative step of 3e-7, the
two runs of every difference keep the same contact counts at every step
(asserted) and the gradients with respect to k_n, gamma_n, mu and the
initial velocities (along a random direction) agree within 1e-4 relative.
The loss difference is taken from the position differences,
mean((x+ - x-) . (x+ + x- - 2 x_target)), which does not cancel two
losses.  The full 2,000-step, checkpoint-100 run is the benchmark's; its
gradient is checked against dense FP64 autograd at N = 2,000 in
test_gpu_adjoint.py."""
import numpy
import pytest
import torch

from sphere_b200 import adjoint, scenes
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

N, STEPS, CKPT, REL_STEP = 50000, 50, 20, 3e-7
BASE = (1.5e8, 20.0, 0.5)


@pytest.fixture(scope="module")
def workload():
    s = scenes.loose_pack(N, seed=0, device=0)
    tgt = scenes.reparam(s, k_n=1e8, gamma_n=50.0, mu=0.4)
    st = Stepper([tgt], precision="fp64", length="fp64", device=0)
    st.upload()
    st.step(STEPS)
    hp, _ = st.download()
    st.close()
    return s, numpy.ascontiguousarray(hp.x[:, :3])


def _run(s, kn, gn, mu, vel):
    """(final positions, live contacts after each step)"""
    q = scenes.reparam(s, k_n=kn, gamma_n=gn, mu=mu)
    q.vel[:] = vel
    st = Stepper([q], precision="fp64", length="fp64", device=0)
    st.upload()
    counts = []
    for _ in range(STEPS):
        st.step(1)
        counts.append(st.count_contacts())
    hp, _ = st.download()
    st.close()
    return numpy.ascontiguousarray(hp.x[:, :3]), counts


def test_adjoint_matches_central_differences_at_full_size(workload):
    s, xt = workload
    p = [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in BASE]
    v0 = torch.tensor(s.vel, requires_grad=True)
    x = adjoint.rollout(s, *p, v0, STEPS, ckpt=CKPT, device=0)
    loss = ((x - torch.from_numpy(xt)) ** 2).sum(1).mean()
    loss.backward()
    gp = [q.grad.item() for q in p]
    gv = v0.grad.numpy()
    x0, _ = _run(s, *BASE, s.vel)
    l0 = float(((x0 - xt) ** 2).sum(1).mean())
    assert abs(loss.item() - l0) <= 1e-12 * l0
    u = numpy.random.default_rng(7).normal(size=(N, 3))
    u /= numpy.linalg.norm(u)
    cases = []
    for k, name in enumerate(("k_n", "gamma_n", "mu")):
        h = REL_STEP * BASE[k]
        a, b = list(BASE), list(BASE)
        a[k] += h
        b[k] -= h
        cases.append((name, gp[k], h, (*a, s.vel), (*b, s.vel)))
    h = REL_STEP * float(numpy.linalg.norm(s.vel))
    cases.append(("v0 . u", float((gv * u).sum()), h, (*BASE, s.vel + h * u),
                  (*BASE, s.vel - h * u)))
    for name, ad, h, plus, minus in cases:
        (xp, cp), (xm, cm) = _run(s, *plus), _run(s, *minus)
        assert cp == cm, "%s: the perturbed runs' contact histories differ" % name
        fd = float(((xp - xm) * (xp + xm - 2.0 * xt)).sum(1).mean()) / (2 * h)
        rel = abs(ad - fd) / abs(fd)
        print("%-8s adjoint %.9e  central difference %.9e  relative %.2e" % (name, ad, fd, rel))
        assert rel < 1e-4, (name, ad, fd, rel)
