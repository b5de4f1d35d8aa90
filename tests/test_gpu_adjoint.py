"""The hand-written adjoint (sph_adjoint_forward / sph_adjoint_backward,
behind sphere_b200.adjoint.rollout) against (1) FP64 torch autograd through
the dense restatement torch_dem.py at N = 2000, (2) central finite
differences of the GPU forward with relative step 1e-6, (3) itself with
other checkpoint intervals, and the state it leaves behind."""
import numpy
import pytest
import torch

import torch_dem
from sphere_b200 import adjoint, scenes
from sphere_b200.runner import SphereError, Stepper

pytestmark = pytest.mark.gpu

DEV = 0


def _t(v, grad=False, device="cpu"):
    return torch.tensor(float(v), dtype=torch.float64, requires_grad=grad, device=device)


def _target(n, seed, steps):
    """Final positions of the target run (k_n = 1e8, gamma_n = 50, mu = 0.4)
    from the GPU forward."""
    tgt = scenes.reparam(scenes.loose_pack(n, seed=seed), k_n=1e8, gamma_n=50.0, mu=0.4)
    st = Stepper([tgt], precision="fp64", length="fp64", device=DEV)
    st.upload()
    st.step(steps)
    hp, _ = st.download()
    st.close()
    return torch.from_numpy(numpy.ascontiguousarray(hp.x[:, :3]))


def _adjoint_grads(s, xt, steps, ckpt):
    p = [_t(1.5e8, True), _t(20.0, True), _t(0.5, True)]
    v0 = torch.tensor(s.vel, requires_grad=True)
    x = adjoint.rollout(s, *p, v0, steps, ckpt=ckpt, device=DEV)
    loss = ((x - xt) ** 2).sum(1).mean()
    loss.backward()
    return loss.item(), numpy.array([q.grad.item() for q in p]), v0.grad.numpy().copy(), x


def test_adjoint_matches_torch_autograd_n2000():
    n, steps, seed = 2000, 100, 0
    s = scenes.loose_pack(n, seed=seed)
    xt = _target(n, seed, steps)
    loss_a, gp_a, gv_a, x_a = _adjoint_grads(s, xt, steps, ckpt=30)
    dev = torch.device("cuda", DEV)
    p = [_t(1.5e8, True, dev), _t(20.0, True, dev), _t(0.5, True, dev)]
    v0 = torch.tensor(s.vel, dtype=torch.float64, device=dev, requires_grad=True)
    x = torch_dem.rollout(s, *p, v0, steps)
    loss = ((x - xt.to(dev)) ** 2).sum(1).mean()
    loss.backward()
    gp_t = numpy.array([q.grad.item() for q in p])
    gv_t = v0.grad.cpu().numpy()
    # same forward up to the order of the force sums
    assert numpy.abs(x.detach().cpu().numpy() - x_a.detach().numpy()).max() < 1e-13
    assert abs(loss.item() - loss_a) <= 1e-9 * loss_a
    rel = numpy.abs(gp_a - gp_t) / numpy.abs(gp_t)
    print("param gradients adjoint", gp_a, "autograd", gp_t, "rel", rel)
    assert (rel < 1e-7).all(), rel
    gv_rel = numpy.linalg.norm(gv_a - gv_t) / numpy.linalg.norm(gv_t)
    print("v0 gradient relative error", gv_rel)
    assert gv_rel < 1e-7


def test_adjoint_matches_central_differences():
    """Relative step 1e-6 on k_n, gamma_n, mu and on v0 along one random
    direction; scene chosen so that no contact event or stick/slip switch
    falls inside a difference step (the same scene is checked on the CPU
    with the torch restatement)."""
    n, steps, seed = 120, 60, 5
    s = scenes.loose_pack(n, seed=seed)
    xt = _target(n, seed, steps).numpy()
    _, gp, gv, _ = _adjoint_grads(s, torch.from_numpy(xt), steps, ckpt=25)

    def loss(kn, gn, mu, vel):
        q = scenes.reparam(s, k_n=kn, gamma_n=gn, mu=mu)
        q.vel[:] = vel
        st = Stepper([q], precision="fp64", length="fp64", device=DEV)
        st.upload()
        st.step(steps)
        hp, _ = st.download()
        st.close()
        return float(((hp.x[:, :3] - xt) ** 2).sum(1).mean())

    base = [1.5e8, 20.0, 0.5]
    for k in range(3):
        h = 1e-6 * base[k]
        a, b = list(base), list(base)
        a[k] += h
        b[k] -= h
        fd = (loss(*a, s.vel) - loss(*b, s.vel)) / (2 * h)
        print("param", k, "adjoint", gp[k], "fd", fd)
        assert abs(fd - gp[k]) <= 1e-4 * abs(fd)
    u = numpy.random.default_rng(5).normal(size=(n, 3))
    u /= numpy.linalg.norm(u)
    h = 1e-6 * float(numpy.linalg.norm(s.vel))
    fd = (loss(*base, s.vel + h * u) - loss(*base, s.vel - h * u)) / (2 * h)
    ad = float((gv * u).sum())
    print("v0 direction adjoint", ad, "fd", fd)
    assert abs(fd - ad) <= 1e-4 * abs(fd)


def test_checkpoint_interval_does_not_change_gradients():
    n, steps, seed = 400, 50, 3
    s = scenes.loose_pack(n, seed=seed)
    xt = _target(n, seed, steps)
    ref = _adjoint_grads(s, xt, steps, ckpt=50)
    for ckpt in (1, 7, 64):
        got = _adjoint_grads(s, xt, steps, ckpt=ckpt)
        assert got[0] == ref[0]
        assert numpy.array_equal(got[1], ref[1]) or \
            (numpy.abs(got[1] - ref[1]) <= 1e-12 * numpy.abs(ref[1])).all()
        assert numpy.abs(got[2] - ref[2]).max() <= 1e-12 * numpy.abs(ref[2]).max()


def test_backward_leaves_the_forward_final_state():
    n, steps = 300, 40
    s = scenes.loose_pack(n, seed=2)
    st = Stepper([s], precision="fp64", length="fp64", device=DEV)
    st.upload()
    st.adjoint_forward(steps, 16)
    hp1, _ = st.download()
    st.adjoint_backward(numpy.ones((n, 3)))
    hp2, _ = st.download()
    assert numpy.array_equal(hp1.x, hp2.x) and numpy.array_equal(hp1.vel, hp2.vel)
    st.step(1)       # the handle steps on from there
    with pytest.raises(SphereError):
        st.adjoint_backward(numpy.ones((n, 3)))    # checkpoints were released
    st.close()


def test_adjoint_rejects_unsupported_setups():
    s = scenes.loose_pack(200, seed=1)
    st = Stepper([s], precision="mixed", length="fp64", device=DEV)
    st.upload()
    with pytest.raises(SphereError) as e:
        st.adjoint_forward(10, 5)
    assert e.value.status == 8       # SPH_ERR_UNSUPPORTED
    st.close()
    st = Stepper([s], precision="fp64", length="reference", device=DEV)
    st.upload()
    with pytest.raises(SphereError):
        st.adjoint_forward(10, 5)
    st.close()
