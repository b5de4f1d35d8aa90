"""Step outputs against golden vectors recorded from the reference's own
kernels run on the CPU (tests/golden/steps_*.npz, made by
tests/golden/make_golden.py with oracle/_ref).  The CPU oracle must match
them bit for bit here; the GPU variant below does the same for the CUDA
step.  These fixtures need neither the reference sources nor its build."""
import os

import numpy
import pytest

import cases
import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["periodic_xy_wall_stress", "walls_all_sides", "contact_model_1", "bonds_breaking",
         "shear_stress_wall"]


def _golden(name):
    return numpy.load(os.path.join(GOLDEN, "steps_%s.npz" % name))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(name):
    g = _golden(name)
    s = cases.make(name)[0]
    run = O.CpuRun(s, "oracle")
    for k in (1, 10):
        run.step(1 if k == 1 else 9)
        for f in ("x", "vel", "angvel", "angpos", "xyzsum", "force", "torque", "es", "ev",
                  "es_dot", "ev_dot", "p", "contacts", "delta_t", "perm", "bonds", "bonds_delta",
                  "bonds_omega"):
            assert numpy.array_equal(getattr(run, f), g["%s_%d" % (f, k)]), (f, k)
        nx = numpy.array([list(run.box.walls.nx[w]) for w in range(6)])
        assert numpy.array_equal(nx, g["walls_nx_%d" % k])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_golden(name):
    from sphere_b200.runner import Stepper
    g = _golden(name)
    s = cases.make(name)[0]
    n = int(s.np[0])
    st = Stepper([s])
    st.upload()
    for k in (1, 10):
        st.step(1 if k == 1 else 9)
        hp, hb = st.download()
        assert numpy.array_equal(hp.x, g["x_%d" % k])
        assert numpy.array_equal(hp.vel, g["vel_%d" % k])
        for f in ("force", "torque", "angvel", "angpos", "xyzsum"):
            assert numpy.array_equal(getattr(hp, f), g["%s_%d" % (f, k)][:, :3]), f
        for f in ("es", "ev", "es_dot", "ev_dot", "p"):
            assert numpy.array_equal(getattr(hp, f), g["%s_%d" % (f, k)]), f
        c, dt, _ = st.contacts()
        assert numpy.array_equal(c, g["contacts_%d" % k])
        assert numpy.array_equal(dt, g["delta_t_%d" % k])
        _, perm, _, _ = st.sort_products()
        assert numpy.array_equal(perm, g["perm_%d" % k][:n])
    st.close()
