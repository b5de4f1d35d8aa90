"""The FP64 gravity-settling workload at its full size: 10,000 spheres,
radii U[0.010, 0.012] m, jittered cubic lattice (spacing 2.5 r_max) in a
0.5 x 0.5 m box with wall sides, linear contacts k_n = k_t = 1.16e9 without
damping, mu = 0.5, dt = 0.17 sqrt(m_min / k_n), 1,000 steps
(scenes.gravity_settling).  The GPU step equals the C oracle bit for bit
after steps 1, 100 and 1,000 in both length modes, in every field the
parity cases check, and so does a run of 1,000 steps queued at once
(sph_step_async, the overlapped wall stage) against single steps."""
import numpy
import pytest

import oracle as O
from sphere_b200 import scenes
from sphere_b200.runner import Stepper
from test_gpu_parity import check_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def settling():
    return scenes.gravity_settling(n=10000, seed=0, steps=1000)


@pytest.mark.parametrize("length", ["reference", "fp64"])
def test_settling_matches_oracle(settling, length):
    s = settling
    cpu = O.CpuRun(s, "oracle", length_mode=0 if length == "reference" else 1)
    st = Stepper([s], precision="fp64", length=length)
    st.upload()
    done = 0
    for k in (1, 100, 1000):
        st.step(k - done)
        cpu.step(k - done)
        done = k
        check_same(st, cpu, s)
    # the spheres fall freely for these 1,000 steps (5.2e-4 s): the lattice
    # is 2.5 r_max apart and the lowest layer above the floor
    assert int((cpu.contacts != 10000).sum()) == 0
    assert float(cpu.vel[:, 2].max()) < 0.0
    st.close()


def test_settling_one_run_equals_single_steps(settling):
    a = Stepper([settling], precision="fp64")
    b = Stepper([settling], precision="fp64")
    a.upload()
    b.upload()
    a.step(1000)
    for _ in range(1000):
        b.step(1)
    ha, _ = a.download()
    hb, _ = b.download()
    for name in ("x", "vel", "angvel", "xyzsum", "force"):
        assert numpy.array_equal(getattr(ha, name), getattr(hb, name)), name
    assert a.boxes()[0].t_current == b.boxes()[0].t_current
    a.close()
    b.close()
