"""The Darcy coupling on the GPU (sph_darcy.cu through the C ABI) against
the Darcy oracle (oracle/sphere_oracle.c, itself pinned to the reference's
own Darcy kernels by tests/test_darcy_oracle.py), bit for bit: every fluid
field, the pressure force on each sphere, the sphere state after the
coupled steps and the Jacobi record of every fluid step, on the scenes of
tests/darcy_cases.py.  The Jacobi loop runs on the device (a conditional
node of the step graph), so splitting the steps into calls must not change
a bit either; run() writes the reference's conv.log and output files."""
import copy
import os

import numpy
import pytest

import darcy_cases
import oracle as O
import sphere_b200
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu


def gpu_run(s, chunks):
    st = Stepper([copy.deepcopy(s)], precision="fp64", length="reference")
    st.upload()
    log = ([], [], [])
    for k in chunks:
        st.step(k)
        for acc, part in zip(log, st.darcy_log()):
            acc.extend(part.tolist())
    hp, _ = st.download()
    fluid = st.darcy_get()
    st.close()
    return hp, fluid, log


def oracle_run(s, steps):
    r = O.CpuRun(copy.deepcopy(s), which="oracle")
    assert r.step(steps) == 0
    return r


def compare(hp, fluid, log, r, name):
    for f, g in (("p_f", "p"), ("v_f", "v"), ("phi", "phi"), ("dphi_raw", "dphi"), ("k", "k")):
        assert numpy.array_equal(fluid[f], r.fluid_cells(g)), (name, f)
    assert numpy.array_equal(fluid["f_p"], r.fluid["f_p"][:r.n, :3]), (name, "f_p")
    assert numpy.array_equal(hp.x, r.x), (name, "x")
    assert numpy.array_equal(hp.vel, r.vel), (name, "vel")
    assert numpy.array_equal(hp.force, r.force[:, :3]), (name, "force")
    assert numpy.array_equal(hp.angvel, r.angvel[:, :3]), (name, "angvel")
    assert numpy.array_equal(hp.torque, r.torque[:, :3]), (name, "torque")
    step, iters, ok = r.darcy_log()
    assert log[0] == step.tolist() and log[1] == iters.tolist() and log[2] == ok.tolist(), name


@pytest.mark.parametrize("name", darcy_cases.CASES)
def test_darcy_step_equals_oracle(name):
    s, steps = darcy_cases.make(name)
    hp, fluid, log = gpu_run(s, [steps])
    compare(hp, fluid, log, oracle_run(s, steps), name)


def test_darcy_grid_with_more_cells_than_threads():
    """82,800 cells: the Jacobi threads take several cells each (the other
    form of the loop); still the oracle's every bit."""
    s = darcy_cases.big_fluid_box()
    hp, fluid, log = gpu_run(s, [3])
    r = oracle_run(s, 3)
    for f, g in (("p_f", "p"), ("v_f", "v"), ("phi", "phi"), ("k", "k")):
        assert numpy.array_equal(fluid[f], r.fluid_cells(g)), f
    step, iters, ok = r.darcy_log()
    assert log[1] == iters.tolist() and log[2] == ok.tolist()
    assert min(iters) > 10


@pytest.mark.parametrize("name", ["darcy_pack_wall", "darcy_pack_modulated", "darcy_pack_bcs"])
def test_darcy_steps_split_into_calls_change_no_bit(name):
    s, steps = darcy_cases.make(name)
    a = gpu_run(s, [steps])
    b = gpu_run(s, [1, 6, steps - 7])
    for f in a[1]:
        assert numpy.array_equal(a[1][f], b[1][f]), f
    assert numpy.array_equal(a[0].x, b[0].x) and numpy.array_equal(a[0].force, b[0].force)
    assert a[2] == b[2]


def test_darcy_run_writes_conv_log_and_outputs(tmp_path):
    """tests/cfd_tests_darcy.py restated: run() of the pure-fluid box with
    no forcing (pressure stays zero, no iteration in any solve, flow below
    1e-6) and with a pressure step at the top, run until it is close to the
    steady state (linear pressure profile within 0.1 of the top value, flow
    towards -z everywhere, few iterations per solve at the end)."""
    root = str(tmp_path)
    s = darcy_cases.fluid_box()
    s.time_total[0] = s.time_dt[0] * 10
    assert s.run(verbose=False, root=root) == 0
    py = sphere_b200.sim(sid=s.sid, fluid=True)
    py.readlast(verbose=False, root=root)
    assert numpy.array_equal(py.p_f, numpy.zeros(py.p_f.shape))
    it = numpy.loadtxt(os.path.join(root, "output", s.sid + "-conv.log"), ndmin=2)
    assert it[:, 1].sum() == 0.0
    assert (numpy.abs(py.v_f) < 1.0e-6).all()

    s = darcy_cases.fluid_box(p_top=1.0, dt=1.0e-6)
    s.time_total[0] = s.time_dt[0] * 3000
    s.time_file_dt[0] = s.time_dt[0] * 500
    assert s.run(verbose=False, root=root) == 0
    py = sphere_b200.sim(sid=s.sid, fluid=True)
    py.readlast(verbose=False, root=root)
    ideal = numpy.linspace(s.p_f[0, 0, 0], s.p_f[0, 0, -1], s.num[2])
    assert (numpy.abs(ideal - py.p_f[0, 0, :]) < 1.0e-1).all()
    assert (py.v_f[:, :, :, 2] < 0.0).all() and (numpy.abs(py.v_f[:, :, :, 0:2]) < 1.0e-7).all()
    it = numpy.loadtxt(os.path.join(root, "output", s.sid + "-conv.log"), ndmin=2)
    assert it[0, 0] == 1 and (it[:, 0] % 10 == 1).all()
    assert (it[-5:, 1] < 20).all()


def test_darcy_run_output_matches_oracle(tmp_path):
    """run() of a sphere pack in a fluid: the last output file holds the
    oracle's state after the same steps, the fluid block as the reference's
    writer stores it (dphi per fluid step)."""
    root = str(tmp_path)
    s, steps = darcy_cases.make("darcy_pack_wall")
    s.time_total[0] = s.time_dt[0] * (steps - 0.5)
    s.time_file_dt[0] = s.time_dt[0] * 5
    assert s.run(verbose=False, root=root) == 0
    py = sphere_b200.sim(sid=s.sid, fluid=True)
    py.ndem = s.ndem
    py.readlast(verbose=False, root=root)
    r = oracle_run(s, steps)
    assert numpy.array_equal(py.p_f, r.fluid_cells("p"))
    # the file holds the solver's dphi; the reader divides by time_dt * ndem
    assert numpy.array_equal(py.dphi, r.fluid_cells("dphi") / (py.time_dt * s.ndem))
    assert numpy.array_equal(py.x, r.x[:, :3])
    assert numpy.array_equal(py.f_p, r.fluid["f_p"][:r.n, :3])


def test_darcy_rejects_what_it_does_not_cover():
    s, _ = darcy_cases.make("darcy_pack_wall")
    st = Stepper([s, copy.deepcopy(s)], precision="fp64")
    st.upload()
    with pytest.raises(sphere_b200.runner.SphereError) as e:
        st.darcy_set(s)
    assert e.value.status == 8   # SPH_ERR_UNSUPPORTED: one box only
    st.close()
    st = Stepper([s], precision="mixed")
    with pytest.raises(sphere_b200.runner.SphereError):
        st.upload()              # the FP32-mixed form
    st.close()
