"""The Darcy oracle (oracle/sphere_oracle.c, the C restatement of
src/darcy.cuh and the Darcy part of src/device.cu:1891-2419) against the
reference's own Darcy kernels compiled for the CPU (oracle/_ref,
oracle/ref_emu/ref_harness.cpp), bit for bit: every fluid field, the
pressure force on each sphere, the sphere state and the per-step Jacobi
record, on the scenes of tests/darcy_cases.py.  Plus the checks of the
reference's own Darcy tests (tests/cfd_tests_darcy.py), on the oracle."""
import numpy
import pytest

import darcy_cases
import oracle as O

FIELDS = ("p", "v", "phi", "dphi", "k", "grad_p", "grad_k", "vp_avg", "norm", "p_old",
          "dp_expl", "f_p")
PARTICLE = ("x", "vel", "force", "angvel", "torque", "angpos", "xyzsum")


def run(name, which):
    s, steps = darcy_cases.make(name)
    r = O.CpuRun(s, which=which)
    flags = r.step(steps)
    return r, flags


@pytest.mark.skipif(not O.available("ref") and O.reference_root() is None,
                    reason="the reference's kernels are not built here")
@pytest.mark.parametrize("name", darcy_cases.CASES)
def test_darcy_oracle_equals_reference_kernels(name):
    a, fa = run(name, "oracle")
    b, fb = run(name, "ref")
    assert fa == fb == 0
    for f in FIELDS:
        assert numpy.array_equal(a.fluid[f], b.fluid[f]), f
    for f in PARTICLE:
        assert numpy.array_equal(getattr(a, f), getattr(b, f)), f
    for x, y in zip(a.darcy_log(), b.darcy_log()):
        assert numpy.array_equal(x, y)
    assert a.darcy.wall0_iz == b.darcy.wall0_iz
    assert a.darcy.filetimeclock == b.darcy.filetimeclock


def test_no_forcing_gives_no_flow():
    """tests/cfd_tests_darcy.py, "No forcing": no gravity, no pressure
    gradient: the pressure stays zero, every solve converges at once and
    the flow is below 1e-6."""
    r, flags = run("darcy_still_fluid", "oracle")
    assert flags == 0
    assert numpy.array_equal(r.fluid_cells("p"), numpy.zeros(r.fluid_cells("p").shape))
    step, iters, ok = r.darcy_log()
    assert iters.sum() == 0 and ok.all()
    assert (numpy.abs(r.fluid_cells("v")) < 1.0e-6).all()


def test_pressure_step_drives_flow_down():
    """tests/cfd_tests_darcy.py, "Pressure gradient": p = 1 in the top
    layer: fluid flows towards -z (against the gradient) in every cell and
    not sideways; the first solves need many iterations, later ones few."""
    r, flags = run("darcy_pressure_step", "oracle")
    assert flags == 0
    v = r.fluid_cells("v")
    assert (v[:, :, :, 2] < 0.0).all()
    assert (numpy.abs(v[:, :, :, 0:2]) < 1.0e-7).all()
    step, iters, ok = r.darcy_log()
    assert ok.all() and iters[0] > iters[-1]
