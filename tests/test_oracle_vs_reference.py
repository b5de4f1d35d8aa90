"""The C oracle against the reference's own kernels run on the CPU.

oracle/_ref/libsphere_ref.so is the reference's src/*.cuh step kernels
compiled for the CPU (oracle/ref_emu); oracle/_build/libsphere_oracle.so is
this project's restatement.  On every parity case they must agree bit for
bit: positions, velocities, forces, torques, energies, contact lists,
tangential histories, the sorted permutation and the walls.
"""
import os

import numpy
import pytest

import cases
import oracle as O

FIELDS = ["x", "vel", "angvel", "angpos", "xyzsum", "force", "torque", "es", "ev", "es_dot",
          "ev_dot", "p", "contacts", "delta_t", "perm", "cell_id", "bonds", "bonds_delta",
          "bonds_omega"]

needs_ref = pytest.mark.skipif(not O.available("ref") and O.reference_root() is None,
                               reason="reference sources unavailable to build oracle/_ref")


def _same(a, b):
    return numpy.array_equal(a, b) or (a.dtype.kind == "f" and numpy.array_equal(a, b, equal_nan=True))


@needs_ref
@pytest.mark.parametrize("name", [c for c in cases.CASES if cases.make(c)[1]])
def test_oracle_matches_reference_kernels(name):
    if not O.available("ref"):
        O.build()
    s, ref_ok, steps = cases.make(name)
    a = O.CpuRun(s, "oracle")
    b = O.CpuRun(s, "ref")
    for chunk in range(2):
        a.step(steps // 2)
        b.step(steps // 2)
        for f in FIELDS:
            A, B = getattr(a, f), getattr(b, f)
            assert _same(A, B), "%s differs after %d steps (max %g)" % (
                f, (chunk + 1) * steps // 2,
                float(numpy.nanmax(numpy.abs(A.astype(float) - B.astype(float)))))
        live = a.contacts != s.np[0]
        assert numpy.array_equal(a.distmod[live], b.distmod[live])
        for w in range(int(s.nw[0])):
            assert list(a.box.walls.nx[w]) == list(b.box.walls.nx[w])
            assert list(a.box.walls.mvfd[w]) == list(b.box.walls.mvfd[w])
        assert a.box.grid.L[2] == b.box.grid.L[2]
        assert a.box.t_current == b.box.t_current
    assert int((a.contacts != s.np[0]).sum()) > 0 or s.contactmodel[0] == 1


# the reference's own output files (its checkout's output/ directory)
FIXTURES = os.path.join(O.reference_root() or "", "output")


@needs_ref
@pytest.mark.skipif(O.reference_root() is None or not os.path.isdir(FIXTURES),
                    reason="the reference's output fixtures are not present")
@pytest.mark.parametrize("fname,steps", [("cube-init.output00029.bin", 20),
                                         ("init-1e4.output00199.bin", 6)])
def test_oracle_matches_reference_kernels_on_its_fixtures(fname, steps):
    """The reference's own output files as inputs (output/cube-init: 1,000
    spheres in a 3 x 3 x 112 periodic grid, the smallest grid with periodic
    images on both sides; output/init-1e4: 10,000 settled spheres)."""
    from sphere_b200 import sim
    if not O.available("ref"):
        O.build()
    s = sim()
    s.readbin(os.path.join(FIXTURES, fname), verbose=False)
    a = O.CpuRun(s, "oracle")
    b = O.CpuRun(s, "ref")
    for chunk in range(2):
        a.step(steps // 2)
        b.step(steps // 2)
        for f in FIELDS:
            A, B = getattr(a, f), getattr(b, f)
            assert _same(A, B), "%s differs after %d steps" % (f, (chunk + 1) * steps // 2)
    assert int((a.contacts != s.np[0]).sum()) > 0


def test_capillary_case_exercises_the_capillary_law():
    """The capillary case is only a check of capillaryCohesion_exp if that
    law carries a real share of the forces: one step with kappa = 0 must
    differ from the case's forces by more than 10 % (relative L2)."""
    import copy
    s, _ok, _steps = cases.make("capillary_cohesion")
    a = O.CpuRun(s, "oracle")
    a.step(1)
    s0 = copy.deepcopy(s)
    s0.kappa[0] = 0.0
    b = O.CpuRun(s0, "oracle")
    b.step(1)
    rel = numpy.linalg.norm(a.force - b.force) / numpy.linalg.norm(a.force)
    assert rel > 0.1, rel
