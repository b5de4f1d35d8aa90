"""Seeded Darcy-coupled scenes (fluid == 1, cfd_solver == 1) shared by the
CPU and GPU parity tests.

Two pure-fluid boxes follow the reference's own Darcy checks
(tests/cfd_tests_darcy.py): no forcing, and a pressure step at the top.
The sphere packs each exercise a part of the Darcy step (src/device.cu:
1891-2419): the pressure force with buoyancy, the porosity estimate and its
change, the top wall's cell index (wall0_iz, taken from the host's copy of
the wall, refreshed at outputs), the file clock that keeps dphi on output
steps, every boundary code (fixed pressure, no flow, periodic, flux), the
frictionless y sides of periodic == 2, top-pressure modulation, cells of
constant pressure, ndem > 1 and a solve that runs out of iterations.
"""
import numpy

import sphere_b200
from sphere_b200 import scenes


def fluid_box(p_top=0.0, dt=1.0e-7, file_every=0.99):
    """The 4 x 3 x 4 cell box of the reference's Darcy test, no spheres."""
    s = sphere_b200.sim(np=0, nd=3, nw=0, sid="cfdtest", fluid=True)
    s.defaultParams()
    s.defineWorldBoundaries([0.4, 0.3, 0.4], dx=0.1)
    s.initFluid(cfd_solver=1)
    s.initTemporal(total=0.2, file_dt=0.01, dt=dt)
    s.time_file_dt[0] = s.time_dt[0] * file_every
    s.p_f[:, :, -1] = p_top
    return s


def big_fluid_box():
    """A pure-fluid box of 46 x 45 x 40 = 82,800 cells: more cells than one
    Jacobi launch has threads on a B200 (148 blocks of 512), so that threads
    take their cells in turn; no-flow x sides and a fixed flux at the
    bottom, a pressure step at the top."""
    s = sphere_b200.sim(np=0, nd=3, nw=0, sid="cfdbig", fluid=True)
    s.defaultParams()
    s.defineWorldBoundaries([4.6, 4.5, 4.0], dx=0.1)
    s.initFluid(cfd_solver=1)
    s.initTemporal(total=0.2, file_dt=0.01, dt=1.0e-6)
    s.time_file_dt[0] = s.time_dt[0] * 0.99
    s.setFluidXNoFlow()
    s.setFluidBottomFixedFlux(1.0e-5)
    s.p_f[:, :, -1] = 1.0
    return s


fluid_pack = scenes.darcy_pack


def make(name):
    """Return (sim, steps) for a named Darcy case."""
    if name == "darcy_still_fluid":
        return fluid_box(), 10
    if name == "darcy_pressure_step":
        return fluid_box(p_top=1.0, dt=1.0e-6), 30
    if name == "darcy_pack_wall":
        return fluid_pack(300, 21), 20
    if name == "darcy_pack_bcs":
        s = fluid_pack(300, 22, periodic=0, nw=0, wmode=0)
        s.setFluidBottomNoFlow()
        s.setFluidTopFixedFlux(1.0e-4)
        s.setFluidXNoFlow()
        s.setFluidYFixedPressure()
        rng = numpy.random.default_rng(22)
        s.p_f_constant[tuple(rng.integers(0, s.num[d], 6) for d in range(3))] = 1
        s.setDEMstepsPerCFDstep(2)
        return s, 20
    if name == "darcy_pack_periodic2":
        s = fluid_pack(300, 23, periodic=2, wmode=2, wvel=-0.01)
        s.setFluidYNoFlow()
        return s, 20
    if name == "darcy_pack_modulated":
        s = fluid_pack(300, 24)
        s.setFluidPressureModulation(A=2.0e3, f=5.0e3, phi=0.3)
        return s, 20
    if name == "darcy_pack_maxiter":
        s = fluid_pack(200, 25, beta_f=4.5e-10)
        s.setTolerance(1.0e-12)
        s.setMaxIterations(7)
        return s, 10
    if name == "darcy_pack_top_noflow":
        s = fluid_pack(300, 26)
        s.setFluidTopNoFlow()
        s.setFluidBottomFixedFlux(-2.0e-4)
        return s, 20
    raise KeyError(name)


CASES = ["darcy_still_fluid", "darcy_pressure_step", "darcy_pack_wall", "darcy_pack_bcs",
         "darcy_pack_periodic2", "darcy_pack_modulated", "darcy_pack_maxiter",
         "darcy_pack_top_noflow"]
