"""The reference's known-answer tests for the DEM step, as scenarios.

Restated from the reference's tests/contactmodel.py, contactmodel_young.py,
contactmodel_wall.py and contactmodel_wall_young.py: two unit spheres (or
one sphere and the floor) in a 10 m box, checked after 0.1-1.0 s of
simulated time against physical invariants with the reference's
tolerances (pytestutils.compareFloats: relative 1e-3 by default).

Each scenario returns (sim, check) where check(orig, after) asserts.
"""
import numpy

from sphere_b200.sim import sim


def rel_close(first, second, tol=1e-3):
    assert abs((first - second) / first) < tol, (first, second, abs((first - second) / first))


def _pair(radii, x1z, young, **kw):
    s = sim(np=2, sid='contactmodeltest')
    s.radius[:] = radii
    s.x[0, :] = [5.0, 5.0, 2.0]
    s.x[1, :] = [5.0, 5.0, x1z]
    s.vel[0, 2] = 1.0
    for k, v in kw.items():
        getattr(s, k)[0] = v
    s.defineWorldBoundaries(L=[10, 10, 10])
    if young:
        s.setYoungsModulus(7.0e9)
    s.initTemporal(total=0.1, file_dt=0.01)
    return s


def _oblique(young, **kw):
    s = _pair([1.0, 1.0], 4.05, young)
    s.vel[0, 0] = 1.0
    for k, v in kw.items():
        getattr(s, k)[0] = v
    return s


def _wall(young, vx=0.0, total=1.0, gamma_wn=0.0, gamma_wt=0.0):
    s = sim(np=1, nw=0, sid='contactmodeltest')
    s.radius[:] = 1.0
    s.x[0, :] = [5.0, 5.0, 1.05]
    s.vel[0, 2] = -0.1
    s.vel[0, 0] = vx
    s.defineWorldBoundaries(L=[10, 10, 10])
    s.gamma_wn[0] = gamma_wn
    s.gamma_wt[0] = gamma_wt
    if young:
        s.setYoungsModulus(7.0e9)
    s.initTemporal(total=total, file_dt=0.01)
    return s


def scenarios(young=False):
    out = {}

    # elastic normal collisions (contactmodel.py:15-70)
    def chk(o, a):
        rel_close(o.vel[0, 2], a.vel[1, 2])
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy())
    out["elastic_equal"] = (_pair([1.0, 1.0], 4.05, young), chk)

    def chk_ke(o, a):
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy())
    out["elastic_big_small"] = (_pair([2.0, 1.0], 5.05, young), chk_ke)
    out["elastic_small_big"] = (_pair([1.0, 2.0], 5.05, young), chk_ke)

    # viscoelastic normal collisions (contactmodel.py:74-140)
    def chk_visc(o, a):
        assert o.vel[0, 2] > a.vel[1, 2]
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy() + a.totalViscousEnergy(), 0.05)
    out["viscous_equal"] = (_pair([1.0, 1.0], 4.05, young, gamma_n=1.0e6), chk_visc)

    def chk_visc2(o, a):
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy() + a.totalViscousEnergy(), 0.05)
    out["viscous_big_small"] = (_pair([2.0, 1.0], 5.05, young, gamma_n=1.0e6), chk_visc2)
    out["viscous_small_big"] = (_pair([1.0, 2.0], 5.05, young, gamma_n=1.0e6), chk_visc2)

    # oblique collisions (contactmodel.py:146-230)
    def chk_noslip(o, a):
        assert (a.angvel[:, 1] < 0.0).all()
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy() + a.totalRotationalEnergy(), 0.05)
    out["oblique_noslip"] = (_oblique(young, mu_s=1e9, mu_d=1e9), chk_noslip)

    def chk_slip(o, a):
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy() + a.totalRotationalEnergy() +
                  a.totalFrictionalEnergy(), 0.05)
        assert (a.angvel[:, 1] < 0.0).all()
        assert a.totalFrictionalEnergy() > 0.0
    out["oblique_slip"] = (_oblique(young, mu_s=0.3, mu_d=0.3), chk_slip)

    def chk_slip_visc(o, a):
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy() + a.totalRotationalEnergy() +
                  a.totalFrictionalEnergy() + a.totalViscousEnergy(), 0.05)
        assert (a.angvel[:, 1] < 0.0).all()
        assert a.totalFrictionalEnergy() > 0.0
    out["oblique_slip_viscous"] = (_oblique(young, mu_s=0.3, mu_d=0.3, gamma_t=1.0e3),
                                   chk_slip_visc)

    # walls (contactmodel_wall.py:13-107)
    def chk_wall(o, a):
        rel_close(a.vel[0, 2], 0.1)
        rel_close(o.totalKineticEnergy(), a.totalKineticEnergy())
    out["wall_elastic"] = (_wall(young), chk_wall)
    out["wall_oblique"] = (_wall(young, vx=0.1, total=0.3), chk_ke)

    def chk_wall_visc(o, a):
        assert o.energy('kin') > a.energy('kin')
        rel_close(o.energy('kin'), a.energy('kin') + a.energy('visc_n'), 0.05)
    out["wall_viscous"] = (_wall(young, gamma_wn=1.0e6), chk_wall_visc)

    def chk_wall_oblique_visc(o, a):
        assert o.energy('kin') > a.energy('kin')
        assert a.angvel[0, 0] == 0.0 and a.angvel[0, 1] > 0.0 and a.angvel[0, 2] == 0.0
    out["wall_oblique_viscous"] = (_wall(young, vx=0.1, gamma_wn=1.0e6, gamma_wt=1.0e6),
                                   chk_wall_oblique_visc)
    return out


def n_steps(s):
    """Iterations of the reference loop `while (t <= total) { step; t += dt }`
    (src/device.cu:1031, 2536)."""
    t = float(s.time_current[0])
    total = float(s.time_total[0])
    dt = float(s.time_dt[0])
    k = 0
    while t <= total:
        t += dt
        k += 1
    return k
