"""Generate the golden fixtures in tests/golden/ (run in a container that
holds the reference sources; the fixtures are committed, the script is the
record of how they were made):

    python tests/golden/make_golden.py <reference checkout>

(the reference checkout may instead be given as $SPHERE_REFERENCE)

1. bin_*.bin: .bin files written by the reference's own python/sphere.py
   (sim.writebin) for seeded scenes built with the reference's own set-up
   helpers.  tests/test_binio.py rebuilds the same scenes with
   sphere_b200.sim and requires byte-identical files, and reads each file
   back through sphere_b200.binio.
2. steps_*.npz: outputs of the reference's own step kernels compiled for
   the CPU (oracle/_ref/libsphere_ref.so) after 1 and 10 steps of small
   seeded scenes.  tests/test_golden_steps.py checks the CPU oracle (and the
   GPU) against them bit for bit.

The reference module is imported with two stand-ins for what this Python
lacks: a stub matplotlib (plotting only) and numpy.random.random_integers
(removed from numpy 2; unused by these scenes).
"""
import importlib.util
import os
import sys
import types

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


class _Stub(types.ModuleType):
    """A module whose every attribute is a do-nothing callable/object."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Noop()


class _Noop(object):
    def __call__(self, *a, **k):
        return _Noop()

    def __getattr__(self, name):
        return _Noop()

    def update(self, *a, **k):
        return None

    def __setitem__(self, key, value):
        pass

    def __getitem__(self, key):
        return _Noop()


def load_reference_sphere(ref_root):
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.collections",
                 "matplotlib.font_manager"):
        sys.modules[name] = _Stub(name)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    # numpy 2 removed these aliases; the reference uses them
    if not hasattr(numpy, "infty"):
        numpy.infty = numpy.inf
    spec = importlib.util.spec_from_file_location(
        "reference_sphere", os.path.join(ref_root, "python", "sphere.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def bin_scenes(S):
    """Seeded scenes built with a sim class S (the reference's or ours)."""
    out = {}
    numpy.random.seed(1)
    s = S(np=40, nw=0, sid="golden_grid")
    s.generateRadii(psd='uni', mean=0.01, variance=0.001)
    s.periodicBoundariesXY()
    s.initRandomGridPos(gridnum=numpy.array([12, 12, 24]))
    s.defaultParams(gamma_n=100.0, mu_s=0.4, mu_d=0.4)
    s.initTemporal(total=0.01, file_dt=0.002)
    out["grid"] = s
    numpy.random.seed(2)
    s = S(np=30, nw=0, sid="golden_consolidate")
    s.generateRadii(psd='logn', mean=0.01, variance=1e-6)
    s.initRandomGridPos(gridnum=numpy.array([10, 10, 20]))
    s.consolidate(normal_stress=2.0e4)
    s.initTemporal(total=0.01, file_dt=0.002)
    out["consolidate"] = s
    numpy.random.seed(3)
    s = S(np=36, nw=0, sid="golden_shear")
    s.generateRadii(psd='uni', mean=0.01, variance=0.001)
    s.periodicBoundariesXY()
    s.initRandomGridPos(gridnum=numpy.array([12, 12, 24]))
    s.consolidate(normal_stress=1.0e4)
    s.shear(shear_strain_rate=0.5)
    s.setYoungsModulus(7.0e9)
    s.initTemporal(total=0.01, file_dt=0.002)
    out["shear"] = s
    numpy.random.seed(4)
    s = S(np=20, nw=0, sid="golden_bonds")
    s.generateRadii(psd='uni', mean=0.01, variance=0.001)
    s.initRandomGridPos(gridnum=numpy.array([10, 10, 20]))
    s.bond(0, 1)
    s.bond(2, 3)
    s.bond(4, 7)
    s.uniaxialStrainRate(wvel=-0.002)
    s.initTemporal(total=0.01, file_dt=0.002)
    out["bonds"] = s
    numpy.random.seed(5)
    s = S(np=24, nw=0, sid="golden_darcy", fluid=True)
    s.generateRadii(psd='uni', mean=0.01, variance=0.001)
    s.periodicBoundariesXY()
    s.initRandomGridPos(gridnum=numpy.array([8, 8, 16]))
    s.consolidate(normal_stress=1.0e4)
    s.initFluid(mu=1.0e-3, rho=1.0e3, p=1.0e3, hydrostatic=True, cfd_solver=1)
    s.setFluidBottomNoFlow()
    s.setFluidTopFixedFlux(2.0e-5)
    s.setFluidXNoFlow()
    s.setPermeabilityPrefactor(1.0e-9, verbose=False)
    s.setFluidCompressibility(1.0e-8)
    s.setFluidPressureModulation(A=100.0, f=2.0, phi=0.25)
    s.setDEMstepsPerCFDstep(3)
    s.setTolerance(1.0e-4)
    s.setMaxIterations(500)
    s.p_f_constant[0, 1, 2] = 1
    s.dphi[:, :, 1] = 0.5
    s.v_f[:, :, :, 2] = -1.0e-3
    s.f_p[:, 2] = 0.25
    s.initTemporal(total=0.01, file_dt=0.002)
    out["darcy"] = s
    numpy.random.seed(6)
    s = S(np=18, nw=0, sid="golden_ns", fluid=True)
    s.generateRadii(psd='uni', mean=0.01, variance=0.001)
    s.periodicBoundariesXY()
    s.initRandomGridPos(gridnum=numpy.array([8, 8, 16]))
    s.consolidate(normal_stress=1.0e4)
    s.initFluid(mu=1.0e-3, rho=1.0e3, p=2.0e3, hydrostatic=True, cfd_solver=0)
    s.setFluidBottomNoFlow()
    s.setFluidTopFixedPressure()
    s.setFluidPressureModulation(A=50.0, f=1.0, phi=0.5)
    s.setGamma(0.1)
    s.setTheta(0.9)
    s.setBeta(0.2)
    s.setTolerance(1.0e-5)
    s.setMaxIterations(800)
    s.setDEMstepsPerCFDstep(2)
    s.p_f_constant[1, 0, 1] = 1
    s.dphi[:, :, 1] = 0.25
    s.v_f[:, :, :, 0] = 2.0e-3
    s.f_d[:, 0] = 0.5
    s.f_p[:, 1] = -0.25
    s.f_v[:, 2] = 0.125
    s.f_sum[:] = s.f_d + s.f_p + s.f_v
    s.initTemporal(total=0.01, file_dt=0.002)
    out["ns"] = s
    return out


def step_scenes():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import cases
    return {name: cases.make(name)[0] for name in
            ("periodic_xy_wall_stress", "walls_all_sides", "contact_model_1", "bonds_breaking",
             "shear_stress_wall")}


STEP_FIELDS = ["x", "vel", "angvel", "angpos", "xyzsum", "force", "torque", "es", "ev", "es_dot",
               "ev_dot", "p", "contacts", "delta_t", "perm", "bonds", "bonds_delta", "bonds_omega"]


class _IndexArray(numpy.ndarray):
    """A one-element count array usable as an index, as numpy 1.x allowed
    (the reference writes range(self.np) with self.np = array([n]))."""

    def __index__(self):
        return int(numpy.asarray(self).reshape(-1)[0])


def ref_sim_factory(ref):
    def make(**kw):
        s = ref.sim(**kw)
        s.np = s.np.view(_IndexArray)
        s.nb0 = s.nb0.view(_IndexArray)
        return s
    return make


def main(ref_root):
    ref = load_reference_sphere(ref_root)
    for name, s in bin_scenes(ref_sim_factory(ref)).items():
        s.writebin(folder=HERE, verbose=False)
        os.replace(os.path.join(HERE, s.sid + ".bin"), os.path.join(HERE, "bin_%s.bin" % name))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    for name, s in step_scenes().items():
        run = O.CpuRun(s, "ref")
        rec = {}
        for k in (1, 10):
            run.step(k - (1 if k == 10 else 0))
            for f in STEP_FIELDS:
                rec["%s_%d" % (f, k)] = numpy.array(getattr(run, f))
            rec["walls_nx_%d" % k] = numpy.array([list(run.box.walls.nx[w]) for w in range(6)])
            rec["walls_mvfd_%d" % k] = numpy.array([list(run.box.walls.mvfd[w]) for w in range(6)])
        numpy.savez_compressed(os.path.join(HERE, "steps_%s.npz" % name), **rec)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPHERE_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set SPHERE_REFERENCE)")
    main(ref)
