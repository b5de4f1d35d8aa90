"""Drop-in replacement for the DEM part of python/sphere.py's ``sim`` class.

Attribute names, shapes and dtypes follow python/sphere.py:57-454, the set-up
helpers keep their names and argument meanings (python/sphere.py:795-4480),
and files keep the reference's paths: ``<root>/input/<sid>.bin`` and
``<root>/output/<sid>.outputNNNNN.bin`` + ``<sid>.status.dat`` where the
reference's scripts use ``root = '..'``.  What changes is ``run()``: instead
of executing the ``sphere`` binary (python/sphere.py:4482-4540) it steps the
simulation in-process on a B200 through the C ABI of include/sphere_b200.h.
Fluid coupling, plotting and VTK output are outside this package.
"""
import math
import os
import sys

import numpy

from . import binio

VERSION = binio.VERSION


def default_root():
    """Folder holding input/ and output/ ('..' as in the reference scripts,
    or $SPHERE_ROOT)."""
    return os.environ.get("SPHERE_ROOT", "..")


def V_sphere(r):
    """Volume of a sphere of radius r (python/sphere.py:7760)."""
    return 4.0 / 3.0 * math.pi * r ** 3.0


def _seqsum(a):
    """Left-to-right sum, as the reference's Python loops accumulate."""
    a = numpy.asarray(a, dtype=numpy.float64).ravel()
    return float(numpy.cumsum(a)[-1]) if a.size else 0.0


class sim(object):
    """DEM simulation object (python/sphere.py:33 ``class sim``)."""

    def __init__(self, sid='unnamed', np=0, nd=3, nw=0, fluid=False, cfd_solver=0):
        self.version = numpy.ones(1, dtype=numpy.float64) * VERSION
        self.nd = numpy.ones(1, dtype=numpy.int32) * int(nd)
        self.np = numpy.ones(1, dtype=numpy.uint32) * int(np)
        self.sid = sid
        self.time_dt = numpy.zeros(1, dtype=numpy.float64)
        self.time_current = numpy.zeros(1, dtype=numpy.float64)
        self.time_total = numpy.zeros(1, dtype=numpy.float64)
        self.time_file_dt = numpy.zeros(1, dtype=numpy.float64)
        self.time_step_count = numpy.zeros(1, dtype=numpy.uint32)
        self.origo = numpy.zeros(self.nd, dtype=numpy.float64)
        self.L = numpy.zeros(self.nd, dtype=numpy.float64)
        self.num = numpy.zeros(self.nd, dtype=numpy.uint32)
        self.periodic = numpy.zeros(1, dtype=numpy.uint32)
        self.adaptive = numpy.zeros(1, dtype=numpy.uint32)
        n = int(np)
        d = int(nd)
        self.x = numpy.zeros((n, d), dtype=numpy.float64)
        self.radius = numpy.ones(n, dtype=numpy.float64)
        self.xyzsum = numpy.zeros((n, 3), dtype=numpy.float64)
        self.vel = numpy.zeros((n, d), dtype=numpy.float64)
        self.fixvel = numpy.zeros(n, dtype=numpy.float64)
        self.force = numpy.zeros((n, d), dtype=numpy.float64)
        self.angpos = numpy.zeros((n, d), dtype=numpy.float64)
        self.angvel = numpy.zeros((n, d), dtype=numpy.float64)
        self.torque = numpy.zeros((n, d), dtype=numpy.float64)
        self.es_dot = numpy.zeros(n, dtype=numpy.float64)
        self.es = numpy.zeros(n, dtype=numpy.float64)
        self.ev_dot = numpy.zeros(n, dtype=numpy.float64)
        self.ev = numpy.zeros(n, dtype=numpy.float64)
        self.p = numpy.zeros(n, dtype=numpy.float64)
        self.g = numpy.array([0.0, 0.0, 0.0], dtype=numpy.float64)
        self.k_n = numpy.ones(1, dtype=numpy.float64) * 1.16e9
        self.k_t = numpy.ones(1, dtype=numpy.float64) * 1.16e9
        self.k_r = numpy.zeros(1, dtype=numpy.float64)
        self.E = numpy.zeros(1, dtype=numpy.float64)
        self.gamma_n = numpy.zeros(1, dtype=numpy.float64)
        self.gamma_t = numpy.zeros(1, dtype=numpy.float64)
        self.gamma_r = numpy.zeros(1, dtype=numpy.float64)
        self.mu_s = numpy.ones(1, dtype=numpy.float64) * 0.5
        self.mu_d = numpy.ones(1, dtype=numpy.float64) * 0.5
        self.mu_r = numpy.zeros(1, dtype=numpy.float64)
        self.gamma_wn = numpy.ones(1, dtype=numpy.float64) * 1.0e3
        self.gamma_wt = numpy.zeros(1, dtype=numpy.float64)
        self.mu_ws = numpy.ones(1, dtype=numpy.float64) * 0.5
        self.mu_wd = numpy.ones(1, dtype=numpy.float64) * 0.5
        self.rho = numpy.ones(1, dtype=numpy.float64) * 2600.0
        self.contactmodel = numpy.ones(1, dtype=numpy.uint32) * 2
        self.kappa = numpy.zeros(1, dtype=numpy.float64)
        self.db = numpy.zeros(1, dtype=numpy.float64)
        self.V_b = numpy.zeros(1, dtype=numpy.float64)
        self.nw = numpy.ones(1, dtype=numpy.uint32) * int(nw)
        w = int(nw)
        self.wmode = numpy.zeros(w, dtype=numpy.int32)
        self.w_n = numpy.zeros((w, d), dtype=numpy.float64)
        for i, (axis, sign) in enumerate(((2, -1.0), (0, -1.0), (0, 1.0), (1, -1.0), (1, 1.0))):
            if w > i:
                self.w_n[i, axis] = sign
        self.w_x = numpy.ones(w, dtype=numpy.float64)
        self.w_m = numpy.zeros(w, dtype=numpy.float64)
        self.w_vel = numpy.zeros(w, dtype=numpy.float64)
        self.w_force = numpy.zeros(w, dtype=numpy.float64)
        self.w_sigma0 = numpy.zeros(w, dtype=numpy.float64)
        self.w_sigma0_A = numpy.zeros(1, dtype=numpy.float64)
        self.w_sigma0_f = numpy.zeros(1, dtype=numpy.float64)
        self.w_tau_x = numpy.zeros(1, dtype=numpy.float64)
        self.lambda_bar = numpy.ones(1, dtype=numpy.float64)
        self.nb0 = numpy.zeros(1, dtype=numpy.uint32)
        self.sigma_b = numpy.ones(1, dtype=numpy.float64) * numpy.inf
        self.tau_b = numpy.ones(1, dtype=numpy.float64) * numpy.inf
        self.bonds = numpy.zeros((0, 2), dtype=numpy.uint32)
        self.bonds_delta_n = numpy.zeros(0, dtype=numpy.float64)
        self.bonds_delta_t = numpy.zeros((0, d), dtype=numpy.float64)
        self.bonds_omega_n = numpy.zeros(0, dtype=numpy.float64)
        self.bonds_omega_t = numpy.zeros((0, d), dtype=numpy.float64)
        self.fluid = False
        self.color = numpy.zeros(n, dtype=numpy.int32)
        if fluid:
            # the fluid fields (python/sphere.py:310-440): those of the Darcy
            # solver, or of the Navier-Stokes solver (cfd_solver 0), whose
            # fields and .bin block are kept but whose solver is not built
            self.fluid = True
            self.cfd_solver = numpy.ones(1, dtype=numpy.int32) * int(cfd_solver)
            if int(cfd_solver) == 0:
                self._ns_defaults(0.0)
            else:
                self._darcy_defaults(0.0)

    # ------------------------------------------------------------- fluid
    def _ns_defaults(self, p):
        """The Navier-Stokes fields with their defaults on the current grid
        (python/sphere.py:3418-3489 initFluid with cfd_solver 0): the
        cell fields and boundary codes shared with the Darcy solver, the
        solver parameters gamma, theta, beta, tolerance, maxiter, ndem,
        c_phi, c_v, dt_dem_fac and the per-sphere drag, pressure, viscous and
        total fluid forces."""
        num = tuple(int(v) for v in self.num)
        n, nd = int(self.np[0]), int(self.nd[0])
        self.mu = numpy.zeros(1, dtype=numpy.float64)
        self.rho_f = numpy.ones(1, dtype=numpy.float64) * 1.0e3
        self.p_f = numpy.ones(num, dtype=numpy.float64) * p
        self.v_f = numpy.zeros(num + (nd,), dtype=numpy.float64)
        self.phi = numpy.ones(num, dtype=numpy.float64)
        self.dphi = numpy.zeros(num, dtype=numpy.float64)
        self.p_mod_A = numpy.zeros(1, dtype=numpy.float64)
        self.p_mod_f = numpy.zeros(1, dtype=numpy.float64)
        self.p_mod_phi = numpy.zeros(1, dtype=numpy.float64)
        self.bc_bot = numpy.zeros(1, dtype=numpy.int32)
        self.bc_top = numpy.zeros(1, dtype=numpy.int32)
        self.free_slip_bot = numpy.ones(1, dtype=numpy.int32)
        self.free_slip_top = numpy.ones(1, dtype=numpy.int32)
        self.bc_bot_flux = numpy.zeros(1, dtype=numpy.float64)
        self.bc_top_flux = numpy.zeros(1, dtype=numpy.float64)
        self.p_f_constant = numpy.zeros(num, dtype=numpy.int32)
        self.gamma = numpy.array(0.0)
        self.theta = numpy.array(1.0)
        self.beta = numpy.array(0.0)
        self.tolerance = numpy.array(1.0e-3)
        self.maxiter = numpy.array(1e4)
        self.ndem = numpy.array(1)
        self.c_phi = numpy.ones(1, dtype=numpy.float64)
        self.c_v = numpy.ones(1, dtype=numpy.float64)
        self.dt_dem_fac = numpy.ones(1, dtype=numpy.float64)
        for name in ("f_d", "f_p", "f_v", "f_sum"):
            setattr(self, name, numpy.zeros((n, nd), dtype=numpy.float64))

    def _darcy_defaults(self, p):
        """The Darcy fields with their defaults on the current grid."""
        num = tuple(int(v) for v in self.num)
        n = int(self.np[0])
        self.mu = numpy.zeros(1, dtype=numpy.float64)
        self.rho_f = numpy.ones(1, dtype=numpy.float64) * 1.0e3
        self.p_f = numpy.ones(num, dtype=numpy.float64) * p
        self.v_f = numpy.zeros(num + (int(self.nd[0]),), dtype=numpy.float64)
        self.phi = numpy.ones(num, dtype=numpy.float64)
        self.dphi = numpy.zeros(num, dtype=numpy.float64)
        self.p_mod_A = numpy.zeros(1, dtype=numpy.float64)
        self.p_mod_f = numpy.zeros(1, dtype=numpy.float64)
        self.p_mod_phi = numpy.zeros(1, dtype=numpy.float64)
        for name in ("bc_xn", "bc_xp", "bc_yn", "bc_yp"):
            setattr(self, name, numpy.ones(1, dtype=numpy.int32) * 2)
        self.bc_bot = numpy.zeros(1, dtype=numpy.int32)
        self.bc_top = numpy.zeros(1, dtype=numpy.int32)
        self.free_slip_bot = numpy.ones(1, dtype=numpy.int32)
        self.free_slip_top = numpy.ones(1, dtype=numpy.int32)
        self.bc_bot_flux = numpy.zeros(1, dtype=numpy.float64)
        self.bc_top_flux = numpy.zeros(1, dtype=numpy.float64)
        self.p_f_constant = numpy.zeros(num, dtype=numpy.int32)
        self.tolerance = numpy.array(1.0e-3)
        self.maxiter = numpy.array(1e4)
        self.ndem = numpy.array(1)
        self.c_phi = numpy.ones(1, dtype=numpy.float64)
        self.f_p = numpy.zeros((n, int(self.nd[0])), dtype=numpy.float64)
        self.beta_f = numpy.ones(1, dtype=numpy.float64) * 4.5e-10
        self.k_c = numpy.ones(1, dtype=numpy.float64) * 4.6e-10

    def initFluid(self, mu=8.9e-4, rho=1.0e3, p=0.0, hydrostatic=False, cfd_solver=0):
        """Fluid arrays and viscosity on the current grid
        (python/sphere.py:3395).  cfd_solver 1: the Darcy solver, which
        run() steps; cfd_solver 0: the Navier-Stokes solver's fields, which
        can be set up, written and read (its .bin block), but run() refuses
        them: that solver is not built.  With hydrostatic=True the cells
        below the top wall (or below the top of the grid) get the hydrostatic
        pressure of the fluid column above them, p at the top."""
        if int(cfd_solver) not in (0, 1):
            raise Exception('Value of cfd_solver not understood (%s)' % cfd_solver)
        self.fluid = True
        self.cfd_solver = numpy.ones(1, dtype=numpy.int32) * int(cfd_solver)
        if int(cfd_solver) == 0:
            self._ns_defaults(p)
        else:
            self._darcy_defaults(p)
        self.mu = numpy.ones(1, dtype=numpy.float64) * mu
        self.rho_f = numpy.ones(1, dtype=numpy.float64) * rho
        if hydrostatic:
            dz = self.L[2] / self.num[2]
            if int(self.nw[0]) == 1:
                wall0_iz = int(self.w_x[0] / (self.L[2] / self.num[2]))
                self.p_f[:, :, wall0_iz:] = p
                top = self.w_x[0]
                layers = numpy.arange(wall0_iz - 1)
            else:
                top = self.L[2]
                layers = numpy.arange(self.num[2] - 1)
            for iz in layers:
                depth = top - (dz * iz + 0.5 * dz)
                self.p_f[:, :, iz] = p + (depth - dz) * rho * -self.g[2]

    def _check_darcy(self, what):
        if not self.fluid or int(numpy.asarray(self.cfd_solver).ravel()[0]) != 1:
            raise Exception(what + '() is only relevant for the Darcy solver (cfd_solver = 1)')

    # boundary conditions of the fluid (python/sphere.py:3527-3685):
    # 0 fixed pressure, 1 no flow, 2 periodic (x, y) / no slip (z), 4 flux
    def setFluidBottomNoFlow(self):
        self.bc_bot[0] = 1

    def setFluidBottomNoFlowNoSlip(self):
        self.bc_bot[0] = 2

    def setFluidBottomFixedPressure(self):
        self.bc_bot[0] = 0

    def setFluidBottomFixedFlux(self, specific_flux):
        self.bc_bot[0] = 4
        self.bc_bot_flux[0] = specific_flux

    def setFluidTopNoFlow(self):
        self.bc_top[0] = 1

    def setFluidTopNoFlowNoSlip(self):
        self.bc_top[0] = 2

    def setFluidTopFixedPressure(self):
        self.bc_top[0] = 0

    def setFluidTopFixedFlux(self, specific_flux):
        self.bc_top[0] = 4
        self.bc_top_flux[0] = specific_flux

    def _sides(self, names, code):
        for name in names:
            getattr(self, name)[0] = code

    def setFluidXFixedPressure(self):
        self._sides(("bc_xn", "bc_xp"), 0)

    def setFluidXNoFlow(self):
        self._sides(("bc_xn", "bc_xp"), 1)

    def setFluidXPeriodic(self):
        self._sides(("bc_xn", "bc_xp"), 2)

    def setFluidYFixedPressure(self):
        self._sides(("bc_yn", "bc_yp"), 0)

    def setFluidYNoFlow(self):
        self._sides(("bc_yn", "bc_yp"), 1)

    def setFluidYPeriodic(self):
        self._sides(("bc_yn", "bc_yp"), 2)

    def setPermeabilityPrefactor(self, k_c, verbose=False):
        """Kozeny-Carman prefactor k_c of k = k_c phi^3 / (1 - phi)^2
        (python/sphere.py:3701)."""
        self._check_darcy('setPermeabilityPrefactor')
        self.k_c[0] = k_c

    def setPermeabilityGrainSize(self, verbose=False):
        """k_c from the mean grain diameter, d^2 / 180 (python/sphere.py:3687)."""
        self.setPermeabilityPrefactor(numpy.mean(self.radius * 2.0) ** 2.0 / 180.0, verbose)

    def setFluidCompressibility(self, beta_f):
        self._check_darcy('setFluidCompressibility')
        self.beta_f[0] = beta_f

    def setFluidViscosity(self, mu):
        self.mu[0] = mu

    def setFluidDensity(self, rho_f):
        self.rho_f[0] = rho_f

    def setFluidPressureModulation(self, A, f, phi=0.0, plot=False):
        """Top pressure p_top + A sin(2 pi f t + phi) (python/sphere.py:6219)."""
        self.p_mod_A[0] = A
        self.p_mod_f[0] = f
        self.p_mod_phi[0] = phi

    def disableFluidPressureModulation(self):
        self.setFluidPressureModulation(A=0.0, f=0.0)

    # the Navier-Stokes solver's parameters (python/sphere.py:6294-6352)
    def setGamma(self, gamma):
        self.gamma = numpy.asarray(gamma)

    def setTheta(self, theta):
        self.theta = numpy.asarray(theta)

    def setBeta(self, beta):
        self.beta = numpy.asarray(beta)

    def setTolerance(self, tolerance):
        self.tolerance = numpy.asarray(tolerance)

    def setMaxIterations(self, maxiter):
        self.maxiter = numpy.asarray(maxiter)

    def setDEMstepsPerCFDstep(self, ndem):
        self.ndem = numpy.asarray(ndem)

    def findPermeabilities(self):
        """Cell permeabilities from the porosities as the solver finds them
        (src/darcy.cuh:1485-1532)."""
        self._check_darcy('findPermeabilities')
        phi = numpy.minimum(numpy.asarray(self.phi, dtype=numpy.float64), 0.9999)
        self.k = numpy.minimum(2.7e-10, self.k_c * phi ** 3 / (1.0 - phi) ** 2)
        return self.k

    # ------------------------------------------------------------ identity
    def id(self, sid=''):
        if sid == '':
            return self.sid
        self.sid = sid

    def idAppend(self, string):
        self.sid += string

    # ----------------------------------------------------------- particles
    def addParticle(self, x, radius, xyzsum=numpy.zeros(3), vel=numpy.zeros(3),
                    fixvel=numpy.zeros(1), force=numpy.zeros(3), angpos=numpy.zeros(3),
                    angvel=numpy.zeros(3), torque=numpy.zeros(3), es_dot=numpy.zeros(1),
                    es=numpy.zeros(1), ev_dot=numpy.zeros(1), ev=numpy.zeros(1),
                    p=numpy.zeros(1), color=0):
        """Append one particle (python/sphere.py:821)."""
        self.np = self.np + 1
        self.x = numpy.append(self.x, [x], axis=0)
        self.radius = numpy.append(self.radius, radius)
        self.vel = numpy.append(self.vel, [vel], axis=0)
        self.xyzsum = numpy.append(self.xyzsum, [xyzsum], axis=0)
        self.fixvel = numpy.append(self.fixvel, fixvel)
        self.force = numpy.append(self.force, [force], axis=0)
        self.angpos = numpy.append(self.angpos, [angpos], axis=0)
        self.angvel = numpy.append(self.angvel, [angvel], axis=0)
        self.torque = numpy.append(self.torque, [torque], axis=0)
        self.es_dot = numpy.append(self.es_dot, es_dot)
        self.es = numpy.append(self.es, es)
        self.ev_dot = numpy.append(self.ev_dot, ev_dot)
        self.ev = numpy.append(self.ev, ev)
        self.p = numpy.append(self.p, p)
        self.color = numpy.append(self.color, color)
        if self.fluid:
            self.f_p = numpy.append(self.f_p, [numpy.zeros(3)], axis=0)

    _PER_PARTICLE = ("x", "radius", "vel", "xyzsum", "fixvel", "force", "angpos", "angvel",
                     "torque", "es_dot", "es", "ev_dot", "ev", "p", "color")

    def deleteParticle(self, i):
        """Delete particle(s) i (python/sphere.py:892)."""
        if isinstance(i, tuple):
            raise Exception('Cannot parse tuples as index value. '
                            'Valid types are int, list and numpy.ndarray')
        idx = numpy.atleast_1d(numpy.asarray(i))
        self.np = self.np - idx.size
        for name in self._PER_PARTICLE:
            setattr(self, name, numpy.delete(getattr(self, name), i, axis=0))
        if self.fluid:
            self.f_p = numpy.delete(self.f_p, i, axis=0)

    def deleteAllParticles(self):
        self.np[0] = 0
        d = int(self.nd[0])
        self.x = numpy.zeros((0, d))
        self.radius = numpy.ones(0)
        self.xyzsum = numpy.zeros((0, 3))
        self.vel = numpy.zeros((0, d))
        self.fixvel = numpy.zeros(0)
        self.force = numpy.zeros((0, d))
        self.angpos = numpy.zeros((0, d))
        self.angvel = numpy.zeros((0, d))
        self.torque = numpy.zeros((0, d))
        for name in ("es_dot", "es", "ev_dot", "ev", "p"):
            setattr(self, name, numpy.zeros(0))
        self.color = numpy.zeros(0, dtype=numpy.int32)
        if self.fluid:
            self.f_p = numpy.zeros((0, 3))

    # ----------------------------------------------------------------- I/O
    def readbin(self, targetbin, verbose=True, bonds=True, sigma0mod=True, esysparticle=False):
        """Read a .bin file (python/sphere.py:965)."""
        binio.read_bin(targetbin, self, verbose=verbose)

    def writebin(self, folder="../input/", verbose=True):
        """Write <folder>/<sid>.bin (python/sphere.py:1355)."""
        targetbin = folder + "/" + self.sid + ".bin"
        if verbose:
            print("Output file: {0}".format(targetbin))
        binio.write_bin(targetbin, self)

    def _outdir(self, root=None):
        return os.path.join(root if root is not None else default_root(), "output")

    def readfirst(self, verbose=True, root=None):
        self.readbin(os.path.join(self._outdir(root), self.sid + ".output00000.bin"), verbose)

    def readsecond(self, verbose=True, root=None):
        self.readbin(os.path.join(self._outdir(root), self.sid + ".output00001.bin"), verbose)

    def readstep(self, step, verbose=True, root=None):
        fn = os.path.join(self._outdir(root), "{0}.output{1:0=5}.bin".format(self.sid, step))
        self.readbin(fn, verbose)

    def readlast(self, verbose=True, root=None):
        """Read the last output file (python/sphere.py:2314)."""
        lastfile = status(self.sid, root=root)
        self.readstep(lastfile, verbose, root=root)

    def readTime(self, time, verbose=True, root=None):
        self.readfirst(verbose=False, root=root)
        t_first = self.currentTime()
        n_first = self.time_step_count[0]
        self.readlast(verbose=False, root=root)
        t_last = self.currentTime()
        n_last = self.time_step_count[0]
        if time < t_first or time > t_last:
            raise Exception('Error: The specified time {} s is outside the range of output '
                            'files [{}; {}] s.'.format(time, t_first, t_last))
        dt_dn = (t_last - t_first) / (n_last - n_first)
        step = int((time - t_first) / dt_dn) + n_first + 1
        self.readstep(step, verbose=verbose, root=root)

    def currentTime(self, value=-1):
        if value != -1:
            self.time_current[0] = value
        else:
            return self.time_current[0]

    # ------------------------------------------------------------- set-up
    def generateRadii(self, psd='logn', mean=440e-6, variance=8.8e-9, histogram=False):
        """Draw radii (python/sphere.py:2358)."""
        n = int(self.np[0])
        if psd == 'logn':
            mu = math.log((mean ** 2) / math.sqrt(variance + mean ** 2))
            sigma = math.sqrt(math.log(variance / (mean ** 2) + 1))
            self.radius = numpy.random.lognormal(mu, sigma, n)
        elif psd == 'uni':
            self.radius = numpy.random.uniform(mean - variance, mean + variance, n)
        else:
            raise Exception('Particle size distribution type not understood (' + str(psd) +
                            '). Valid values are \'uni\' or \'logn\'')

    def generateBimodalRadii(self, r_small=0.005, r_large=0.05, ratio=0.2, verbose=True):
        if r_small >= r_large:
            raise Exception("r_large should be larger than r_small")
        V_small = V_sphere(r_small)
        V_large = V_sphere(r_large)
        nlarge = int(V_small / V_large * ratio * self.np[0])
        self.radius[:] = r_small
        self.radius[0:nlarge] = r_large
        numpy.random.shuffle(self.radius)
        if verbose:
            print("generateBimodalRadii created " + str(nlarge) + " large particles, and " +
                  str(self.np[0] - nlarge) + " small")

    def contactModel(self, contactmodel):
        self.contactmodel[0] = contactmodel

    def wall0iz(self):
        if self.nw[0] > 0:
            return int(self.w_x[0] / (self.L[2] / self.num[2]))
        raise Exception('No dynamic top wall present!')

    def normalBoundariesXY(self):
        self.periodic[0] = 0

    def periodicBoundariesXY(self):
        self.periodic[0] = 1

    def periodicBoundariesX(self):
        self.periodic[0] = 2

    def adaptiveGrid(self):
        self.adaptive[0] = 1

    def staticGrid(self):
        self.adaptive[0] = 0

    def _cellsize_min(self, dx):
        if dx > 0.0:
            return dx
        return 2.1 * numpy.amax(self.radius)

    def defineWorldBoundaries(self, L, origo=[0.0, 0.0, 0.0], dx=-1):
        """Set domain and grid (python/sphere.py:2607)."""
        if dx <= 0.0 and self.np[0] < 1:
            raise Exception('Error: You need to define dx in defineWorldBoundaries if there '
                            'are no particles in the simulation.')
        cellsize_min = self._cellsize_min(dx)
        self.origo[:] = origo[:]
        self.L[:] = L[:]
        for d in range(3):
            self.num[d] = numpy.ceil((self.L[d] - self.origo[d]) / cellsize_min)
        if self.num[0] < 3 or self.num[1] < 3 or self.num[2] < 3:
            raise Exception("Error: The grid must be at least 3 cells in each direction\n"
                            "Grid: x={}, y={}, z={}\nPlease increase the world size."
                            .format(self.num[0], self.num[1], self.num[2]))

    def initGrid(self, dx=-1):
        cellsize_min = self._cellsize_min(dx)
        for d in range(3):
            self.num[d] = numpy.ceil((self.L[d] - self.origo[d]) / cellsize_min)
        if self.num[0] < 4 or self.num[1] < 4 or self.num[2] < 4:
            raise Exception("Error: The grid must be at least 3 cells in each direction\n"
                            "Grid: x={}, y={}, z={}".format(self.num[0], self.num[1],
                                                            self.num[2]))
        if self.nw > 0:
            self.w_x[0] = self.L[0]

    def initGridAndWorldsize(self, margin=2.0):
        r_max = numpy.amax(self.radius)
        self.origo = numpy.array([numpy.amin(self.x[:, d] - self.radius[:]) for d in range(3)]) \
            - margin * r_max
        self.L = numpy.array([numpy.amax(self.x[:, d] + self.radius[:]) for d in range(3)]) \
            + margin * r_max
        cellsize_min = 2.1 * r_max
        for d in range(3):
            self.num[d] = numpy.ceil((self.L[d] - self.origo[d]) / cellsize_min)
        if self.num[0] < 4 or self.num[1] < 4 or self.num[2] < 4:
            raise Exception("Error: The grid must be at least 3 cells in each direction, "
                            "num = " + str(self.num))
        if self.nw > 0:
            self.w_x[0] = self.L[0]

    def initGridPos(self, gridnum=numpy.array([12, 12, 36])):
        """Cubic lattice positions (python/sphere.py:2725)."""
        self.num = numpy.asarray(gridnum).astype(numpy.uint32)
        r_max = numpy.amax(self.radius)
        cellsize = 2.1 * r_max
        self.L = self.num * cellsize
        n = int(self.np[0])
        if (self.num[0] * self.num[1] * self.num[2] - (2 ** 3)) < n:
            raise NameError('Error! The grid is not sufficiently large.')
        if self.periodic[0] == 1:
            self.num[0] -= 1
            self.num[1] -= 1
        if (self.num[0] * self.num[1] * self.num[2] - (2 * 3 * 3)) < n:
            raise NameError('Error! The grid is not sufficiently large.')
        i = numpy.arange(n)
        gp = numpy.empty((n, 3), dtype=numpy.uint32)
        gp[:, 0] = i % self.num[0]
        gp[:, 1] = numpy.floor(i / self.num[0]) % self.num[0]
        gp[:, 2] = numpy.floor(i / (self.num[0] * self.num[1]))
        self.x = gp * cellsize + 0.5 * cellsize
        if self.periodic[0] == 1:
            odd = (gp[:, 2] % 2).astype(bool)
            self.x[odd, 0] += 0.5 * cellsize
            self.x[odd, 1] += 0.5 * cellsize
            self.num[0] += 1
            self.num[1] += 1

    def initRandomGridPos(self, gridnum=numpy.array([12, 12, 32]), padding=2.1):
        """Jittered cubic lattice (python/sphere.py:2787)."""
        coarsegrid = numpy.floor(numpy.asarray(gridnum) / 2)
        r_max = numpy.amax(self.radius)
        cellsize = padding * r_max * 2
        n = int(self.np[0])
        if ((coarsegrid[0] - 1) * (coarsegrid[1] - 1) * (coarsegrid[2] - 1)) < n:
            raise NameError('Error! The grid is not sufficiently large.')
        i = numpy.arange(n)
        gp = numpy.empty((n, 3), dtype=numpy.uint32)
        gp[:, 0] = i % coarsegrid[0]
        gp[:, 1] = numpy.floor(i / coarsegrid[0]) % coarsegrid[1]
        gp[:, 2] = numpy.floor(i / (coarsegrid[0] * coarsegrid[1]))
        r = (self.radius * 1.05)[:, None]
        self.x = gp * cellsize + ((cellsize - r) - r) * numpy.random.random_sample((n, 3)) + r
        x_max = numpy.max(self.x[:, 0] + self.radius)
        y_max = numpy.max(self.x[:, 1] + self.radius)
        z_max = numpy.max(self.x[:, 2] + self.radius)
        self.num[0] = numpy.ceil(x_max / cellsize)
        self.num[1] = numpy.ceil(y_max / cellsize)
        self.num[2] = numpy.ceil(z_max / cellsize)
        self.L = self.num * cellsize

    def createBondPair(self, i, j, spacing=-0.1):
        """Place j next to i at a random orientation and bond them
        (python/sphere.py:2848)."""
        x_i = self.x[i]
        r_i = self.radius[i]
        r_j = self.radius[j]
        dist_ij = (r_i + r_j) * (1.0 + spacing)
        azi = numpy.radians(numpy.random.rand(1) * 360.0)
        ang = numpy.radians(numpy.random.rand(1) * 180.0 - 90.0)
        x_j = numpy.copy(x_i)
        x_j[0] = x_j[0] + dist_ij * numpy.cos(azi) * numpy.cos(ang)
        x_j[1] = x_j[1] + dist_ij * numpy.sin(azi) * numpy.cos(ang)
        x_j[2] = x_j[2] + dist_ij * numpy.sin(ang) * numpy.cos(azi)
        self.x[j] = x_j
        for d in range(3):
            if self.x[j, d] < self.origo[d]:
                self.x[j, d] += x_i[d] - x_j[d]
        for d in range(3):
            if self.x[j, d] > self.L[d]:
                self.x[j, d] -= abs(x_j[d] - x_i[d])
        self.bond(i, j)
        x_ij = self.x[i] - self.x[j]
        x_ij_length = numpy.sqrt(x_ij.dot(x_ij))
        if (x_ij_length - dist_ij) > dist_ij * 0.01:
            raise Exception("Error, something went wrong in createBondPair")

    def randomBondPairs(self, ratio=0.3, spacing=-0.1):
        """Bond random particle pairs (python/sphere.py:2905); draws with
        numpy.random.randint, the successor of random_integers."""
        bp = numpy.unique(numpy.random.randint(0, self.np[0], size=int(self.np[0] * ratio)))
        if bp.size % 2 > 0:
            bp = bp[:-1].copy()
        bp = bp.reshape(int(bp.size / 2), 2).copy()
        for k in range(bp.shape[0]):
            self.createBondPair(bp[k, 0], bp[k, 1], spacing)

    def zeroKinematics(self):
        n, d = int(self.np[0]), int(self.nd[0])
        self.force = numpy.zeros((n, d))
        self.torque = numpy.zeros((n, d))
        self.vel = numpy.zeros((n, d), dtype=numpy.float64)
        self.angvel = numpy.zeros((n, d), dtype=numpy.float64)
        self.angpos = numpy.zeros((n, d), dtype=numpy.float64)
        self.es = numpy.zeros(n, dtype=numpy.float64)
        self.ev = numpy.zeros(n, dtype=numpy.float64)
        self.xyzsum = numpy.zeros((n, 3), dtype=numpy.float64)

    def adjustUpperWall(self, z_adjust=1.1):
        self.nw = numpy.ones(1, dtype=numpy.int32)
        self.wmode = numpy.zeros(1)
        self.w_n = numpy.zeros((1, int(self.nd[0])), dtype=numpy.float64)
        self.w_n[0, 2] = -1.0
        self.w_vel = numpy.zeros(1)
        self.w_force = numpy.zeros(1)
        self.w_sigma0 = numpy.zeros(1)
        self.w_x = numpy.zeros(1)
        self.w_m = numpy.zeros(1)
        self.adjustWall(idx=0, adjust=z_adjust)

    def adjustWall(self, idx, adjust=1.1, wall_mass_factor=1.0):
        """Fit grid and wall idx to the particles (python/sphere.py:2972)."""
        if idx == 0:
            dim = 2
        elif idx in (1, 2):
            dim = 0
        elif idx in (3, 4):
            dim = 1
        else:
            print("adjustWall: idx value not understood")
        xmin = numpy.min(self.x[:, dim] - self.radius)
        xmax = numpy.max(self.x[:, dim] + self.radius)
        cellsize = self.L[0] / self.num[0]
        self.num[dim] = numpy.ceil(((xmax - xmin) * adjust + xmin) / cellsize)
        self.L[dim] = (xmax - xmin) * adjust + xmin
        self.w_x[idx] = xmax if idx in (0, 1, 3) else xmin
        self.w_m[idx] = self.totalMass()

    def consolidate(self, normal_stress=10e3):
        """Top wall at a constant normal stress (python/sphere.py:3019)."""
        self.nw[0] = 1
        if normal_stress <= 0.0:
            raise Exception('consolidate() error: The normal stress should be a positive '
                            'value, but is ' + str(normal_stress) + ' Pa')
        self.zeroKinematics()
        self.adjustUpperWall()
        self.wmode = numpy.array([1])
        self.w_sigma0 = numpy.ones(1) * normal_stress
        self.w_m[0] = self.totalMass()

    def uniaxialStrainRate(self, wvel=-0.001):
        """Top wall at a constant velocity (python/sphere.py:3050)."""
        self.zeroKinematics()
        self.adjustUpperWall()
        self.wmode = numpy.array([2])
        self.w_vel = numpy.array([wvel])

    def triaxial(self, wvel=-0.001, normal_stress=10.0e3):
        self.zeroKinematics()
        self.nw[0] = 5
        self.wmode = numpy.array([2, 1, 1, 1, 1])
        self.w_vel = numpy.array([1, 0, 0, 0, 0]) * wvel
        self.w_sigma0 = numpy.array([0, 1, 1, 1, 1]) * normal_stress
        self.w_n = numpy.array(([0, 0, -1], [-1, 0, 0], [1, 0, 0], [0, -1, 0], [0, 1, 0]),
                               dtype=numpy.float64)
        self.w_x = numpy.zeros(5)
        self.w_m = numpy.zeros(5)
        self.w_force = numpy.zeros(5)
        for i in range(5):
            self.adjustWall(idx=i)

    def shear(self, shear_strain_rate=1.0, shear_stress=False):
        """Shear set-up: fixed bottom layer, top layer moving along +x
        (python/sphere.py:3097)."""
        self.nw[0] = 1
        z_min = numpy.min(self.x[:, 2] - self.radius)
        z_max = numpy.max(self.x[:, 2] + self.radius)
        cellsize = self.L[0] / self.num[0]
        self.num[2] += 1
        self.L[2] = self.num[2] * cellsize
        self.zeroKinematics()
        self.wmode = numpy.array([1])
        d_max_below = numpy.max(self.radius[numpy.nonzero(self.x[:, 2] <
                                                           (z_max - z_min) * 0.3)]) * 2.0
        I = numpy.nonzero(self.x[:, 2] < (z_min + d_max_below))
        self.fixvel[I] = 1
        self.angvel[I, :] = 0.0
        self.vel[I, 0] = 0.0
        self.vel[I, 1] = 0.0
        self.color[I] = -1
        d_max_top = numpy.max(self.radius[numpy.nonzero(self.x[:, 2] >
                                                         (z_max - z_min) * 0.7)]) * 2.0
        I = numpy.nonzero(self.x[:, 2] > (z_max - d_max_top))
        self.fixvel[I] = 1
        self.angvel[I, :] = 0.0
        if shear_stress is False:
            self.vel[I, 0] = (z_max - z_min) * shear_strain_rate
        else:
            self.vel[I, 0] = 0.0
            self.wmode[0] = 3
            self.w_tau_x[0] = float(shear_stress)
        self.vel[I, 1] = 0.0
        self.color[I] = -1
        self.gamma_wt[0] = 0.0
        self.mu_ws[0] = 0.0
        self.mu_wd[0] = 0.0

    def cellSize(self):
        self.dx = self.L / self.num

    def initTemporal(self, total, current=0.0, file_dt=0.05, step_count=0, dt=-1,
                     epsilon=0.01):
        """Time step and output cadence (python/sphere.py:3307)."""
        if dt > 0.0:
            self.time_dt[0] = dt
            if self.np[0] > 0:
                print("Warning: Manually specifying the time step length when simulating "
                      "particles may produce instabilities.")
        elif self.np[0] > 0:
            r_min = numpy.min(self.radius)
            m_min = self.rho[0] * 4.0 / 3.0 * numpy.pi * r_min ** 3
            if self.E[0] > 0.001:
                k_max = numpy.max(numpy.pi / 2.0 * self.E[0] * self.radius)
            else:
                k_max = numpy.max([self.k_n[:], self.k_t[:]])
            self.time_dt[0] = epsilon / (numpy.sqrt(k_max / m_min))
        elif not self.fluid:
            raise Exception('Error: Could not automatically set a time step.')
        if self.fluid:
            self.time_dt[0] = numpy.min([self.largestFluidTimeStep(), self.time_dt[0]])
        self.time_current[0] = current
        self.time_total[0] = total
        self.time_file_dt[0] = file_dt
        self.time_step_count[0] = 0

    def dry(self):
        self.fluid = False

    def wet(self):
        """Total fluid saturation with the default fluid
        (python/sphere.py:3386): initFluid() with its defaults."""
        self.fluid = True
        self.initFluid()

    def largestFluidTimeStep(self, safety=0.5, v_max=-1.0):
        """The largest stable fluid time step (python/sphere.py:3167): the
        advective (CFL) limit, the smallest cell width over the largest
        fluid speed (1e-7 m/s when the fluid is at rest); for the
        Navier-Stokes solver the smaller of that and the diffusive limit
        0.5 dx^2 / mu, times `safety`."""
        if not self.fluid:
            return None
        v = numpy.asarray(self.v_f, dtype=numpy.float64).reshape(-1, 3)
        v_max_obs = numpy.amax(numpy.sqrt((v * v).sum(axis=1))) if v.size else 0.0
        if v_max_obs == 0:
            v_max_obs = 1.0e-7
        if v_max < 0.0:
            v_max = v_max_obs
        dx_min = numpy.min(self.L / self.num)
        if int(numpy.asarray(self.cfd_solver).ravel()[0]) == 0:
            dt_von_neumann = 0.5 * dx_min ** 2 / (self.mu[0] + 1.0e-16)
            return numpy.min([dt_von_neumann, dx_min / v_max]) * safety
        self._check_darcy('largestFluidTimeStep')
        self.cellSize()
        return dx_min / v_max

    def defaultParams(self, mu_s=0.5, mu_d=0.5, mu_r=0.0, rho=2600, k_n=1.16e9, k_t=1.16e9,
                      k_r=0, gamma_n=0.0, gamma_t=0.0, gamma_r=0.0, gamma_wn=1.0e4,
                      gamma_wt=1.0e4, capillaryCohesion=0):
        """Material defaults (python/sphere.py:3762)."""
        self.rho = numpy.ones(1, dtype=numpy.float64) * rho
        self.k_n = numpy.ones(1, dtype=numpy.float64) * k_n
        self.k_t = numpy.ones(1, dtype=numpy.float64) * k_t
        self.k_r = numpy.ones(1, dtype=numpy.float64) * k_r
        self.gamma_n = numpy.ones(1, dtype=numpy.float64) * gamma_n
        self.gamma_t = numpy.ones(1, dtype=numpy.float64) * gamma_t
        self.gamma_r = numpy.ones(1, dtype=numpy.float64) * gamma_r
        self.mu_s = numpy.ones(1, dtype=numpy.float64) * mu_s
        self.mu_d = numpy.ones(1, dtype=numpy.float64) * mu_d
        self.mu_r = numpy.ones(1, dtype=numpy.float64) * mu_r
        self.gamma_wn[0] = gamma_wn
        self.gamma_wt[0] = gamma_wt
        self.mu_ws = self.mu_s
        self.mu_wd = self.mu_d
        theta = 0.0
        if capillaryCohesion == 1:
            self.kappa[0] = 2.0 * math.pi * gamma_t * numpy.cos(theta)
            self.V_b[0] = 1e-12
        else:
            self.kappa[0] = 0.0
            self.V_b[0] = 0.0
        self.db[0] = (1.0 + theta / 2.0) * self.V_b[0] ** (1.0 / 3.0)

    def setStiffnessNormal(self, k_n):
        self.k_n[0] = k_n

    def setStiffnessTangential(self, k_t):
        self.k_t[0] = k_t

    def setYoungsModulus(self, E):
        """Use k_n = k_t = pi/2*E*R (python/sphere.py:3895)."""
        self.E[0] = E

    def setDampingNormal(self, gamma, over_damping=False):
        self.gamma_n[0] = gamma
        critical_gamma = 2.0 * numpy.sqrt(self.smallestMass() * self.k_n[0])
        damping_ratio = gamma / critical_gamma
        if damping_ratio > 1.0 and not over_damping:
            raise Exception('Warning: The system is over-dampened (ratio = ' +
                            str(damping_ratio) + ') in the normal component.\n'
                            'Call this function once more with `over_damping=True` if this '
                            'is what you want. \nCritical damping = ' + str(critical_gamma) + '.')

    def setDampingTangential(self, gamma, over_damping=False):
        self.gamma_t[0] = gamma
        damping_ratio = gamma / (2.0 * numpy.sqrt(self.smallestMass() * self.k_t[0]))
        if damping_ratio > 1.0 and not over_damping:
            raise Exception('Warning: The system is over-dampened (ratio = ' +
                            str(damping_ratio) + ') in the tangential component.\n'
                            'Call this function once more with `over_damping=True` if this '
                            'is what you want.')

    def setStaticFriction(self, mu_s):
        self.mu_s[0] = mu_s

    def setDynamicFriction(self, mu_d):
        self.mu_d[0] = mu_d

    def scaleSize(self, factor):
        self.L *= factor
        self.x *= factor
        self.radius *= factor
        self.xyzsum *= factor
        self.vel *= factor
        self.force *= factor
        self.torque *= factor
        self.w_x *= factor
        self.w_m *= factor
        self.w_vel *= factor
        self.w_force *= factor

    def bond(self, i, j):
        """Register a bond between particles i and j (python/sphere.py:4075)."""
        self.lambda_bar[0] = 1.0
        self.bonds = numpy.vstack((numpy.asarray(self.bonds, dtype=numpy.uint32).reshape(-1, 2),
                                   [i, j])).astype(numpy.uint32)
        self.bonds_delta_n = numpy.append(numpy.asarray(self.bonds_delta_n, dtype=numpy.float64),
                                          [0.0])
        self.bonds_delta_t = numpy.vstack((numpy.asarray(self.bonds_delta_t).reshape(-1, 3),
                                           [0.0, 0.0, 0.0]))
        self.bonds_omega_n = numpy.append(numpy.asarray(self.bonds_omega_n, dtype=numpy.float64),
                                          [0.0])
        self.bonds_omega_t = numpy.vstack((numpy.asarray(self.bonds_omega_t).reshape(-1, 3),
                                           [0.0, 0.0, 0.0]))
        self.nb0 += 1

    # ------------------------------------------------------------ analysis
    def currentNormalStress(self, type='defined'):
        if type == 'defined':
            return self.w_sigma0[0] + self.w_sigma0_A[0] * numpy.sin(
                2.0 * numpy.pi * self.w_sigma0_f[0] * self.time_current[0])
        elif type == 'effective':
            return self.w_force[0] / (self.L[0] * self.L[1])
        raise Exception('Normal stress type ' + type + ' not understood')

    def surfaceArea(self, idx):
        return 4.0 * numpy.pi * self.radius[idx] ** 2

    def volume(self, idx):
        return V_sphere(self.radius[idx])

    def mass(self, idx):
        return self.rho[0] * self.volume(idx)

    def totalMass(self):
        return _seqsum(self.rho[0] * V_sphere(self.radius))

    def smallestMass(self):
        """As in python/sphere.py:4186, the volume of the smallest particle."""
        return V_sphere(numpy.min(self.radius))

    def largestMass(self):
        return V_sphere(numpy.max(self.radius))

    def momentOfInertia(self, idx):
        return 2.0 / 5.0 * self.mass(idx) * self.radius[idx] ** 2

    def kineticEnergy(self, idx):
        return 0.5 * self.mass(idx) * numpy.sqrt(numpy.dot(self.vel[idx, :],
                                                           self.vel[idx, :])) ** 2

    def _kin(self):
        m = self.rho[0] * V_sphere(self.radius)
        v = numpy.sqrt(numpy.einsum('ij,ij->i', self.vel, self.vel))
        return 0.5 * m * v ** 2

    def totalKineticEnergy(self):
        return _seqsum(self._kin())

    def rotationalEnergy(self, idx):
        return 0.5 * self.momentOfInertia(idx) * numpy.sqrt(
            numpy.dot(self.angvel[idx, :], self.angvel[idx, :])) ** 2

    def _rot(self):
        m = self.rho[0] * V_sphere(self.radius)
        inertia = 2.0 / 5.0 * m * self.radius ** 2
        w = numpy.sqrt(numpy.einsum('ij,ij->i', self.angvel, self.angvel))
        return 0.5 * inertia * w ** 2

    def totalRotationalEnergy(self):
        return _seqsum(self._rot())

    def viscousEnergy(self, idx):
        return self.ev[idx]

    def totalViscousEnergy(self):
        return _seqsum(self.ev)

    def frictionalEnergy(self, idx):
        return self.es[idx]

    def totalFrictionalEnergy(self):
        return _seqsum(self.es)

    def energy(self, method):
        """Energy sums (python/sphere.py:4311)."""
        if method == 'pot':
            m = numpy.ones(self.np) * 4.0 / 3.0 * math.pi * self.radius ** 3 * self.rho
            return numpy.sum(m * math.sqrt(numpy.dot(self.g, self.g)) * self.x[:, 2])
        elif method == 'kin':
            m = numpy.ones(self.np) * 4.0 / 3.0 * math.pi * self.radius ** 3 * self.rho
            v = numpy.sqrt(numpy.einsum('ij,ij->i', self.vel, self.vel))
            return _seqsum(0.5 * m * v ** 2)
        elif method == 'rot':
            m = numpy.ones(self.np) * 4.0 / 3.0 * math.pi * self.radius ** 3 * self.rho
            w = numpy.sqrt(numpy.einsum('ij,ij->i', self.angvel, self.angvel))
            return _seqsum(0.5 * 2.0 / 5.0 * m * self.radius ** 2 * w ** 2)
        elif method == 'shear':
            return numpy.sum(self.es)
        elif method == 'shearrate':
            return numpy.sum(self.es_dot)
        elif method == 'visc_n':
            return numpy.sum(self.ev)
        elif method == 'visc_n_rate':
            return numpy.sum(self.ev_dot)
        elif method == 'bondpot':
            if self.nb0 > 0:
                b = numpy.asarray(self.bonds, dtype=numpy.int64)
                R_bar = self.lambda_bar * numpy.minimum(self.radius[b[:, 0]],
                                                        self.radius[b[:, 1]])
                A = numpy.pi * R_bar ** 2
                I = 0.25 * numpy.pi * R_bar ** 4
                J = I * 2.0
                fn = numpy.sum(0.5 * A * self.k_n * numpy.abs(self.bonds_delta_n) ** 2)
                ft = numpy.sum(0.5 * A * self.k_t * numpy.linalg.norm(self.bonds_delta_t) ** 2)
                tn = numpy.sum(0.5 * J * self.k_t * numpy.abs(self.bonds_omega_n) ** 2)
                tt = numpy.sum(0.5 * I * self.k_n * numpy.linalg.norm(self.bonds_omega_t) ** 2)
                return fn + ft + tn + tt
            return 0.0
        raise Exception('Unknownw energy() method "' + method + '"')

    def voidRatio(self):
        V_t = (self.L[0] - self.origo[0]) * (self.L[1] - self.origo[1]) * \
            (self.w_x[0] - self.origo[2])
        V_s = numpy.sum(4.0 / 3.0 * math.pi * self.radius ** 3)
        return (V_t - V_s) / V_s

    def bulkPorosity(self, trim=True):
        if trim:
            lo = numpy.min(self.x - self.radius[:, None], axis=0)
            hi = numpy.max(self.x + self.radius[:, None], axis=0)
            V_total = numpy.prod(hi - lo)
        elif self.nw == 0:
            V_total = self.L[0] * self.L[1] * self.L[2]
        else:
            V_total = self.L[0] * self.L[1] * self.w_x[0]
            if V_total <= 0.0:
                raise Exception("Could not determine total volume")
        V_solid = numpy.sum(V_sphere(self.radius))
        return (V_total - V_solid) / V_total

    def momentum(self, idx):
        return self.rho[0] * V_sphere(self.radius[idx]) * self.vel[idx, :]

    def totalMomentum(self):
        m = self.rho[0] * V_sphere(self.radius)
        return numpy.sum(m[:, None] * self.vel, axis=0)

    # ------------------------------------------------------- shear analysis
    def shearDisplacement(self):
        """Shear displacement: the largest x displacement (xyzsum) of the
        spheres with a prescribed velocity (python/sphere.py:4777)."""
        fixed = numpy.nonzero(self.fixvel > 0.0)
        return numpy.max(self.xyzsum[fixed, 0])

    def shearVelocity(self):
        """Shear velocity: the largest x velocity of the spheres with a
        prescribed velocity (python/sphere.py:4794)."""
        fixed = numpy.nonzero(self.fixvel > 0.0)
        return numpy.max(self.vel[fixed, 0])

    def shearVel(self):
        return self.shearVelocity()

    def shearStrain(self):
        """Shear displacement over the top wall height (python/sphere.py:4816)."""
        return self.shearDisplacement() / self.w_x[0]

    def shearStrainRate(self):
        """Shear velocity over the top wall height (python/sphere.py:4837)."""
        return self.shearVelocity() / self.w_x[0]

    def shearStress(self, type='effective'):
        """'defined': the prescribed top-wall shear stress; 'effective': minus
        the x force on the spheres moving at positive prescribed x velocity,
        per unit box area (python/sphere.py:6407)."""
        if type == 'defined':
            return self.w_tau_x[0]
        if type == 'effective':
            moving = (self.fixvel > 0.0) & (self.vel[:, 0] > 0.0)
            force = numpy.zeros(3)
            for i in numpy.nonzero(moving)[0]:      # in index order, as summed there
                force += -self.force[i, :]
            return force[0] / (self.L[0] * self.L[1])
        raise Exception('Shear stress type ' + type + ' not understood')

    def inertiaParameterPlanarShear(self):
        """I = shear strain rate * mean radius * sqrt(rho / normal stress)
        (python/sphere.py:4855)."""
        return self.shearStrainRate() * numpy.mean(self.radius) * \
            numpy.sqrt(self.rho[0] / self.currentNormalStress())

    def acceleration(self, idx=-1):
        """Acceleration force / mass + g of one or more spheres
        (python/sphere.py:6278)."""
        if idx == -1:
            idx = range(int(self.np[0]))
        return self.force[idx, :] / (V_sphere(self.radius[idx]) * self.rho[0]) + self.g

    def setTopWallNormalStressModulation(self, A, f, plot=False):
        """Sine modulation of the top wall's normal stress, amplitude A and
        frequency f (python/sphere.py:6188); plotting is not provided."""
        self.w_sigma0_A[0] = A
        self.w_sigma0_f[0] = f

    def disableTopWallNormalStressModulation(self):
        self.setTopWallNormalStressModulation(A=0.0, f=0.0)

    # ---------------------------------------- contact and porosity analysis
    def _analysis_stepper(self, device=-1):
        from .runner import Stepper
        st = Stepper([self], precision='fp64', length='reference', device=device)
        st.upload()
        return st

    def porosity(self, slices=10, verbose=False, device=-1):
        """Porosity in `slices` horizontal slabs and the slab mid-depths:
        the reference's `porosity` program (src/sphere.cpp:487-606), run on
        the GPU (sph_porosity) at full FP64 precision.  Returns (porosity,
        depth) as python/sphere.py:4437 does."""
        st = self._analysis_stepper(device)
        try:
            z, p = st.porosity(slices)
        finally:
            st.close()
        return p, z

    def findOverlaps(self, device=-1):
        """All overlapping sphere pairs: the reference's n^2 search
        (src/sphere.cpp:677-725, `sphere --contacts`), on the GPU
        (sph_overlaps).  Sets self.pairs ([2, n] int32, i < j) and
        self.overlaps (the negative distances), as python/sphere.py:4868."""
        st = self._analysis_stepper(device)
        try:
            pairs, d = st.overlaps()
        finally:
            st.close()
        self.pairs = numpy.array((pairs[:, 0], pairs[:, 1]), dtype=numpy.int32)
        self.overlaps = numpy.array(d)

    def findCoordinationNumber(self):
        """Contacts per sphere from self.pairs (python/sphere.py:4885)."""
        self.coordinationnumber = numpy.zeros(int(self.np[0]), dtype=numpy.int64)
        numpy.add.at(self.coordinationnumber, self.pairs[0, :], 1)
        numpy.add.at(self.coordinationnumber, self.pairs[1, :], 1)

    def findMeanCoordinationNumber(self):
        return numpy.mean(self.coordinationnumber)

    def findNormalForces(self):
        """|f_n| = k_n |overlap| of every overlapping pair
        (python/sphere.py:4906)."""
        self.findOverlaps()
        self.f_n_magn = self.k_n * numpy.abs(self.overlaps)

    def contactSurfaceArea(self, i, j, overlap):
        """Area of the circle where spheres i and j intersect
        (python/sphere.py:4919)."""
        r_i = self.radius[i]
        r_j = self.radius[j]
        d = r_i + r_j + overlap
        contact_radius = 1. / (2. * d) * ((-d + r_i - r_j) * (-d - r_i + r_j) *
                                          (-d + r_i + r_j) * (d + r_i + r_j)) ** 0.5
        return numpy.pi * contact_radius ** 2.

    def contactParticleArea(self, i, j):
        """Cross-section of the pair's mean radius (python/sphere.py:4941)."""
        r_bar = (self.radius[i] + self.radius[j]) * 0.5
        return numpy.pi * r_bar ** 2.

    def findAllContactSurfaceAreas(self):
        return self.contactSurfaceArea(self.pairs[0, :], self.pairs[1, :], self.overlaps)

    def findAllAverageParticlePairAreas(self):
        return self.contactParticleArea(self.pairs[0, :], self.pairs[1, :])

    def findContactStresses(self, area='average'):
        """Normal stress of every contact: |f_n| over the mean-radius area
        ('average') or the contact area ('contact') (python/sphere.py:4980)."""
        self.findNormalForces()
        if area == 'average':
            areas = self.findAllAverageParticlePairAreas()
        elif area == 'contact':
            areas = self.findAllContactSurfaceAreas()
        else:
            raise Exception('Contact area type "' + area + '" not understood')
        self.sigma_contacts = self.f_n_magn / areas

    def findLoadedContacts(self, threshold):
        """Indexes of the contacts whose stress is at least `threshold`
        (python/sphere.py:5004)."""
        self.findContactStresses()
        return numpy.nonzero(self.sigma_contacts >= threshold)

    def forcechains(self, lc=200.0, uc=650.0, outformat='txt', disp='2d', path=None):
        """Force-chain data as the reference's `forcechains` program writes it
        (src/sphere.cpp:727-902): every overlapping pair with f_n = -k_n
        delta_n >= lc, as text rows (outformat 'txt') or as a gnuplot script
        (other formats), written to `path` (default <sid>-fc.txt / .gp) and
        returned as a string.  The script is not rendered here."""
        self.findOverlaps()
        threedim = disp != '2d'
        x = self.x
        pairs = self.pairs.T
        d = self.overlaps
        lines = []
        if outformat == 'txt':
            head = ["x_1, [m]"] + (["y_1, [m]"] if threedim else []) + ["z_1, [m]", "x_2, [m]"] + \
                (["y_2, [m]"] if threedim else []) + ["z_2, [m]", "||f_n||, [N]i", "j"]
            lines.append("\t".join(head))
        else:
            lines.append("set size ratio -1")
            lines.append("set cbrange [%g:%g]" % (lc, uc))
        f_n_max = -self.k_n[0] * (numpy.min(d) if d.size else 0.0)
        for n, ((i, j), dn) in enumerate(zip(pairs, d)):
            f_n = -self.k_n[0] * dn
            if f_n < lc:
                continue
            a = [x[i, 0]] + ([x[i, 1]] if threedim else []) + [x[i, 2]]
            b = [x[j, 0]] + ([x[j, 1]] if threedim else []) + [x[j, 2]]
            if outformat == 'txt':
                lines.append("\t".join("%.17g" % v for v in a + b) + "\t%.17g%d\t%d" % (f_n, i, j))
            elif f_n > lc and (self.fixvel[i] + self.fixvel[j]) == 0.0:
                lines.append("set arrow %d from %s to %s nohead lw %.17g lc palette cb %.17g" %
                             (n + 1, ",".join("%.17g" % v for v in a),
                              ",".join("%.17g" % v for v in b),
                              f_n / f_n_max * 16.0, f_n))
        text = "\n".join(lines) + "\n"
        if path is None:
            path = self.sid + ('-fc.txt' if outformat == 'txt' else '-fc.gp')
        with open(path, 'w') as fh:
            fh.write(text)
        return text

    # ------------------------------------------------------------ ray tracer
    def renderImage(self, method='pres', max_val=1e3, lower_cutoff=0.0, width=800, height=800,
                    device=-1):
        """RGB image [height, width, 3] uint8 of the current state by the
        reference's ray tracer (src/raytracer.cuh:379-560, `sphere
        --render`), on the GPU (sph_render).  method: 'normal', 'pres',
        'vel', 'angvel', 'xdisp' or 'angpos' (src/main.cpp:130-147)."""
        if method not in RENDER_METHODS:
            raise ValueError("Visualization method not understood: " + str(method))
        st = self._analysis_stepper(device)
        try:
            return st.render(method=RENDER_METHODS[method], maxval=max_val,
                             lower_cutoff=lower_cutoff, width=width, height=height)
        finally:
            st.close()

    def render(self, method='pres', max_val=1e3, lower_cutoff=0.0, graphics_format='png',
               verbose=True, root=None, device=-1):
        """Render every output file of this simulation
        (<root>/output/<sid>*.bin) into <root>/img_out/<name>.ppm with the
        ray tracer, then convert the images to graphics_format
        (python/sphere.py:4693).  'png' is written here (no Imagemagick);
        'ppm' keeps the ray tracer's own files.  Returns the image paths."""
        import glob
        root = root if root is not None else default_root()
        if verbose:
            print("Rendering {} images with the raytracer".format(self.sid))
        files = sorted(glob.glob(os.path.join(root, "output", self.sid + "*.bin")))
        return [render(f, method=method, max_val=max_val, lower_cutoff=lower_cutoff,
                       graphics_format=graphics_format, verbose=verbose, root=root,
                       device=device) for f in files]

    # ---------------------------------------------------------------- run
    def run(self, verbose=True, hideinputfile=False, dry=False, valgrind=False,
            cudamemcheck=False, device=-1, precision='fp64', length='reference', root=None,
            strict=False):
        """Run the simulation on a B200 (python/sphere.py:4482).

        Writes <root>/input/<sid>.bin, then steps the simulation in-process
        and writes <root>/output/<sid>.outputNNNNN.bin at t = 0 and every
        time_file_dt, plus <root>/output/<sid>.status.dat, exactly as the
        reference binary does.  valgrind/cudamemcheck have no in-process
        meaning and are ignored.  Keyword extensions: precision ('fp64' or
        'mixed'), length ('reference': FP32-rounded vector lengths as in the
        reference; 'fp64'), root (folder of input/ and output/), strict
        (raise instead of warning on a non-zero status).
        """
        from . import runner
        root = root if root is not None else default_root()
        os.makedirs(os.path.join(root, "input"), exist_ok=True)
        os.makedirs(os.path.join(root, "output"), exist_ok=True)
        self.writebin(folder=os.path.join(root, "input"), verbose=False)
        if dry:
            runner.report_values(self)
            return 0
        st = runner.run_sim(self, root=root, verbose=verbose, device=device,
                            precision=precision, length=length)
        if st != 0:
            msg = "Warning: the sphere run returned with status " + str(st)
            if strict:
                raise RuntimeError(msg)
            print(msg)
        return st

    def cleanup(self, root=None):
        cleanup(self, root=root)


RENDER_METHODS = {'normal': 0, 'pres': 1, 'vel': 2, 'angvel': 3, 'xdisp': 4, 'angpos': 5}


def write_ppm(path, img):
    """Binary PPM of an RGB image [height, width, 3] uint8, the layout of
    DEM::writePPM (src/file_io.cpp:734-757)."""
    img = numpy.ascontiguousarray(img, dtype=numpy.uint8)
    with open(path, 'wb') as fh:
        fh.write("P6 {} {} 255\n".format(img.shape[1], img.shape[0]).encode())
        fh.write(img.tobytes())


def read_ppm(path):
    """RGB image of a binary PPM written by write_ppm."""
    with open(path, 'rb') as fh:
        data = fh.read()
    head = data.split(b"\n", 1)
    tag, w, h, depth = head[0].split()
    if tag != b"P6" or depth != b"255":
        raise ValueError("not an 8-bit binary PPM: " + path)
    w, h = int(w), int(h)
    return numpy.frombuffer(head[1][:w * h * 3], dtype=numpy.uint8).reshape(h, w, 3)


def write_png(path, img):
    """8-bit RGB PNG of an image [height, width, 3] uint8 (filter 0 on every
    row, one zlib stream)."""
    import struct
    import zlib
    img = numpy.ascontiguousarray(img, dtype=numpy.uint8)
    h, w = img.shape[:2]
    raw = numpy.zeros((h, 1 + 3 * w), dtype=numpy.uint8)
    raw[:, 1:] = img.reshape(h, 3 * w)

    def chunk(kind, body):
        return (struct.pack(">I", len(body)) + kind + body +
                struct.pack(">I", zlib.crc32(kind + body) & 0xffffffff))

    with open(path, 'wb') as fh:
        fh.write(b"\x89PNG\r\n\x1a\n")
        fh.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        fh.write(chunk(b"IDAT", zlib.compress(raw.tobytes(), 6)))
        fh.write(chunk(b"IEND", b""))


def convert(graphics_format='png', folder='../img_out'):
    """Convert every PPM image in folder to graphics_format and remove the
    PPM files (python/sphere.py:7450).  Only 'png' is written here; 'ppm'
    leaves the files as they are."""
    import glob
    if graphics_format == 'ppm':
        return
    if graphics_format != 'png':
        raise ValueError("graphics_format must be 'png' or 'ppm' here")
    for f in sorted(glob.glob(os.path.join(folder, "*.ppm"))):
        write_png(f[:-4] + ".png", read_ppm(f))
        os.remove(f)


def render(binary, method='pres', max_val=1e3, lower_cutoff=0.0, graphics_format='png',
           verbose=True, root=None, device=-1):
    """Render one .bin file with the ray tracer into <root>/img_out/<name>.ppm
    (`sphere --render`, src/raytracer.cuh:556, name = the file name without
    its extension), then convert it (python/sphere.py:7472).  Returns the
    image path."""
    root = root if root is not None else default_root()
    s = sim(fluid=False)
    s.readbin(binary, verbose=False)
    img = s.renderImage(method=method, max_val=max_val, lower_cutoff=lower_cutoff,
                        device=device)
    outdir = os.path.join(root, "img_out")
    os.makedirs(outdir, exist_ok=True)
    name = os.path.splitext(os.path.basename(binary))[0]
    path = os.path.join(outdir, name + ".ppm")
    write_ppm(path, img)
    if verbose:
        print("  Saving image: " + path)
    if graphics_format == 'ppm':
        return path
    if graphics_format != 'png':
        raise ValueError("graphics_format must be 'png' or 'ppm' here")
    png = path[:-4] + ".png"
    write_png(png, img)
    os.remove(path)
    return png


def status(project, root=None):
    """Last output file number of a run (python/sphere.py:7721)."""
    root = root if root is not None else default_root()
    with open(os.path.join(root, "output", "{0}.status.dat".format(project))) as fh:
        return int(fh.read().split()[2])


def cleanup(sim_obj, root=None):
    """Remove a simulation's input/output files (python/sphere.py:7743)."""
    import glob
    root = root if root is not None else default_root()
    pats = [os.path.join(root, "input", sim_obj.sid + ".bin"),
            os.path.join(root, "output", sim_obj.sid + ".*.bin"),
            os.path.join(root, "output", sim_obj.sid + ".status.dat")]
    for pat in pats:
        for f in glob.glob(pat):
            os.remove(f)
