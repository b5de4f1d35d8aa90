"""Reader and writer of sphere's binary input/output format (.bin).

Layout: python/sphere.py:1355-1553 (writebin) and :965-1353 (readbin),
src/file_io.cpp:30-731 (C++ readbin/writebin).  Files are little-endian;
every block below is written in the order the reference writes it.  The
writer produces files byte-identical to python/sphere.py:writebin for
simulations without a fluid, with a Darcy fluid (cfd_solver 1) and with a
Navier-Stokes fluid (cfd_solver 0: the block is read and written, the
solver itself is not built); the reader accepts versions >= 2.1 (older
optional fields default as in python/sphere.py:readbin).
"""
import numpy

from ._abi import cells_from_file, cells_to_file

VERSION = 2.15


class _Reader(object):
    def __init__(self, buf):
        self.buf = memoryview(buf)
        self.pos = 0

    def take(self, dtype, count):
        dtype = numpy.dtype(dtype)
        n = dtype.itemsize * int(count)
        if self.pos + n > len(self.buf):
            raise ValueError("truncated .bin file: need %d bytes at offset %d, have %d"
                             % (n, self.pos, len(self.buf) - self.pos))
        a = numpy.frombuffer(self.buf[self.pos:self.pos + n], dtype=dtype).copy()
        self.pos += n
        return a


def _read_darcy(r, s, n):
    """The fluid block (python/sphere.py:1157-1345 readbin,
    src/file_io.cpp:251-404): the cell fields and boundary codes, then the
    Darcy solver's parameters and pressure force (cfd_solver 1) or the
    Navier-Stokes solver's parameters and its four per-sphere fluid forces
    (cfd_solver 0; the fields are kept, the solver is not built).  dphi is
    stored in the file as the change per fluid step; the sim holds it per
    unit time, divided by time_dt * ndem with the ndem the sim held before
    this read, as the reference's reader divides."""
    version = float(s.version[0])
    if version >= 2.0:
        s.cfd_solver = r.take(numpy.int32, 1)
    else:
        s.cfd_solver = numpy.zeros(1, dtype=numpy.int32)
    solver = int(s.cfd_solver[0])
    if solver not in (0, 1):
        raise ValueError("Value of cfd_solver not understood (%d)" % solver)
    num = [int(v) for v in s.num]
    ncell = num[0] * num[1] * num[2]
    ndem_before = numpy.asarray(getattr(s, "ndem", numpy.array(1)))
    s.mu = r.take(numpy.float64, 1)
    blk = r.take(numpy.float64, ncell * 6).reshape(ncell, 6)
    s.v_f = cells_from_file(blk[:, 0:3], num, 3)
    s.p_f = cells_from_file(blk[:, 3], num)
    s.phi = cells_from_file(blk[:, 4], num)
    s.dphi = cells_from_file(blk[:, 5], num) / (s.time_dt * ndem_before)
    s.rho_f = r.take(numpy.float64, 1)
    s.p_mod_A = r.take(numpy.float64, 1)
    s.p_mod_f = r.take(numpy.float64, 1)
    s.p_mod_phi = r.take(numpy.float64, 1)
    if version >= 2.12 and solver == 1:   # the sides: Darcy only
        for name in ("bc_xn", "bc_xp", "bc_yn", "bc_yp"):
            setattr(s, name, r.take(numpy.int32, 1))
    for name in ("bc_bot", "bc_top", "free_slip_bot", "free_slip_top"):
        setattr(s, name, r.take(numpy.int32, 1))
    if version >= 2.11:
        s.bc_bot_flux = r.take(numpy.float64, 1)
        s.bc_top_flux = r.take(numpy.float64, 1)
    else:
        s.bc_bot_flux = numpy.zeros(1, dtype=numpy.float64)
        s.bc_top_flux = numpy.zeros(1, dtype=numpy.float64)
    if version >= 2.15:
        s.p_f_constant = cells_from_file(r.take(numpy.int32, ncell), num)
    else:
        s.p_f_constant = numpy.zeros(num, dtype=numpy.int32)
    if version < 2.0:
        return
    if solver == 0:
        s.gamma = r.take(numpy.float64, 1)
        s.theta = r.take(numpy.float64, 1)
        s.beta = r.take(numpy.float64, 1)
        s.tolerance = r.take(numpy.float64, 1)
        s.maxiter = r.take(numpy.uint32, 1)
        s.ndem = r.take(numpy.uint32, 1)
        s.c_phi = r.take(numpy.float64, 1)
        s.c_v = r.take(numpy.float64, 1)
        s.dt_dem_fac = r.take(numpy.float64, 1)
        for name in ("f_d", "f_p", "f_v", "f_sum"):
            setattr(s, name, r.take(numpy.float64, n * 3).reshape(n, 3))
        return
    s.tolerance = r.take(numpy.float64, 1)
    s.maxiter = r.take(numpy.uint32, 1)
    s.ndem = r.take(numpy.uint32, 1)
    s.c_phi = r.take(numpy.float64, 1)
    s.f_p = r.take(numpy.float64, n * 3).reshape(n, 3)
    s.beta_f = r.take(numpy.float64, 1)
    s.k_c = r.take(numpy.float64, 1)


def read_bin(target, sim, verbose=False, fluid=None):
    """Read a sphere .bin file into the attributes of `sim`
    (python/sphere.py:965 readbin).  As in the reference, whether the file
    holds a fluid block is the sim's `fluid` flag (or `fluid` when given)."""
    if fluid is None:
        fluid = bool(getattr(sim, "fluid", False))
    if verbose:
        print("Input file: {0}".format(target))
    with open(target, "rb") as fh:
        r = _Reader(fh.read())
    s = sim
    s.version = r.take(numpy.float64, 1)
    s.nd = r.take(numpy.int32, 1)
    s.np = r.take(numpy.uint32, 1)
    nd = int(s.nd[0])
    n = int(s.np[0])
    if nd != 3:
        raise ValueError("only 3-D files are supported (nd = %d)" % nd)
    s.time_dt = r.take(numpy.float64, 1)
    s.time_current = r.take(numpy.float64, 1)
    s.time_total = r.take(numpy.float64, 1)
    s.time_file_dt = r.take(numpy.float64, 1)
    s.time_step_count = r.take(numpy.uint32, 1)
    s.origo = r.take(numpy.float64, nd)
    s.L = r.take(numpy.float64, nd)
    s.num = r.take(numpy.uint32, nd)
    s.periodic = r.take(numpy.int32, 1)
    if s.version[0] >= 2.14:
        s.adaptive = r.take(numpy.int32, 1)
    else:
        s.adaptive = numpy.zeros(1, dtype=numpy.float64)
    xr = r.take(numpy.float64, n * (nd + 1)).reshape(n, nd + 1)
    s.x = numpy.ascontiguousarray(xr[:, :nd])
    s.radius = numpy.ascontiguousarray(xr[:, nd])
    if s.version[0] >= 1.03:
        s.xyzsum = r.take(numpy.float64, n * 3).reshape(n, 3)
    else:
        s.xyzsum = r.take(numpy.float64, n * 2).reshape(n, 2)
    vr = r.take(numpy.float64, n * (nd + 1)).reshape(n, nd + 1)
    s.vel = numpy.ascontiguousarray(vr[:, :nd])
    s.fixvel = numpy.ascontiguousarray(vr[:, nd])
    s.force = r.take(numpy.float64, n * nd).reshape(n, nd)
    s.angpos = r.take(numpy.float64, n * nd).reshape(n, nd)
    s.angvel = r.take(numpy.float64, n * nd).reshape(n, nd)
    s.torque = r.take(numpy.float64, n * nd).reshape(n, nd)
    s.es_dot = r.take(numpy.float64, n)
    s.es = r.take(numpy.float64, n)
    s.ev_dot = r.take(numpy.float64, n)
    s.ev = r.take(numpy.float64, n)
    s.p = r.take(numpy.float64, n)
    s.g = r.take(numpy.float64, nd)
    s.k_n = r.take(numpy.float64, 1)
    s.k_t = r.take(numpy.float64, 1)
    s.k_r = r.take(numpy.float64, 1)
    if s.version[0] >= 2.13:
        s.E = r.take(numpy.float64, 1)
    else:
        s.E = numpy.zeros(1, dtype=numpy.float64)
    for name in ("gamma_n", "gamma_t", "gamma_r", "mu_s", "mu_d", "mu_r", "gamma_wn",
                 "gamma_wt", "mu_ws", "mu_wd", "rho"):
        setattr(s, name, r.take(numpy.float64, 1))
    s.contactmodel = r.take(numpy.uint32, 1)
    s.kappa = r.take(numpy.float64, 1)
    s.db = r.take(numpy.float64, 1)
    s.V_b = r.take(numpy.float64, 1)
    s.nw = r.take(numpy.uint32, 1)
    nw = int(s.nw[0])
    s.wmode = r.take(numpy.int32, nw)
    wn = r.take(numpy.float64, nw * (nd + 1)).reshape(nw, nd + 1)
    s.w_n = numpy.ascontiguousarray(wn[:, :nd])
    s.w_x = numpy.ascontiguousarray(wn[:, nd])
    wm = r.take(numpy.float64, nw * 4).reshape(nw, 4)
    s.w_m = numpy.ascontiguousarray(wm[:, 0])
    s.w_vel = numpy.ascontiguousarray(wm[:, 1])
    s.w_force = numpy.ascontiguousarray(wm[:, 2])
    s.w_sigma0 = numpy.ascontiguousarray(wm[:, 3])
    s.w_sigma0_A = r.take(numpy.float64, 1)
    s.w_sigma0_f = r.take(numpy.float64, 1)
    if s.version[0] >= 2.1:
        s.w_tau_x = r.take(numpy.float64, 1)
    else:
        s.w_tau_x = numpy.zeros(1, dtype=numpy.float64)
    s.lambda_bar = r.take(numpy.float64, 1)
    s.nb0 = r.take(numpy.uint32, 1)
    s.sigma_b = r.take(numpy.float64, 1)
    s.tau_b = r.take(numpy.float64, 1)
    nb0 = int(s.nb0[0])
    s.bonds = r.take(numpy.uint32, nb0 * 2).reshape(nb0, 2)
    s.bonds_delta_n = r.take(numpy.float64, nb0)
    s.bonds_delta_t = r.take(numpy.float64, nb0 * nd).reshape(nb0, nd)
    s.bonds_omega_n = r.take(numpy.float64, nb0)
    s.bonds_omega_t = r.take(numpy.float64, nb0 * nd).reshape(nb0, nd)
    if fluid:
        s.fluid = True
        _read_darcy(r, s, n)
    if s.version[0] >= 1.02:
        s.color = r.take(numpy.int32, n)
    else:
        s.color = numpy.zeros(n, dtype=numpy.int32)
    s.version[0] = VERSION
    return s


def _f64(a):
    return numpy.ascontiguousarray(numpy.asarray(a), dtype=numpy.float64).tobytes()


def _u32(a):
    return numpy.ascontiguousarray(numpy.asarray(a).astype(numpy.uint32)).tobytes()


def _i32(a):
    return numpy.ascontiguousarray(numpy.asarray(a).astype(numpy.int32)).tobytes()


def _encode_darcy(s, w, dphi_raw=None):
    """The fluid block in the order of python/sphere.py:1471-1539 and
    src/file_io.cpp:577-716: the Darcy solver's (cfd_solver 1), or the
    Navier-Stokes solver's (cfd_solver 0: no side codes, then gamma, theta,
    beta, tolerance, maxiter, ndem, c_phi, c_v, dt_dem_fac and the drag,
    pressure, viscous and total fluid forces).  dphi goes to the file as
    dphi * time_dt * ndem (the reference's Python writer); dphi_raw, when
    given, is written as it is (the values of the solver, as its C++ writer
    writes them)."""
    solver = int(numpy.asarray(s.cfd_solver).ravel()[0])
    if solver not in (0, 1):
        raise ValueError("Value of cfd_solver not understood (%d)" % solver)
    n = int(s.np[0])
    w(_i32(numpy.asarray(s.cfd_solver).ravel()[:1]))
    w(_f64(s.mu))
    if dphi_raw is None:
        dphi_raw = numpy.asarray(s.dphi, dtype=numpy.float64) * s.time_dt * s.ndem
    num = [int(v) for v in s.num]
    ncell = num[0] * num[1] * num[2]
    blk = numpy.empty((ncell, 6))
    blk[:, 0:3] = cells_to_file(s.v_f).reshape(ncell, 3)
    blk[:, 3] = cells_to_file(s.p_f).reshape(ncell)
    blk[:, 4] = cells_to_file(s.phi).reshape(ncell)
    blk[:, 5] = cells_to_file(dphi_raw).reshape(ncell)
    w(blk.tobytes())
    for name in ("rho_f", "p_mod_A", "p_mod_f", "p_mod_phi"):
        w(_f64(getattr(s, name)))
    sides = ("bc_xn", "bc_xp", "bc_yn", "bc_yp") if solver == 1 else ()
    for name in sides + ("bc_bot", "bc_top", "free_slip_bot", "free_slip_top"):
        w(_i32(getattr(s, name)))
    w(_f64(s.bc_bot_flux))
    w(_f64(s.bc_top_flux))
    w(_i32(cells_to_file(s.p_f_constant).reshape(ncell)))
    if solver == 0:
        for name in ("gamma", "theta", "beta", "tolerance"):
            w(_f64(numpy.asarray(getattr(s, name)).ravel()[:1]))
        w(_u32(numpy.asarray(s.maxiter).ravel()[:1]))
        w(_u32(numpy.asarray(s.ndem).ravel()[:1]))
        for name in ("c_phi", "c_v", "dt_dem_fac"):
            w(_f64(numpy.asarray(getattr(s, name)).ravel()[:1]))
        for name in ("f_d", "f_p", "f_v", "f_sum"):
            w(_f64(numpy.asarray(getattr(s, name), dtype=numpy.float64).reshape(-1, 3)[:n]))
        return
    w(_f64(numpy.asarray(s.tolerance).ravel()[:1]))
    w(_u32(numpy.asarray(s.maxiter).ravel()[:1]))
    w(_u32(numpy.asarray(s.ndem).ravel()[:1]))
    w(_f64(s.c_phi))
    w(_f64(numpy.asarray(s.f_p, dtype=numpy.float64).reshape(-1, 3)[:n]))
    w(_f64(s.beta_f))
    w(_f64(s.k_c))


def encode_bin(sim, dphi_raw=None):
    """Bytes of `sim` in the .bin layout of python/sphere.py:1355 writebin
    (with the Darcy fluid block when sim.fluid)."""
    s = sim
    n = int(s.np[0])
    nd = int(s.nd[0])
    out = []
    w = out.append
    w(_f64(s.version))
    w(_i32(s.nd))
    w(_u32(s.np))
    w(_f64(s.time_dt))
    w(_f64(s.time_current))
    w(_f64(s.time_total))
    w(_f64(s.time_file_dt))
    w(_u32(s.time_step_count))
    w(_f64(s.origo))
    w(_f64(s.L))
    w(_u32(s.num))
    w(_u32(s.periodic))
    w(_u32(s.adaptive))
    xr = numpy.empty((n, nd + 1))
    xr[:, :nd] = s.x
    xr[:, nd] = s.radius
    w(xr.tobytes())
    if n > 0:
        w(_f64(s.xyzsum))
    vr = numpy.empty((n, nd + 1))
    vr[:, :nd] = s.vel
    vr[:, nd] = s.fixvel
    w(vr.tobytes())
    if n > 0:
        for name in ("force", "angpos", "angvel", "torque", "es_dot", "es", "ev_dot", "ev", "p"):
            w(_f64(getattr(s, name)))
    w(_f64(s.g))
    for name in ("k_n", "k_t", "k_r", "E", "gamma_n", "gamma_t", "gamma_r", "mu_s", "mu_d",
                 "mu_r", "gamma_wn", "gamma_wt", "mu_ws", "mu_wd", "rho"):
        w(_f64(getattr(s, name)))
    w(_u32(s.contactmodel))
    w(_f64(s.kappa))
    w(_f64(s.db))
    w(_f64(s.V_b))
    nw = int(s.nw[0])
    w(_u32(s.nw))
    w(_i32(numpy.asarray(s.wmode)[:nw]))
    wn = numpy.empty((nw, nd + 1))
    wn[:, :nd] = numpy.asarray(s.w_n)[:nw]
    wn[:, nd] = numpy.asarray(s.w_x)[:nw]
    w(wn.tobytes())
    wm = numpy.empty((nw, 4))
    wm[:, 0] = numpy.asarray(s.w_m)[:nw]
    wm[:, 1] = numpy.asarray(s.w_vel)[:nw]
    wm[:, 2] = numpy.asarray(s.w_force)[:nw]
    wm[:, 3] = numpy.asarray(s.w_sigma0)[:nw]
    w(wm.tobytes())
    w(_f64(s.w_sigma0_A))
    w(_f64(s.w_sigma0_f))
    w(_f64(s.w_tau_x))
    w(_f64(s.lambda_bar))
    nb0 = int(s.nb0[0])
    w(_u32(s.nb0))
    w(_f64(s.sigma_b))
    w(_f64(s.tau_b))
    w(_u32(numpy.asarray(s.bonds).reshape(-1, 2)[:nb0]))
    w(_f64(numpy.asarray(s.bonds_delta_n).reshape(-1)[:nb0]))
    w(_f64(numpy.asarray(s.bonds_delta_t).reshape(-1, 3)[:nb0]))
    w(_f64(numpy.asarray(s.bonds_omega_n).reshape(-1)[:nb0]))
    w(_f64(numpy.asarray(s.bonds_omega_t).reshape(-1, 3)[:nb0]))
    if getattr(s, "fluid", False):
        _encode_darcy(s, w, dphi_raw)
    w(_i32(s.color))
    return b"".join(out)


def write_bin(target, sim, dphi_raw=None):
    """Write `sim` to `target` (python/sphere.py:1355 writebin layout)."""
    data = encode_bin(sim, dphi_raw)
    with open(target, "wb") as fh:
        fh.write(data)
    return len(data)
