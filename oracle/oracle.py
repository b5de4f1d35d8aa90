"""TEST INFRASTRUCTURE ONLY: Python driver of the CPU oracles.

Two CPU implementations of the reference's DEM step share one state layout
(oracle/sphere_oracle.h):
  * 'oracle' -- oracle/_build/libsphere_oracle.so, the C restatement
    (oracle/sphere_oracle.c);
  * 'ref'    -- oracle/_ref/libsphere_ref.so, the reference's own kernels
    compiled for the CPU (oracle/ref_emu/ref_harness.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference
legs use this module, as the checker; the product never imports it.
"""
import ctypes as C
import sys
import os
import subprocess

import numpy

from sphere_b200._abi import NC, SphBox, SphDarcy, box_from_sim, darcy_from_sim

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "oracle": os.path.join(HERE, "_build", "libsphere_oracle.so"),
    "ref": os.path.join(HERE, "_ref", "libsphere_ref.so"),
}
ENTRY = {"oracle": "or_step", "ref": "ref_step"}

_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)
_bp = C.POINTER(C.c_uint8)


class OrDarcy(C.Structure):
    _fields_ = [
        ("prm", SphDarcy),
        ("p", _dp), ("p_old", _dp), ("p_new", _dp), ("dp_expl", _dp), ("phi", _dp),
        ("dphi", _dp), ("norm", _dp), ("k", _dp), ("div_v_p", _dp),
        ("v", _dp), ("vp_avg", _dp), ("grad_k", _dp), ("grad_p", _dp),
        ("p_constant", C.POINTER(C.c_int32)),
        ("f_p", _dp),
        ("p_top_orig", C.c_double), ("filetimeclock", C.c_double), ("wall_w_host", C.c_double),
        ("wall0_iz", C.c_uint32), ("log_cap", C.c_uint32), ("log_n", C.c_uint32),
        ("log_step", C.POINTER(C.c_uint64)), ("log_iters", _up), ("log_ok", _up),
    ]


class OrState(C.Structure):
    _fields_ = [
        ("box", SphBox),
        ("length_mode", C.c_int32), ("velocity_state", C.c_int32),
        ("iter", C.c_uint64),
        ("error_flags", C.c_int32), ("nthreads", C.c_int32),
        ("x", _dp), ("xyzsum", _dp), ("vel", _dp), ("force", _dp), ("angpos", _dp),
        ("angvel", _dp), ("torque", _dp), ("acc", _dp), ("angacc", _dp),
        ("es_dot", _dp), ("es", _dp), ("ev_dot", _dp), ("ev", _dp), ("p", _dp),
        ("contacts", _up), ("distmod", _dp), ("delta_t", _dp),
        ("bonds", _up), ("bonds_delta", _dp), ("bonds_omega", _dp), ("bonds_broken", _bp),
        ("walls_acc", C.c_double * 6),
        ("cell_id", _up), ("perm", _up), ("cell_start", _up), ("cell_end", _up),
        ("x_sorted", _dp), ("vel_sorted", _dp), ("angvel_sorted", _dp),
        ("walls_force_pp", _dp), ("walls_force_partial", _dp),
        ("tau_eff_x_pp", _dp), ("tau_eff_x_partial", _dp),
        ("darcy", C.POINTER(OrDarcy)),
    ]


_loaded = {}


def reference_root():
    """The reference's checkout: $SPHERE_REFERENCE, else a directory named
    'reference' beside this repository; None when neither exists (the
    reference builds and the tests that read its files are then skipped)."""
    cand = os.environ.get("SPHERE_REFERENCE") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference")
    return cand if os.path.isdir(os.path.join(cand, "src")) else None


def build():
    """Compile the CPU oracles in place (make -C oracle); the reference's
    kernels too when its checkout is found (reference_root)."""
    env = dict(os.environ)
    root = reference_root()
    if root:
        env["SPHERE_REFERENCE"] = root
    subprocess.check_call(["make", "-s", "-C", HERE], env=env)


def available(which):
    return os.path.exists(LIBS[which])


def _lib(which):
    if which not in _loaded:
        if not os.path.exists(LIBS[which]):
            build()
        lib = C.CDLL(LIBS[which])
        fn = getattr(lib, ENTRY[which])
        fn.argtypes = [C.POINTER(OrState), C.c_uint64]
        fn.restype = C.c_int
        _loaded[which] = fn
    return _loaded[which]


def _f4(a3, w=None):
    a3 = numpy.asarray(a3, dtype=numpy.float64).reshape(-1, 3)
    out = numpy.zeros((a3.shape[0], 4))
    out[:, :3] = a3
    if w is not None:
        out[:, 3] = w
    return out


class CpuRun(object):
    """One simulation box stepped by a CPU oracle.  All arrays are numpy
    arrays in the reference's device layouts and may be inspected after
    each call to step()."""

    def __init__(self, s, which="oracle", length_mode=0, nthreads=0):
        self.which = which
        self.fn = _lib(which)
        n = int(s.np[0])
        nb0 = int(s.nb0[0])
        nw = int(s.nw[0])
        self.n = n
        self.x = _f4(s.x, s.radius)
        self.xyzsum = _f4(s.xyzsum)
        self.vel = _f4(s.vel, s.fixvel)
        self.force = _f4(s.force)
        self.angpos = _f4(s.angpos)
        self.angvel = _f4(s.angvel)
        self.torque = _f4(s.torque)
        self.acc = numpy.zeros((n, 4))
        self.angacc = numpy.zeros((n, 4))
        self.es_dot = numpy.array(s.es_dot, dtype=numpy.float64)
        self.es = numpy.array(s.es, dtype=numpy.float64)
        self.ev_dot = numpy.array(s.ev_dot, dtype=numpy.float64)
        self.ev = numpy.array(s.ev, dtype=numpy.float64)
        self.p = numpy.array(s.p, dtype=numpy.float64)
        self.contacts = numpy.full(n * NC, n, dtype=numpy.uint32)
        self.distmod = numpy.zeros((n * NC, 4))
        self.delta_t = numpy.zeros((n * NC, 4))
        self.bonds = numpy.array(numpy.asarray(s.bonds).reshape(-1, 2)[:nb0], dtype=numpy.uint32)
        self.bonds_delta = numpy.zeros((max(nb0, 1), 4))
        self.bonds_omega = numpy.zeros((max(nb0, 1), 4))
        if nb0:
            self.bonds_delta[:nb0, :3] = numpy.asarray(s.bonds_delta_t).reshape(-1, 3)[:nb0]
            self.bonds_delta[:nb0, 3] = numpy.asarray(s.bonds_delta_n).reshape(-1)[:nb0]
            self.bonds_omega[:nb0, :3] = numpy.asarray(s.bonds_omega_t).reshape(-1, 3)[:nb0]
            self.bonds_omega[:nb0, 3] = numpy.asarray(s.bonds_omega_n).reshape(-1)[:nb0]
        if self.bonds.size == 0:
            self.bonds = numpy.zeros((1, 2), dtype=numpy.uint32)
        self.bonds_broken = numpy.zeros(max(nb0, 1), dtype=numpy.uint8)
        ncells = int(s.num[0]) * int(s.num[1]) * int(s.num[2])
        self.cell_id = numpy.zeros(max(n, 1), dtype=numpy.uint32)
        self.perm = numpy.zeros(max(n, 1), dtype=numpy.uint32)
        self.cell_start = numpy.full(ncells, 0xffffffff, dtype=numpy.uint32)
        self.cell_end = numpy.zeros(ncells, dtype=numpy.uint32)
        self.x_sorted = numpy.zeros((max(n, 1), 4))
        self.vel_sorted = numpy.zeros((max(n, 1), 4))
        self.angvel_sorted = numpy.zeros((max(n, 1), 4))
        blocks = max((n + 255) // 256, 1)
        self.walls_force_pp = numpy.zeros(max(nw * n, 1))
        self.walls_force_partial = numpy.zeros(blocks)
        self.tau_eff_x_pp = numpy.zeros(max(n, 1))
        self.tau_eff_x_partial = numpy.zeros(blocks)
        st = OrState()
        st.box = box_from_sim(s)
        st.length_mode = int(length_mode)
        st.velocity_state = 1
        st.iter = 0
        st.error_flags = 0
        st.nthreads = int(nthreads)
        for name, _t in OrState._fields_:
            if name in ("box", "length_mode", "velocity_state", "iter", "error_flags",
                        "nthreads", "walls_acc", "darcy"):
                continue
            a = getattr(self, name)
            ct = dict(OrState._fields_)[name]
            setattr(st, name, a.ctypes.data_as(ct))
        self.state = st
        self.darcy = None
        if getattr(s, "fluid", False):
            self._darcy_init(s)

    # ---------------------------------------------------------- Darcy
    _CELL1 = ("p", "p_old", "p_new", "dp_expl", "phi", "dphi", "norm", "k", "div_v_p")
    _CELL3 = ("v", "vp_avg", "grad_k", "grad_p")

    def _darcy_init(self, s, log_cap=100000):
        """Ghost-padded fluid fields of a Darcy sim ([z+2, y+2, x+2](, 3))
        and the start-of-run set-up (or_darcy_start)."""
        num = [int(v) for v in s.num]
        self.num = num
        shape = (num[2] + 2, num[1] + 2, num[0] + 2)
        f = {}
        for name in self._CELL1:
            f[name] = numpy.zeros(shape)
        for name in self._CELL3:
            f[name] = numpy.zeros(shape + (3,))
        f["p_constant"] = numpy.zeros(shape, dtype=numpy.int32)
        inner = (slice(1, -1), slice(1, -1), slice(1, -1))
        t = lambda a: numpy.asarray(a).transpose((2, 1, 0) + tuple(range(3, numpy.ndim(a))))
        f["p"][inner] = t(s.p_f)
        f["v"][inner] = t(s.v_f)
        f["phi"][inner] = t(s.phi)
        f["dphi"][inner] = t(numpy.asarray(s.dphi, dtype=numpy.float64) * s.time_dt * s.ndem)
        f["p_constant"][inner] = t(s.p_f_constant)
        f["f_p"] = numpy.zeros((max(self.n, 1), 4))
        if self.n:
            f["f_p"][:self.n, :3] = numpy.asarray(s.f_p, dtype=numpy.float64).reshape(-1, 3)
        f["log_step"] = numpy.zeros(log_cap, dtype=numpy.uint64)
        f["log_iters"] = numpy.zeros(log_cap, dtype=numpy.uint32)
        f["log_ok"] = numpy.zeros(log_cap, dtype=numpy.uint32)
        d = OrDarcy()
        d.prm = darcy_from_sim(s)
        for name, ct in OrDarcy._fields_:
            if name in f:
                setattr(d, name, f[name].ctypes.data_as(ct))
        d.log_cap = log_cap
        self.fluid = f
        self.darcy = d
        self.state.darcy = C.pointer(d)
        lib = C.CDLL(LIBS["oracle"])
        lib.or_darcy_start.argtypes = [C.POINTER(OrState)]
        lib.or_darcy_start(C.byref(self.state))

    def fluid_cells(self, name):
        """A fluid field without its ghost layer, in the sim's [x, y, z](, 3)
        layout."""
        a = self.fluid[name][1:-1, 1:-1, 1:-1]
        return numpy.ascontiguousarray(a.transpose((2, 1, 0) + tuple(range(3, a.ndim))))

    def darcy_log(self):
        n = int(self.darcy.log_n)
        return (self.fluid["log_step"][:n].copy(), self.fluid["log_iters"][:n].copy(),
                self.fluid["log_ok"][:n].copy())

    def step(self, nsteps=1):
        """Run nsteps steps; returns the accumulated error-flag bits."""
        return self.fn(C.byref(self.state), int(nsteps))

    @property
    def box(self):
        return self.state.box

    def contact_rows(self):
        return self.contacts.reshape(self.n, NC)

    def to_sim(self, s):
        """Copy the state back into a sim object (as a .bin output would)."""
        s.x = self.x[:, :3].copy()
        s.radius = self.x[:, 3].copy()
        s.xyzsum = self.xyzsum[:, :3].copy()
        s.vel = self.vel[:, :3].copy()
        s.fixvel = self.vel[:, 3].copy()
        s.force = self.force[:, :3].copy()
        s.angpos = self.angpos[:, :3].copy()
        s.angvel = self.angvel[:, :3].copy()
        s.torque = self.torque[:, :3].copy()
        for name in ("es_dot", "es", "ev_dot", "ev", "p"):
            setattr(s, name, getattr(self, name).copy())
        nb0 = int(s.nb0[0])
        if nb0:
            s.bonds = self.bonds[:nb0].copy()
            s.bonds_delta_t = self.bonds_delta[:nb0, :3].copy()
            s.bonds_delta_n = self.bonds_delta[:nb0, 3].copy()
            s.bonds_omega_t = self.bonds_omega[:nb0, :3].copy()
            s.bonds_omega_n = self.bonds_omega[:nb0, 3].copy()
        b = self.state.box
        s.L[2] = b.grid.L[2]
        for i in range(int(b.walls.nw)):
            s.w_x[i] = b.walls.nx[i][3]
            s.w_vel[i] = b.walls.mvfd[i][1]
            s.w_force[i] = b.walls.mvfd[i][2]
        s.time_current[0] = b.t_current
        return s


# ------------------------------------------------------------------ analysis

def _alib():
    lib = C.CDLL(LIBS["oracle"])
    dp = C.POINTER(C.c_double)
    lib.or_porosity.argtypes = [dp, C.c_uint32, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_uint32, dp, dp]
    lib.or_porosity.restype = C.c_int
    lib.or_overlaps.argtypes = [dp, dp, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32), dp]
    lib.or_overlaps.restype = C.c_uint64
    lib.or_render.argtypes = [dp, dp, dp, dp, dp, dp, C.c_uint32, dp, C.c_int, C.c_float,
                              C.c_float, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint8)]
    lib.or_render.restype = None
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def porosity(s, slices):
    """DEM::porosity of sim s (src/sphere.cpp:487-606) by the C restatement:
    (z positions, porosities), or None where the reference exits."""
    x = _f4(s.x, s.radius)
    top = float(s.w_x[0]) if int(s.nw[0]) > 0 else float(s.L[2])
    z = numpy.zeros(slices)
    p = numpy.zeros(slices)
    st = _alib().or_porosity(_dp(x), int(s.np[0]), top, float(s.origo[2]), float(s.L[0]),
                             float(s.L[1]), int(slices), _dp(z), _dp(p))
    return None if st != 0 else (z, p)


def overlaps(s):
    """DEM::findOverlaps of sim s (src/sphere.cpp:677-725) by the C
    restatement: (pairs [n, 2] uint32, delta_n [n])."""
    x = _f4(s.x, s.radius)
    v = _f4(s.vel, s.fixvel)
    lib = _alib()
    n = int(lib.or_overlaps(_dp(x), _dp(v), int(s.np[0]), 0, None, None))
    pairs = numpy.zeros((max(n, 1), 2), dtype=numpy.uint32)
    d = numpy.zeros(max(n, 1))
    lib.or_overlaps(_dp(x), _dp(v), int(s.np[0]), n, pairs.ctypes.data_as(C.POINTER(C.c_uint32)),
                    _dp(d))
    return pairs[:n], d[:n]


def render(s, method=1, maxval=1.0e3, lower_cutoff=0.0, width=800, height=800):
    """DEM::render of sim s (src/raytracer.cuh:379-560) by the C
    restatement, every sphere tested for every pixel: [height, width, 3]
    uint8."""
    x = _f4(s.x, s.radius)
    v = _f4(s.vel, s.fixvel)
    av = _f4(s.angvel, numpy.zeros(len(s.radius)))
    ap = _f4(s.angpos, numpy.zeros(len(s.radius)))
    xs = _f4(s.xyzsum, numpy.zeros(len(s.radius)))
    p = numpy.ascontiguousarray(s.p, dtype=numpy.float64)
    L = numpy.ascontiguousarray(s.L, dtype=numpy.float64)
    img = numpy.zeros((int(height), int(width), 3), dtype=numpy.uint8)
    _alib().or_render(_dp(x), _dp(v), _dp(av), _dp(ap), _dp(xs), _dp(p), int(s.np[0]), _dp(L),
                      int(method), float(maxval), float(lower_cutoff), int(width), int(height),
                      img.ctypes.data_as(C.POINTER(C.c_uint8)))
    return img


def reference_analysis(s, what, slices=10, workdir=None):
    """Run the reference's own analysis code (oracle/_ref/sphere_analysis_ref)
    on sim s written as a .bin file; None when it is not built.  Returns
    (z, porosity) for what='porosity', (pairs, delta_n) for 'contacts'."""
    import os
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "_ref", "sphere_analysis_ref")
    if not os.path.exists(exe):
        return None
    sys.path.insert(0, os.path.dirname(HERE))
    from sphere_b200 import binio
    d = workdir or tempfile.mkdtemp()
    path = os.path.join(d, "analysis.bin")
    binio.write_bin(path, s)
    args = [exe, what, path] + ([str(slices)] if what == "porosity" else [])
    out = subprocess.run(args, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(out.stderr)
    rows = [r.split("\t") for r in out.stdout.strip().splitlines() if r.strip()]
    if what == "porosity":
        a = numpy.array([[float(c) for c in r] for r in rows])
        return a[:, 0], a[:, 1]
    if not rows:
        return numpy.zeros((0, 2), dtype=numpy.uint32), numpy.zeros(0)
    pairs = numpy.array([[int(r[0]), int(r[1])] for r in rows], dtype=numpy.uint32)
    return pairs, numpy.array([float(r[2]) for r in rows])


def reference_render(s, method=1, maxval=1.0e3, lower_cutoff=0.0, width=800, height=800,
                     workdir=None):
    """Run the reference's own ray-tracer kernels and camera
    (oracle/_ref/sphere_render_ref) on sim s written as a .bin file: the
    image [height, width, 3] uint8, or None when the program is not built.
    maxval and lower_cutoff travel as text with 9 significant digits, which
    the program's atof reads back to the same float."""
    import os
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "_ref", "sphere_render_ref")
    if not os.path.exists(exe):
        return None
    sys.path.insert(0, os.path.dirname(HERE))
    from sphere_b200 import binio
    d = workdir or tempfile.mkdtemp()
    path = os.path.join(d, "render.bin")
    out = os.path.join(d, "render.rgb")
    binio.write_bin(path, s)
    args = [exe, path, str(int(method)), "%.9g" % numpy.float32(maxval),
            "%.9g" % numpy.float32(lower_cutoff), str(int(width)), str(int(height)), out]
    r = subprocess.run(args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    return numpy.fromfile(out, dtype=numpy.uint8).reshape(int(height), int(width), 3)


def relax(s, sweeps, alpha=0.6, z_top=1e300, nthreads=0):
    """The packing sweeps of sph_relax (sphere_b200 scene preparation) on
    the CPU, restated in C (or_relax): moves s.x in place for one box and
    returns the largest overlap of the last sweep.  Bit for bit the GPU's
    result (the checker of sph_relax, and the CPU packer of bench.py's
    reference arm)."""
    lib = C.CDLL(LIBS["oracle"])
    dp = C.POINTER(C.c_double)
    lib.or_relax.argtypes = [dp, C.c_uint32, dp, dp, C.POINTER(C.c_uint32), C.c_int, C.c_uint32,
                             C.c_double, C.c_double, C.c_int, dp]
    lib.or_relax.restype = None
    x = _f4(s.x, s.radius)
    origo = numpy.ascontiguousarray(s.origo, dtype=numpy.float64)
    L = numpy.ascontiguousarray(s.L, dtype=numpy.float64)
    num = numpy.ascontiguousarray(s.num, dtype=numpy.uint32)
    worst = C.c_double(0.0)
    lib.or_relax(_dp(x), int(s.np[0]), _dp(origo), _dp(L), num.ctypes.data_as(C.POINTER(C.c_uint32)),
                 int(s.periodic[0]), int(sweeps), float(alpha), float(z_top), int(nthreads),
                 C.byref(worst))
    s.x = x[:, :3].copy()
    return worst.value
