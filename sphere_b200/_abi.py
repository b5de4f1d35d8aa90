"""ctypes mirror of include/sphere_b200.h and loader of the CUDA library.

The structures below must match the C header field for field; tests check
their sizes against the library (``sph_struct_sizes``).
"""
import ctypes as C
import os

import numpy

NC = 32
MAXWALLS = 6
TUNE_VARIANTS = 5   # SPH_TUNE_VARIANTS: launch variants sph_autotune times
PAIR_SHAPES = 13    # SPH_PAIR_SHAPES: launch shapes of the list step (variant 4)
BIN_VERSION = 2.15

SPH_OK = 0
SPH_ERR_INPUT = 1
SPH_ERR_CUDA = 2
SPH_ERR_NC_OVERFLOW = 3
SPH_ERR_OUT_OF_GRID = 4
SPH_ERR_NAN = 5
SPH_ERR_NOMEM = 6
SPH_ERR_STATE = 7
SPH_ERR_UNSUPPORTED = 8

STATUS_NAMES = {
    0: "SPH_OK", 1: "SPH_ERR_INPUT", 2: "SPH_ERR_CUDA", 3: "SPH_ERR_NC_OVERFLOW",
    4: "SPH_ERR_OUT_OF_GRID", 5: "SPH_ERR_NAN", 6: "SPH_ERR_NOMEM",
    7: "SPH_ERR_STATE", 8: "SPH_ERR_UNSUPPORTED", 9: "SPH_ERR_TIMEOUT",
}

PREC_FP64 = 0
PREC_MIXED = 1
LEN_REFERENCE = 0
LEN_FP64 = 1


class SphParams(C.Structure):
    _fields_ = [
        ("g", C.c_double * 3),
        ("k_n", C.c_double), ("k_t", C.c_double), ("k_r", C.c_double), ("E", C.c_double),
        ("gamma_n", C.c_double), ("gamma_t", C.c_double), ("gamma_r", C.c_double),
        ("mu_s", C.c_double), ("mu_d", C.c_double), ("mu_r", C.c_double),
        ("gamma_wn", C.c_double), ("gamma_wt", C.c_double),
        ("mu_ws", C.c_double), ("mu_wd", C.c_double),
        ("rho", C.c_double),
        ("contactmodel", C.c_uint32), ("pad0", C.c_uint32),
        ("kappa", C.c_double), ("db", C.c_double), ("V_b", C.c_double),
        ("lambda_bar", C.c_double), ("sigma_b", C.c_double), ("tau_b", C.c_double),
        ("sigma0_A", C.c_double), ("sigma0_f", C.c_double),
    ]


class SphGrid(C.Structure):
    _fields_ = [
        ("origo", C.c_double * 3), ("L", C.c_double * 3), ("num", C.c_uint32 * 3),
        ("periodic", C.c_int32), ("adaptive", C.c_int32), ("pad0", C.c_int32),
    ]


class SphWalls(C.Structure):
    _fields_ = [
        ("nw", C.c_uint32), ("wmode", C.c_int32 * MAXWALLS), ("pad0", C.c_uint32),
        ("nx", (C.c_double * 4) * MAXWALLS), ("mvfd", (C.c_double * 4) * MAXWALLS),
        ("tau_x", C.c_double),
    ]


class SphBox(C.Structure):
    _fields_ = [
        ("grid", SphGrid), ("params", SphParams), ("walls", SphWalls),
        ("dt", C.c_double), ("t_current", C.c_double),
        ("np", C.c_uint32), ("nb0", C.c_uint32),
    ]


_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)


class SphParticles(C.Structure):
    _fields_ = [(n, _dp) for n in ("x", "xyzsum", "vel", "force", "angpos", "angvel", "torque",
                                  "es_dot", "es", "ev_dot", "ev", "p")]


class SphBonds(C.Structure):
    _fields_ = [("pairs", _up), ("delta_n", _dp), ("delta_t", _dp),
                ("omega_n", _dp), ("omega_t", _dp)]


class SphDarcy(C.Structure):
    _fields_ = [("mu", C.c_double), ("rho_f", C.c_double), ("beta_f", C.c_double),
                ("k_c", C.c_double), ("c_phi", C.c_double), ("tolerance", C.c_double),
                ("p_mod_A", C.c_double), ("p_mod_f", C.c_double), ("p_mod_phi", C.c_double),
                ("bc_bot_flux", C.c_double), ("bc_top_flux", C.c_double),
                ("file_dt", C.c_double),
                ("maxiter", C.c_uint32), ("ndem", C.c_uint32),
                ("bc_xn", C.c_int32), ("bc_xp", C.c_int32), ("bc_yn", C.c_int32),
                ("bc_yp", C.c_int32), ("bc_bot", C.c_int32), ("bc_top", C.c_int32),
                ("free_slip_bot", C.c_int32), ("free_slip_top", C.c_int32)]


DARCY_LOG = 4096   # SPH_DARCY_LOG


def darcy_from_sim(s):
    """The SphDarcy of a sim object with a Darcy fluid (cfd_solver 1)."""
    d = SphDarcy()
    for name in ("mu", "rho_f", "beta_f", "k_c", "c_phi", "p_mod_A", "p_mod_f", "p_mod_phi",
                 "bc_bot_flux", "bc_top_flux"):
        setattr(d, name, float(numpy.asarray(getattr(s, name)).ravel()[0]))
    d.tolerance = float(numpy.asarray(s.tolerance).ravel()[0])
    d.file_dt = float(s.time_file_dt[0])
    d.maxiter = int(numpy.asarray(s.maxiter).ravel()[0])
    d.ndem = int(numpy.asarray(s.ndem).ravel()[0])
    for name in ("bc_xn", "bc_xp", "bc_yn", "bc_yp", "bc_bot", "bc_top", "free_slip_bot",
                 "free_slip_top"):
        setattr(d, name, int(numpy.asarray(getattr(s, name)).ravel()[0]))
    return d


def cells_to_file(a):
    """A sim's cell array [nx, ny, nz(, k)] in the .bin order (x fastest)."""
    a = numpy.asarray(a)
    axes = (2, 1, 0) + tuple(range(3, a.ndim))
    return numpy.ascontiguousarray(a.transpose(axes))


def cells_from_file(flat, num, k=None):
    """The inverse of cells_to_file: [nx, ny, nz(, k)] from x-fastest data."""
    shape = (int(num[2]), int(num[1]), int(num[0])) + ((k,) if k else ())
    a = numpy.asarray(flat).reshape(shape)
    axes = (2, 1, 0) + tuple(range(3, a.ndim))
    return numpy.ascontiguousarray(a.transpose(axes))


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array (or NULL)."""
    if a is None:
        return C.cast(None, _dp)
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def uptr(a):
    if a is None:
        return C.cast(None, _up)
    assert a.dtype.name == "uint32" and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_up)


def box_from_sim(s):
    """Build an SphBox from a sim object (python/sphere.py attribute names)."""
    b = SphBox()
    g = b.grid
    for d in range(3):
        g.origo[d] = float(s.origo[d])
        g.L[d] = float(s.L[d])
        g.num[d] = int(s.num[d])
    g.periodic = int(s.periodic[0])
    g.adaptive = int(s.adaptive[0])
    p = b.params
    for d in range(3):
        p.g[d] = float(s.g[d])
    for name in ("k_n", "k_t", "k_r", "E", "gamma_n", "gamma_t", "gamma_r", "mu_s", "mu_d",
                 "mu_r", "gamma_wn", "gamma_wt", "mu_ws", "mu_wd", "rho", "kappa", "db",
                 "V_b", "lambda_bar", "sigma_b", "tau_b"):
        setattr(p, name, float(getattr(s, name)[0]))
    p.contactmodel = int(s.contactmodel[0])
    p.sigma0_A = float(s.w_sigma0_A[0])
    p.sigma0_f = float(s.w_sigma0_f[0])
    w = b.walls
    nw = int(s.nw[0])
    if nw > MAXWALLS:
        raise ValueError("nw = %d exceeds MAXWALLS = %d" % (nw, MAXWALLS))
    w.nw = nw
    for i in range(nw):
        w.wmode[i] = int(s.wmode[i])
        for d in range(3):
            w.nx[i][d] = float(s.w_n[i, d])
        w.nx[i][3] = float(s.w_x[i])
        w.mvfd[i][0] = float(s.w_m[i])
        w.mvfd[i][1] = float(s.w_vel[i])
        w.mvfd[i][2] = float(s.w_force[i])
        w.mvfd[i][3] = float(s.w_sigma0[i])
    w.tau_x = float(s.w_tau_x[0])
    b.dt = float(s.time_dt[0])
    b.t_current = float(s.time_current[0])
    b.np = int(s.np[0])
    b.nb0 = int(s.nb0[0])
    return b


def sim_from_box(s, b):
    """Copy the time-dependent box state (walls, adaptive L[2], time) to sim."""
    s.L[2] = b.grid.L[2]
    nw = int(b.walls.nw)
    for i in range(nw):
        s.w_x[i] = b.walls.nx[i][3]
        s.w_m[i] = b.walls.mvfd[i][0]
        s.w_vel[i] = b.walls.mvfd[i][1]
        s.w_force[i] = b.walls.mvfd[i][2]
        s.w_sigma0[i] = b.walls.mvfd[i][3]
    s.time_current[0] = b.t_current


_LIB = None
LIB_NAME = "libsphere_b200.so"


def lib_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)


def load_library():
    """Load the in-tree CUDA library.  Raises if it is missing: there is no
    CPU fallback for the step."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError(
            "sphere_b200: CUDA library %s is missing; build it with "
            "`python -m sphere_b200.build` (nvcc, sm_100a)" % path)
    lib = C.CDLL(path)
    H = C.c_void_p
    lib.sph_create.argtypes = [C.POINTER(SphBox), C.c_uint32, C.c_int, C.c_int, C.c_int,
                               C.POINTER(H)]
    lib.sph_upload.argtypes = [H, C.POINTER(SphParticles), C.POINTER(SphBonds)]
    lib.sph_step.argtypes = [H, C.c_uint64]
    lib.sph_advance.argtypes = [H, C.c_double, C.c_double, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.c_uint64, C.POINTER(C.c_uint64)]
    lib.sph_download.argtypes = [H, C.POINTER(SphParticles), C.POINTER(SphBonds)]
    lib.sph_get_boxes.argtypes = [H, C.POINTER(SphBox)]
    lib.sph_get_contacts.argtypes = [H, _up, _dp, _dp]
    lib.sph_set_contacts.argtypes = [H, _up, _dp]
    lib.sph_set_contacts.restype = C.c_int
    lib.sph_get_sort.argtypes = [H, _up, _up, _up, _up]
    lib.sph_total_cells.argtypes = [H]
    lib.sph_total_cells.restype = C.c_uint64
    lib.sph_count_contacts.argtypes = [H, C.POINTER(C.c_uint64)]
    lib.sph_kernel_launches.argtypes = [H]
    lib.sph_kernel_launches.restype = C.c_uint64
    lib.sph_last_error.argtypes = [H, C.c_char_p, C.c_size_t]
    lib.sph_status_string.argtypes = [C.c_int]
    lib.sph_status_string.restype = C.c_char_p
    lib.sph_destroy.argtypes = [H]
    lib.sph_destroy.restype = None
    lib.sph_struct_sizes.argtypes = [C.POINTER(C.c_uint64)]
    lib.sph_struct_sizes.restype = C.c_int
    lib.sph_relax.argtypes = [H, C.c_uint32, C.c_double, C.c_double, _dp]
    lib.sph_relax.restype = C.c_int
    lib.sph_step_async.argtypes = [H, C.c_uint64]
    lib.sph_set_neighbor_lists.argtypes = [H, C.c_uint32]
    lib.sph_porosity.argtypes = [H, C.c_uint32, C.c_uint32, _dp, _dp]
    lib.sph_porosity.restype = C.c_int
    lib.sph_overlaps.argtypes = [H, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32), _dp,
                                 C.POINTER(C.c_uint64)]
    lib.sph_overlaps.restype = C.c_int
    lib.sph_box_state_bytes.argtypes = [H, C.POINTER(C.c_uint64)]
    lib.sph_box_state_bytes.restype = C.c_int
    lib.sph_get_boxes_async.argtypes = [H, C.c_void_p, C.c_uint64]
    lib.sph_get_boxes_async.restype = C.c_int
    lib.sph_step_async_states.argtypes = [H, C.c_uint64, C.c_void_p, C.c_uint64]
    lib.sph_step_async_states.restype = C.c_int
    lib.sph_boxes_from_staging.argtypes = [H, C.c_void_p, C.c_uint64, C.POINTER(SphBox)]
    lib.sph_boxes_from_staging.restype = C.c_int
    lib.sph_render.argtypes = [H, C.c_uint32, C.c_int, C.c_float, C.c_float, C.c_float,
                               C.c_uint32, C.c_uint32, C.POINTER(C.c_uint8)]
    lib.sph_render.restype = C.c_int
    lib.sph_snapshot.argtypes = [H]
    lib.sph_snapshot.restype = C.c_int
    lib.sph_snapshot_read.argtypes = [H, C.POINTER(SphParticles), C.POINTER(SphBonds), C.POINTER(SphBox)]
    lib.sph_snapshot_read.restype = C.c_int
    lib.sph_neighbor_stats.argtypes = [H, C.POINTER(C.c_uint64)]
    lib.sph_neighbor_stats.restype = C.c_int
    lib.sph_autotune.argtypes = [H, C.c_uint32, _dp, C.POINTER(C.c_int)]
    lib.sph_autotune.restype = C.c_int
    lib.sph_set_variant.argtypes = [H, C.c_int]
    lib.sph_set_variant.restype = C.c_int
    lib.sph_set_launch_shape.argtypes = [H, C.c_int]
    lib.sph_set_launch_shape.restype = C.c_int
    lib.sph_get_tuning.argtypes = [H, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.sph_get_tuning.restype = C.c_int
    lib.sph_get_shape_times.argtypes = [H, _dp, C.c_int]
    lib.sph_get_shape_times.restype = C.c_int
    lib.sph_barrier_check.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double]
    lib.sph_barrier_check.restype = C.c_int
    lib.sph_set_neighbor_lists.restype = C.c_int
    lib.sph_adjoint_forward.argtypes = [H, C.c_uint64, C.c_uint32, _dp]
    lib.sph_cell_offsets_static.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    lib.sph_cell_offsets_static.restype = C.c_int
    lib.sph_darcy_set.argtypes = [H, C.POINTER(SphDarcy), _dp, _dp, _dp, _dp,
                                  C.POINTER(C.c_int32), _dp]
    lib.sph_darcy_set.restype = C.c_int
    lib.sph_darcy_get.argtypes = [H, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.sph_darcy_get.restype = C.c_int
    lib.sph_darcy_log.argtypes = [H, C.POINTER(C.c_uint64), _up, _up, C.c_uint32,
                                  C.POINTER(C.c_uint32)]
    lib.sph_darcy_log.restype = C.c_int
    lib.sph_darcy_struct_size.argtypes = [C.POINTER(C.c_uint64)]
    lib.sph_darcy_struct_size.restype = C.c_int
    lib.sph_adjoint_forward.restype = C.c_int
    lib.sph_adjoint_backward.argtypes = [H, _dp, _dp, _dp, _dp]
    lib.sph_adjoint_backward.restype = C.c_int
    lib.sph_sync.argtypes = [H]
    lib.sph_set_stream.argtypes = [H, C.c_void_p]
    lib.sph_profile.argtypes = [H, C.c_int]
    lib.sph_profile_read.argtypes = [H, C.c_char_p, C.c_size_t, _dp, C.c_int, C.POINTER(C.c_int)]
    for name in ("sph_create", "sph_upload", "sph_step", "sph_advance", "sph_download",
                 "sph_get_boxes", "sph_get_contacts", "sph_get_sort", "sph_count_contacts",
                 "sph_last_error", "sph_step_async", "sph_sync", "sph_set_stream",
                 "sph_profile", "sph_profile_read"):
        getattr(lib, name).restype = C.c_int
    _LIB = lib
    return lib
