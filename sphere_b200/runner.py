"""Host driver of the CUDA step: handle wrapper and the run() loop.

``Stepper`` owns one C-ABI handle (include/sphere_b200.h) for one or more
simulation boxes.  ``run_sim`` replaces the ``sphere`` executable that
python/sphere.py:4482 (sim.run) launches: it applies the reference's input
checks (src/sphere.cpp:145-345), then follows DEM::startTime
(src/device.cu:826-2677) for fluid == 0 -- output file 0, status.dat, steps
until time.total with an output file every time.file_dt.
"""
import copy
import ctypes as C
import os

import numpy

from . import _abi, binio
from ._abi import NC

PRECISIONS = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}
LENGTHS = {"reference": _abi.LEN_REFERENCE, "fp64": _abi.LEN_FP64}


class SphereError(RuntimeError):
    def __init__(self, status, message):
        RuntimeError.__init__(self, "%s (%s): %s" % (_abi.STATUS_NAMES.get(status, status),
                                                      status, message))
        self.status = status


def _f(a, shape):
    return numpy.ascontiguousarray(numpy.asarray(a, dtype=numpy.float64).reshape(shape))


class HostParticles(object):
    """Host arrays of all boxes in the .bin block layouts of the C ABI."""

    def __init__(self, n):
        self.x = numpy.zeros((n, 4))
        self.xyzsum = numpy.zeros((n, 3))
        self.vel = numpy.zeros((n, 4))
        self.force = numpy.zeros((n, 3))
        self.angpos = numpy.zeros((n, 3))
        self.angvel = numpy.zeros((n, 3))
        self.torque = numpy.zeros((n, 3))
        for name in ("es_dot", "es", "ev_dot", "ev", "p"):
            setattr(self, name, numpy.zeros(n))

    def struct(self):
        s = _abi.SphParticles()
        for name, _ in _abi.SphParticles._fields_:
            setattr(s, name, _abi.dptr(getattr(self, name)))
        return s

    @classmethod
    def from_sims(cls, sims):
        n = sum(int(s.np[0]) for s in sims)
        h = cls(n)
        o = 0
        for s in sims:
            k = int(s.np[0])
            h.x[o:o + k, :3] = s.x
            h.x[o:o + k, 3] = s.radius
            h.xyzsum[o:o + k] = _f(s.xyzsum, (k, 3))
            h.vel[o:o + k, :3] = s.vel
            h.vel[o:o + k, 3] = s.fixvel
            for name in ("force", "angpos", "angvel", "torque"):
                getattr(h, name)[o:o + k] = _f(getattr(s, name), (k, 3))
            for name in ("es_dot", "es", "ev_dot", "ev", "p"):
                getattr(h, name)[o:o + k] = _f(getattr(s, name), (k,))
            o += k
        return h


class HostBonds(object):
    def __init__(self, nb):
        self.pairs = numpy.zeros((nb, 2), dtype=numpy.uint32)
        self.delta_n = numpy.zeros(nb)
        self.delta_t = numpy.zeros((nb, 3))
        self.omega_n = numpy.zeros(nb)
        self.omega_t = numpy.zeros((nb, 3))

    def struct(self):
        b = _abi.SphBonds()
        b.pairs = _abi.uptr(self.pairs)
        for name in ("delta_n", "delta_t", "omega_n", "omega_t"):
            setattr(b, name, _abi.dptr(getattr(self, name)))
        return b

    @classmethod
    def from_sims(cls, sims):
        nb = sum(int(s.nb0[0]) for s in sims)
        h = cls(nb)
        o = 0
        for s in sims:
            k = int(s.nb0[0])
            if k:
                h.pairs[o:o + k] = numpy.asarray(s.bonds).reshape(-1, 2)[:k]
                h.delta_n[o:o + k] = numpy.asarray(s.bonds_delta_n, dtype=numpy.float64).reshape(-1)[:k]
                h.delta_t[o:o + k] = numpy.asarray(s.bonds_delta_t, dtype=numpy.float64).reshape(-1, 3)[:k]
                h.omega_n[o:o + k] = numpy.asarray(s.bonds_omega_n, dtype=numpy.float64).reshape(-1)[:k]
                h.omega_t[o:o + k] = numpy.asarray(s.bonds_omega_t, dtype=numpy.float64).reshape(-1, 3)[:k]
            o += k
        return h


class Stepper(object):
    """One C-ABI handle stepping one or more independent boxes on a GPU."""

    def __init__(self, sims, precision="fp64", length="reference", device=-1):
        if not isinstance(sims, (list, tuple)):
            sims = [sims]
        self.lib = _abi.load_library()
        self.sims = list(sims)
        self.np = [int(s.np[0]) for s in sims]
        self.nb = [int(s.nb0[0]) for s in sims]
        self.ntot = sum(self.np)
        self.nbonds = sum(self.nb)
        boxes = (_abi.SphBox * len(sims))(*[_abi.box_from_sim(s) for s in sims])
        self._boxes = boxes
        h = C.c_void_p()
        st = self.lib.sph_create(boxes, len(sims), PRECISIONS[precision], LENGTHS[length],
                                 int(device), C.byref(h))
        if st != 0:
            raise SphereError(st, self._msg(None))
        self.h = h

    def _msg(self, h):
        buf = C.create_string_buffer(512)
        self.lib.sph_last_error(h, buf, 512)
        return buf.value.decode(errors="replace")

    def _check(self, st, what):
        if st != 0:
            raise SphereError(st, "%s: %s" % (what, self._msg(self.h)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self):
        """Copy the sims' state to the device; a sim with a Darcy fluid also
        starts its fluid (sph_darcy_set), as the reference sets it up at the
        start of a run."""
        for s in self.sims:
            if getattr(s, "fluid", False) and int(numpy.asarray(s.cfd_solver).ravel()[0]) != 1:
                raise NotImplementedError("the Navier-Stokes fluid solver (cfd_solver 0) is not "
                                          "built; only the Darcy solver (cfd_solver 1) steps")
        self.hp = HostParticles.from_sims(self.sims)
        self.hb = HostBonds.from_sims(self.sims)
        ps = self.hp.struct()
        bs = self.hb.struct()
        self._check(self.lib.sph_upload(self.h, C.byref(ps), C.byref(bs) if self.nbonds else None),
                    "sph_upload")
        if len(self.sims) == 1 and getattr(self.sims[0], "fluid", False):
            self.darcy_set(self.sims[0])

    # ------------------------------------------------------------ Darcy
    def darcy_set(self, s):
        """Start the Darcy coupling from the fluid of sim s (sph_darcy_set).
        dphi goes in as the solver holds it, dphi * time_dt * ndem (what the
        reference's writer puts in its input file).  A Navier-Stokes fluid
        (cfd_solver 0) is refused: that solver is not built."""
        if int(numpy.asarray(s.cfd_solver).ravel()[0]) != 1:
            raise NotImplementedError("the Navier-Stokes fluid solver (cfd_solver 0) is not "
                                      "built; only the Darcy solver (cfd_solver 1) steps")
        self._darcy = _abi.darcy_from_sim(s)
        self._num = [int(v) for v in s.num]
        f = lambda a, t=numpy.float64: numpy.ascontiguousarray(_abi.cells_to_file(numpy.asarray(a, dtype=t)))
        p = f(s.p_f)
        v = f(s.v_f)
        phi = f(s.phi)
        dphi = f(numpy.asarray(s.dphi, dtype=numpy.float64) * s.time_dt * s.ndem)
        pc = f(s.p_f_constant, numpy.int32)
        fp = numpy.ascontiguousarray(numpy.asarray(s.f_p, dtype=numpy.float64).reshape(-1, 3))
        self._check(self.lib.sph_darcy_set(self.h, C.byref(self._darcy), _abi.dptr(p), _abi.dptr(v),
                                           _abi.dptr(phi), _abi.dptr(dphi),
                                           pc.ctypes.data_as(C.POINTER(C.c_int32)),
                                           _abi.dptr(fp) if fp.size else None),
                    "sph_darcy_set")

    def darcy_get(self):
        """The fluid after the steps so far, in a sim's [x, y, z](, 3)
        layout: p_f, v_f, phi, dphi (as the solver holds it, per fluid
        step), k and f_p ([np, 3])."""
        num = self._num
        ncell = num[0] * num[1] * num[2]
        p = numpy.empty(ncell)
        v = numpy.empty(ncell * 3)
        phi = numpy.empty(ncell)
        dphi = numpy.empty(ncell)
        k = numpy.empty(ncell)
        fp = numpy.empty((self.ntot, 3))
        self._check(self.lib.sph_darcy_get(self.h, _abi.dptr(p), _abi.dptr(v), _abi.dptr(phi),
                                           _abi.dptr(dphi), _abi.dptr(k),
                                           _abi.dptr(fp) if self.ntot else None), "sph_darcy_get")
        return {"p_f": _abi.cells_from_file(p, num), "v_f": _abi.cells_from_file(v, num, 3),
                "phi": _abi.cells_from_file(phi, num), "dphi_raw": _abi.cells_from_file(dphi, num),
                "k": _abi.cells_from_file(k, num), "f_p": fp}

    def darcy_log(self):
        """The Jacobi solves since the last call: (step, iterations,
        converged) arrays (sph_darcy_log)."""
        cap = _abi.DARCY_LOG
        step = numpy.zeros(cap, dtype=numpy.uint64)
        it = numpy.zeros(cap, dtype=numpy.uint32)
        ok = numpy.zeros(cap, dtype=numpy.uint32)
        n = C.c_uint32(0)
        self._check(self.lib.sph_darcy_log(self.h, step.ctypes.data_as(C.POINTER(C.c_uint64)),
                                           _abi.uptr(it), _abi.uptr(ok), cap, C.byref(n)),
                    "sph_darcy_log")
        k = int(n.value)
        return step[:k].copy(), it[:k].copy(), ok[:k].copy()

    def step(self, nsteps=1, raise_on_error=True):
        st = self.lib.sph_step(self.h, int(nsteps))
        if raise_on_error:
            self._check(st, "sph_step")
        return st

    def step_async(self, nsteps=1):
        self._check(self.lib.sph_step_async(self.h, int(nsteps)), "sph_step_async")

    def sync(self, raise_on_error=True):
        st = self.lib.sph_sync(self.h)
        if raise_on_error:
            self._check(st, "sph_sync")
        return st

    def set_stream(self, cuda_stream):
        """Run on a caller's cudaStream_t (an int handle, e.g. a torch
        stream's .cuda_stream); 0/None restores the handle's own stream."""
        self._check(self.lib.sph_set_stream(self.h, C.c_void_p(cuda_stream or None)),
                    "sph_set_stream")

    def profile(self, enable=True):
        """Run subsequent steps from the profiled graph ring (sph_profile)."""
        self._check(self.lib.sph_profile(self.h, int(bool(enable))), "sph_profile")

    def profile_read(self):
        """Mean milliseconds per kernel group over the most recent (up to 8)
        profiled steps."""
        names = C.create_string_buffer(1024)
        ms = numpy.zeros(32)
        nk = C.c_int(0)
        self._check(self.lib.sph_profile_read(self.h, names, 1024, _abi.dptr(ms), 32, C.byref(nk)),
                    "sph_profile_read")
        keys = names.value.decode().split(",")
        return dict(zip(keys, ms[:nk.value].tolist()))

    def relax(self, sweeps, alpha=0.6, z_top=1e300):
        """Geometric overlap removal on the device (sph_relax); returns the
        largest overlap of the last sweep."""
        mo = C.c_double(0.0)
        self._check(self.lib.sph_relax(self.h, int(sweeps), float(alpha), float(z_top),
                                       C.byref(mo)), "sph_relax")
        return mo.value

    def set_neighbor_lists(self, capacity):
        """Neighbour-list capacity per sphere (0 = off, cell search only;
        default 48), sph_set_neighbor_lists."""
        self._check(self.lib.sph_set_neighbor_lists(self.h, int(capacity)),
                    "sph_set_neighbor_lists")

    def porosity(self, slices, box=0):
        """(z positions, porosities) of box `box` in `slices` slabs
        (sph_porosity)."""
        z = numpy.zeros(int(slices))
        p = numpy.zeros(int(slices))
        self._check(self.lib.sph_porosity(self.h, int(box), int(slices), _abi.dptr(z),
                                          _abi.dptr(p)), "sph_porosity")
        return z, p

    def overlaps(self, box=0):
        """(pairs [n, 2] uint32, delta_n [n]) of box `box` (sph_overlaps)."""
        n = C.c_uint64(0)
        self._check(self.lib.sph_overlaps(self.h, int(box), 0, None, None, C.byref(n)),
                    "sph_overlaps")
        m = int(n.value)
        pairs = numpy.zeros((max(m, 1), 2), dtype=numpy.uint32)
        d = numpy.zeros(max(m, 1))
        if m:
            self._check(self.lib.sph_overlaps(self.h, int(box), m, _abi.uptr(pairs), _abi.dptr(d),
                                              C.byref(n)), "sph_overlaps")
        return pairs[:m], d[:m]

    def render(self, box=0, method=1, maxval=1.0e3, lower_cutoff=0.0, width=800, height=800,
               focal_length=1.0):
        """RGB image [height, width, 3] uint8 of box `box` by the ray tracer
        (sph_render); method as DEM::render's: 0 normal, 1 pres, 2 vel,
        3 angvel, 4 xdisp, 5 angpos."""
        img = numpy.zeros((int(height), int(width), 3), dtype=numpy.uint8)
        self._check(self.lib.sph_render(self.h, int(box), int(method), float(maxval),
                                        float(lower_cutoff), float(focal_length), int(width),
                                        int(height), img.ctypes.data_as(C.POINTER(C.c_uint8))),
                    "sph_render")
        return img

    def neighbor_stats(self):
        """(spheres with a list, spheres whose list overflowed, entries,
        longest list, builds so far): sph_neighbor_stats."""
        out = (C.c_uint64 * 5)()
        self._check(self.lib.sph_neighbor_stats(self.h, out), "sph_neighbor_stats")
        return dict(zip(("with_list", "overflowed", "entries", "longest", "builds"),
                        [int(v) for v in out]))

    def autotune(self, steps=20):
        """Time each launch variant of the interact kernel for `steps` steps
        from the current state, keep the fastest, restore the state
        (sph_autotune).  Returns (chosen, [ms per step of each variant])."""
        ms = numpy.zeros(_abi.TUNE_VARIANTS)
        ch = C.c_int(-1)
        self._check(self.lib.sph_autotune(self.h, int(steps), _abi.dptr(ms), C.byref(ch)),
                    "sph_autotune")
        return ch.value, ms.tolist()

    def set_variant(self, variant):
        self._check(self.lib.sph_set_variant(self.h, int(variant)), "sph_set_variant")

    def set_launch_shape(self, shape):
        """Launch shape of the list step (sph_set_launch_shape)."""
        self._check(self.lib.sph_set_launch_shape(self.h, int(shape)), "sph_set_launch_shape")

    def tuning(self):
        """(variant, list-step launch shape) in use (sph_get_tuning)."""
        v, sh = C.c_int(0), C.c_int(0)
        self._check(self.lib.sph_get_tuning(self.h, C.byref(v), C.byref(sh)), "sph_get_tuning")
        return v.value, sh.value

    def shape_times(self):
        """The last autotune's ms per step of the list step at each launch
        shape, -1 where not tried (sph_get_shape_times)."""
        ms = numpy.zeros(_abi.PAIR_SHAPES)
        self._check(self.lib.sph_get_shape_times(self.h, _abi.dptr(ms), len(ms)),
                    "sph_get_shape_times")
        return ms

    def adjoint_forward(self, nsteps, ckpt=100):
        """nsteps steps with a checkpoint every ckpt steps kept for
        adjoint_backward (sph_adjoint_forward); returns the device ms."""
        ms = C.c_double(0.0)
        self._check(self.lib.sph_adjoint_forward(self.h, int(nsteps), int(ckpt), C.byref(ms)),
                    "sph_adjoint_forward")
        return ms.value

    def adjoint_backward(self, dx_final):
        """Reverse pass for dLoss/d(final positions) dx_final [np, 3]
        (sph_adjoint_backward).  Returns ({"k_n", "gamma_n", "mu"} gradients,
        dLoss/dv0 [np, 3], device ms)."""
        dx = numpy.ascontiguousarray(dx_final, dtype=numpy.float64).reshape(-1, 3)
        gp = numpy.zeros(3)
        gv = numpy.zeros((dx.shape[0], 3))
        ms = C.c_double(0.0)
        self._check(self.lib.sph_adjoint_backward(self.h, _abi.dptr(dx), _abi.dptr(gp),
                                                  _abi.dptr(gv), C.byref(ms)),
                    "sph_adjoint_backward")
        return {"k_n": gp[0], "gamma_n": gp[1], "mu": gp[2]}, gv, ms.value

    def advance(self, total, file_dt, current, ftc, max_steps=2 ** 62):
        cur = C.c_double(current)
        f = C.c_double(ftc)
        done = C.c_uint64(0)
        st = self.lib.sph_advance(self.h, float(total), float(file_dt), C.byref(cur), C.byref(f),
                                  int(max_steps), C.byref(done))
        return st, cur.value, f.value, done.value

    def download(self):
        hp = HostParticles(self.ntot)
        hb = HostBonds(self.nbonds)
        ps = hp.struct()
        bs = hb.struct()
        self._check(self.lib.sph_download(self.h, C.byref(ps), C.byref(bs) if self.nbonds else None),
                    "sph_download")
        return hp, hb

    def boxes(self):
        out = (_abi.SphBox * len(self.sims))()
        self._check(self.lib.sph_get_boxes(self.h, out), "sph_get_boxes")
        return list(out)

    def box_state_bytes(self):
        """Size of one raw box-state copy (sph_box_state_bytes)."""
        b = C.c_uint64()
        self._check(self.lib.sph_box_state_bytes(self.h, C.byref(b)), "sph_box_state_bytes")
        return b.value

    def get_boxes_async(self, staging):
        """Queue a copy of the box state into `staging` (a C-contiguous
        uint8 numpy array of at least box_state_bytes(); pinned memory keeps
        it asynchronous).  Read it with boxes_from_state after sync()."""
        assert staging.dtype == numpy.uint8 and staging.flags["C_CONTIGUOUS"]
        self._check(self.lib.sph_get_boxes_async(self.h, C.c_void_p(staging.ctypes.data),
                                                 staging.nbytes), "sph_get_boxes_async")

    def step_async_states(self, nsteps, states):
        """Queue nsteps steps and the box state after each into `states`
        (uint8, nsteps x box_state_bytes(), C-contiguous)."""
        assert states.dtype == numpy.uint8 and states.flags["C_CONTIGUOUS"]
        self._check(self.lib.sph_step_async_states(self.h, int(nsteps),
                                                   C.c_void_p(states.ctypes.data), states.nbytes),
                    "sph_step_async_states")

    def boxes_from_state(self, state):
        """SphBox records (as boxes() returns them) from one raw state."""
        return self.boxes_from_states(state, 1)[0]

    def boxes_from_states(self, states, nstates=None):
        """Per state, the list of SphBox records, from `nstates` raw states
        (default: all rows of `states`), decoded in one call."""
        assert states.dtype == numpy.uint8 and states.flags["C_CONTIGUOUS"]
        nb = self.box_state_bytes()
        if nstates is None:
            nstates = states.nbytes // nb
        assert states.nbytes >= nstates * nb
        nbox = len(self.sims)
        out = (_abi.SphBox * (nstates * nbox))()
        self._check(self.lib.sph_boxes_from_staging(self.h, C.c_void_p(states.ctypes.data),
                                                    int(nstates), out),
                    "sph_boxes_from_staging")
        return [list(out[k * nbox:(k + 1) * nbox]) for k in range(nstates)]

    def contacts(self):
        n = self.ntot
        c = numpy.zeros(n * NC, dtype=numpy.uint32)
        dt = numpy.zeros((n * NC, 4))
        dm = numpy.zeros((n * NC, 4))
        self._check(self.lib.sph_get_contacts(self.h, _abi.uptr(c), _abi.dptr(dt), _abi.dptr(dm)),
                    "sph_get_contacts")
        return c, dt, dm

    def set_contacts(self, contacts, delta_t=None):
        """Contact rows and tangential histories in the layout contacts()
        returns (sph_set_contacts), e.g. to continue a run in another handle
        with its contact history."""
        c = numpy.ascontiguousarray(contacts, dtype=numpy.uint32).reshape(-1)
        d = None if delta_t is None else numpy.ascontiguousarray(delta_t,
                                                                 dtype=numpy.float64).reshape(-1)
        self._check(self.lib.sph_set_contacts(self.h, _abi.uptr(c),
                                              _abi.dptr(d) if d is not None else None),
                    "sph_set_contacts")

    def sort_products(self):
        n = self.ntot
        nc = int(self.lib.sph_total_cells(self.h))
        cid = numpy.zeros(max(n, 1), dtype=numpy.uint32)
        perm = numpy.zeros(max(n, 1), dtype=numpy.uint32)
        cs = numpy.zeros(nc, dtype=numpy.uint32)
        ce = numpy.zeros(nc, dtype=numpy.uint32)
        self._check(self.lib.sph_get_sort(self.h, _abi.uptr(cid), _abi.uptr(perm), _abi.uptr(cs),
                                          _abi.uptr(ce)), "sph_get_sort")
        return cid[:n], perm[:n], cs, ce

    def count_contacts(self):
        c = C.c_uint64(0)
        self._check(self.lib.sph_count_contacts(self.h, C.byref(c)), "sph_count_contacts")
        return c.value

    def kernel_launches(self):
        return int(self.lib.sph_kernel_launches(self.h))

    def snapshot(self):
        """Enqueue a device copy of the downloadable state after the steps
        queued so far (sph_snapshot); returns at once."""
        self._check(self.lib.sph_snapshot(self.h), "sph_snapshot")

    def snapshot_read(self):
        """Wait for the last snapshot and read it (sph_snapshot_read).
        Returns (status, HostParticles, HostBonds, boxes); status is the
        first device error raised since the previous snapshot."""
        hp = HostParticles(self.ntot)
        hb = HostBonds(self.nbonds)
        ps = hp.struct()
        bs = hb.struct()
        out = (_abi.SphBox * len(self.sims))()
        st = self.lib.sph_snapshot_read(self.h, C.byref(ps), C.byref(bs) if self.nbonds else None,
                                        out)
        if st not in (0, _abi.SPH_ERR_NAN, _abi.SPH_ERR_OUT_OF_GRID, _abi.SPH_ERR_INPUT,
                      _abi.SPH_ERR_NC_OVERFLOW):
            self._check(st, "sph_snapshot_read")
        return st, hp, hb, list(out)

    def to_sims(self, state=None):
        """Copy device state (or a (HostParticles, HostBonds, boxes) triple
        read earlier) into the sim objects, as an output file would."""
        if state is None:
            hp, hb = self.download()
            boxes = self.boxes()
        else:
            hp, hb, boxes = state
        o = ob = 0
        for s, b, k, kb in zip(self.sims, boxes, self.np, self.nb):
            s.x = hp.x[o:o + k, :3].copy()
            s.radius = hp.x[o:o + k, 3].copy()
            s.xyzsum = hp.xyzsum[o:o + k].copy()
            s.vel = hp.vel[o:o + k, :3].copy()
            s.fixvel = hp.vel[o:o + k, 3].copy()
            for name in ("force", "angpos", "angvel", "torque", "es_dot", "es", "ev_dot", "ev", "p"):
                setattr(s, name, getattr(hp, name)[o:o + k].copy())
            if kb:
                s.bonds = hb.pairs[ob:ob + kb].copy()
                s.bonds_delta_n = hb.delta_n[ob:ob + kb].copy()
                s.bonds_delta_t = hb.delta_t[ob:ob + kb].copy()
                s.bonds_omega_n = hb.omega_n[ob:ob + kb].copy()
                s.bonds_omega_t = hb.omega_t[ob:ob + kb].copy()
            _abi.sim_from_box(s, b)
            o += k
            ob += kb
        if state is None and len(self.sims) == 1 and getattr(self.sims[0], "fluid", False):
            s = self.sims[0]
            f = self.darcy_get()
            s.p_f, s.v_f, s.phi, s.f_p = f["p_f"], f["v_f"], f["phi"], f["f_p"]
            # as a sim reading the output file holds it (per unit time)
            s.dphi = f["dphi_raw"] / (s.time_dt * s.ndem)
            self.dphi_raw = f["dphi_raw"]
        return self.sims


# src/sphere.cpp:145-345 checkValues (host side, before any device work)
def check_values(s):
    if int(s.nd[0]) != 3:
        return "Error: nd = %d, ND = 3" % int(s.nd[0])
    if s.time_current[0] > s.time_total[0] or s.time_current[0] < 0.0:
        return "Error: time.current = %g s, time.total = %g s" % (s.time_current[0], s.time_total[0])
    if (numpy.asarray(s.origo) < 0.0).any():
        return "Error: Negative values in grid.origo are known to cause problems."
    if (numpy.asarray(s.L) <= 0.0).any():
        return "Error: grid.L must be positive"
    if (numpy.asarray(s.num) <= 0).any():
        return "Error: grid.num must be positive"
    if s.periodic[0] == 2 and s.num[0] < 3:
        return "Error: When 1st dimension boundaries are periodic, there must be at least 3 cells in that dimension."
    if s.periodic[0] == 1 and (s.num[0] < 3 or s.num[1] < 3):
        return ("Error: When 1st and 2nd dimension boundaries are periodic, there must be at "
                "least 3 cells in each of those dimensions.")
    n = int(s.np[0])
    if n:
        if (s.radius <= 0.0).any():
            return "Error: Particle %d has a radius of %g m." % (int(numpy.argmax(s.radius <= 0.0)),
                                                                  float(s.radius.min()))
        if numpy.isnan(s.x).any() or numpy.isnan(s.vel).any() or numpy.isnan(s.fixvel).any():
            return "Error: NaN particle position or velocity"
        out = (s.x < numpy.asarray(s.origo)).any(axis=1) | (s.x > numpy.asarray(s.L)).any(axis=1)
        if out.any():
            return "Error: Particle %d is outside of the computational grid" % int(numpy.argmax(out))
        if s.nw[0] > 0 and s.w_x[0] < max(0.0, float(s.x[:, 2].max())):
            return "Error: One or more particles have centres above the upper, dynamic wall"
    if s.k_n[0] <= 0.0:
        return "Error: k_n = %g N/m" % s.k_n[0]
    if s.E[0] < 0.0:
        return "Error: E = %g N/m^3" % s.E[0]
    if s.rho[0] <= 0.0:
        return "Error: rho = %g kg/m3" % s.rho[0]
    return None


def report_values(s):
    """The `--dry` report of src/sphere.cpp:349-466."""
    print("  - Number of dimensions: nd = %d" % s.nd[0])
    print("  - Number of particles:  np = %d" % s.np[0])
    print("  - Compiled for double precision")
    print("  - Timestep length:      time.dt         = %g s" % s.time_dt[0])
    print("  - Start at time:        time.current    = %g s" % s.time_current[0])
    print("  - Total sim. time:      time.total      = %g s" % s.time_total[0])
    print("  - File output interval: time.file_dt    = %g s" % s.time_file_dt[0])
    print("  - Start at step count:  time.step_count = %d" % s.time_step_count[0])
    cm = int(s.contactmodel[0])
    names = {1: "Linear-elastic-viscous (n), visco-frictional (t)",
             2: "Linear-elastic-visco-frictional", 3: "Nonlinear-elastic-visco-frictional"}
    print("  - Contact model: " + names.get(cm, "unknown (%d)" % cm))
    print("  - Using Young's modulus for contact stiffness" if s.E[0] > 0.01 else
          "  - Using global value for contact stiffness")
    print("  - Number of dynamic walls: %d" % s.nw[0])
    print("  - Grid: %d * %d * %d cells" % tuple(int(v) for v in s.num))
    print("  - Domain size: %g * %g * %g m" % tuple(float(v) for v in s.L))
    print("  - No. of particle bonds: %d" % s.nb0[0])


def _write_status(path, s):
    with open(path, "w") as fh:
        cur = float(s.time_current[0])
        tot = float(s.time_total[0])
        fh.write("%2.4e %2.4e %d\n" % (cur, 100.0 * cur / tot if tot else 0.0,
                                       int(s.time_step_count[0])))


def run_sim(s, root="..", verbose=True, device=-1, precision="fp64", length="reference"):
    """Run `s` to time_total, writing the reference's output files.  Returns
    0 or the SphStatus of the first failure (as the binary's exit status)."""
    if getattr(s, "fluid", False) and int(numpy.asarray(s.cfd_solver).ravel()[0]) != 1:
        raise NotImplementedError("the Navier-Stokes fluid solver (cfd_solver 0) is not built; "
                                  "only the Darcy solver (cfd_solver 1) steps")
    msg = check_values(s)
    if msg:
        print(msg)
        return 1
    # the caller's object keeps its input state, as with the reference binary
    s = copy.deepcopy(s)
    outdir = os.path.join(root, "output")
    os.makedirs(outdir, exist_ok=True)
    status_path = os.path.join(outdir, s.sid + ".status.dat")
    # device.cu:840-842: output file 0 before the first step
    if int(s.time_step_count[0]) == 0:
        binio.write_bin(os.path.join(outdir, s.sid + ".output00000.bin"), s)
    st = Stepper([s], precision=precision, length=length, device=device)
    if getattr(s, "fluid", False):
        return _run_fluid(st, s, outdir, status_path, verbose)
    try:
        st.upload()
        _write_status(status_path, s)
        cur = float(s.time_current[0])
        total = float(s.time_total[0])
        file_dt = float(s.time_file_dt[0])
        dt = float(s.time_dt[0])
        ftc = 0.0
        state = {"status": 0, "stop": False}

        def write_snapshot(t_out):
            # the output due at time t_out, read back while later steps run
            code, hp, hb, boxes = st.snapshot_read()
            if code != 0:
                state["status"] = code
                if verbose:
                    print("sphere_b200: " + st._msg(st.h))
                # an overflowing contact list is reported and the run goes
                # on (the reference ignores it); anything else ends the run
                if code != _abi.SPH_ERR_NC_OVERFLOW:
                    state["stop"] = True
                    return
            st.to_sims((hp, hb, boxes))
            s.time_current[0] = t_out
            s.time_step_count[0] += 1
            binio.write_bin(os.path.join(outdir, "%s.output%05d.bin" %
                                         (s.sid, int(s.time_step_count[0]))), s)
            _write_status(status_path, s)

        pending = None   # time of the queued snapshot not yet written
        while cur <= total and not state["stop"]:
            # steps up to the next output, counted as the reference's loop
            # does (src/device.cu:1031 loop condition, :2536-2537
            # increments, :2569 output test)
            k = 0
            while cur <= total:
                cur += dt
                ftc += dt
                k += 1
                if ftc >= file_dt:
                    break
            st.step_async(k)
            if pending is not None:     # overlaps with the steps just queued
                write_snapshot(pending)
                pending = None
            if ftc >= file_dt and not state["stop"]:
                st.snapshot()
                pending = cur
                ftc = 0.0
        if pending is not None and not state["stop"]:
            write_snapshot(pending)
        code = st.sync(raise_on_error=False)
        if code != 0 and state["status"] == 0:
            state["status"] = code
            if verbose:
                print("sphere_b200: " + st._msg(st.h))
        if verbose:
            print("  - Last output file number: %d" % int(s.time_step_count[0]))
        return state["status"]
    finally:
        st.close()


def _run_fluid(st, s, outdir, status_path, verbose):
    """run() with a Darcy fluid: the output-cadence loop of sph_advance
    (src/device.cu:1031, 2536-2537, 2569), each output with the fluid fields
    as the reference's writer stores them (dphi per fluid step), and
    output/<sid>-conv.log with the reference's lines (src/device.cu:2349-2370:
    "step iterations" for converged solves at every tenth step and for every
    solve that did not converge)."""
    conv = open(os.path.join(outdir, s.sid + "-conv.log"), "w")

    def log():
        step, iters, ok = st.darcy_log()
        for a, b, c in zip(step, iters, ok):
            if (c and (int(a) - 1) % 10 == 0) or not c:
                conv.write("%d\t%d\n" % (int(a), int(b)))

    try:
        st.upload()
        _write_status(status_path, s)
        cur = float(s.time_current[0])
        total = float(s.time_total[0])
        file_dt = float(s.time_file_dt[0])
        ftc = 0.0
        status = 0
        while cur <= total:
            # at most SPH_DARCY_LOG steps per call, so that no log entry is lost
            code, cur, ftc, done = st.advance(total, file_dt, cur, ftc, _abi.DARCY_LOG)
            log()
            if code != 0:
                status = code
                if verbose:
                    print("sphere_b200: " + st._msg(st.h))
                if code != _abi.SPH_ERR_NC_OVERFLOW or done == 0:
                    break
            if ftc >= file_dt:
                st.to_sims()
                s.time_current[0] = cur
                s.time_step_count[0] += 1
                binio.write_bin(os.path.join(outdir, "%s.output%05d.bin" %
                                             (s.sid, int(s.time_step_count[0]))), s,
                                dphi_raw=st.dphi_raw)
                _write_status(status_path, s)
                ftc = 0.0
        if verbose:
            print("  - Last output file number: %d" % int(s.time_step_count[0]))
        return status
    finally:
        conv.close()
        st.close()
