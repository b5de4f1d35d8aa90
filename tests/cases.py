"""Seeded parity scenes shared by the CPU and GPU parity tests.

Each case builds a small sim (a few hundred to a few thousand spheres) that
exercises one part of the step: periodic modes, walls and wall modes,
contact models 1/2/3, Young's-modulus stiffness, bonds and bond breaking,
fixed-velocity modes, the shear-stress wall (unfused path) and the adaptive
grid.  `ref_ok` marks cases where the reference's own kernels are defined
(contact model 3 is NaN in the reference; see oracle/sphere_oracle.c).
"""
import numpy

from sphere_b200 import scenes


def _bonds(s, n_bonds, seed, sigma_b=numpy.inf, tau_b=numpy.inf):
    """Bond n_bonds distinct pairs among each particle's three nearest
    neighbours.  n_bonds >= np keeps the reference's broken-bond marker
    (index nb0, cohesion.cuh:205) outside the particle range, where the
    reference and this project agree (see oracle/sphere_oracle.c)."""
    rng = numpy.random.default_rng(seed + 77)
    n = int(s.np[0])
    x = s.x
    pairs = []
    used = set()
    for rnd in range(3):
        for i in rng.permutation(n):
            if len(pairs) >= n_bonds:
                break
            d = numpy.sqrt(((x - x[i]) ** 2).sum(1))
            d[i] = numpy.inf
            j = int(numpy.argsort(d)[rnd])
            if (i, j) in used or (j, i) in used:
                continue
            used.add((i, j))
            pairs.append((i, j))
    assert len(pairs) >= n, "need nb0 >= np"
    for i, j in pairs:
        s.bond(int(i), int(j))
    s.sigma_b[0] = sigma_b
    s.tau_b[0] = tau_b
    return s


def make(name):
    """Return (sim, ref_ok, steps) for a named case."""
    if name == "periodic_xy_wall_stress":
        return scenes.lattice_pack(600, seed=1, periodic=1, nw=1, wmode=1), True, 20
    if name == "walls_all_sides":
        return scenes.lattice_pack(500, seed=2, periodic=0, nw=0), True, 20
    if name == "periodic_x_wall_velocity":
        return scenes.lattice_pack(500, seed=3, periodic=2, nw=1, wmode=2, wvel=-0.01), True, 20
    if name == "contact_model_1":
        return scenes.lattice_pack(500, seed=4, periodic=1, contactmodel=1, gamma_t=1e3), True, 20
    if name == "contact_model_3_hertz":
        return scenes.lattice_pack(400, seed=5, periodic=1, contactmodel=3, E=7e9), False, 10
    if name == "youngs_modulus":
        return scenes.lattice_pack(500, seed=6, periodic=1, E=7e9), True, 20
    if name == "bonds":
        s = scenes.lattice_pack(300, seed=7, periodic=1, nw=0)
        return _bonds(s, 330, 7), True, 20
    if name == "bonds_breaking":
        s = scenes.lattice_pack(200, seed=8, periodic=1, nw=0, vel_sigma=0.2)
        return _bonds(s, 220, 8, sigma_b=1.0e8, tau_b=1.0e8), True, 20
    if name == "fixvel_modes":
        s = scenes.lattice_pack(600, seed=9, periodic=1, nw=1, wmode=1, fixvel_layers=True)
        rng = numpy.random.default_rng(9)
        k = rng.choice(600, 60, replace=False)
        s.fixvel[k[:20]] = 10.0 + rng.uniform(0, 1, 20)
        s.fixvel[k[20:40]] = -1.0
        s.fixvel[k[40:]] = 7.0
        s.time_current[0] = 10.0
        s.time_total[0] = 20.0
        return s, True, 20
    if name == "shear_stress_wall":
        s = scenes.lattice_pack(600, seed=10, periodic=1, nw=1, wmode=3, fixvel_layers=True)
        s.w_tau_x[0] = 500.0
        return s, True, 20
    if name == "adaptive_grid":
        s = scenes.lattice_pack(500, seed=11, periodic=1, nw=1, wmode=2, wvel=-0.02)
        s.adaptive[0] = 1
        return s, True, 20
    if name == "sinusoidal_stress":
        s = scenes.lattice_pack(400, seed=12, periodic=1, nw=1, wmode=1)
        s.w_sigma0_A[0] = 2.0e3
        s.w_sigma0_f[0] = 50.0
        return s, True, 10
    if name == "capillary_cohesion":
        # contact model 1 with capillary bonds (contactsearch.cuh:163-168,
        # cohesion.cuh:237-277): a lattice a little wider than the spheres,
        # so that most neighbours sit at gaps between 0 and db, soft
        # contacts (k_n = 1e4) and kappa = 10, so that the capillary forces
        # are ~1/4 of the force field (relative L2 after one step: 0.23).
        # The capillary force jumps from ~3 N to 0 where a gap passes db;
        # a short time step (dt_scale 0.02) and slow spheres keep the gaps'
        # changes small over the 20 steps, so that the ~1e-11 m by which
        # the FP32 expf roundings (below) move the spheres cannot put a gap
        # on the other side of db in one run than in the other.
        s = scenes.lattice_pack(500, seed=14, periodic=1, contactmodel=1, gamma_n=0.0,
                                gamma_t=1.0, k_n=1.0e4, r_min=0.0095, r_max=0.0105,
                                spacing=0.0203, jitter=0.0006, nw=0, dt_scale=0.02,
                                vel_sigma=0.005, angvel_sigma=0.1)
        s.kappa[0] = 10.0
        s.V_b[0] = 1.0e-9
        s.db[0] = 1.0e-3
        return s, True, 20
    if name == "fast_spheres":
        # fast enough that spheres cross cells and periodic boundaries and
        # the neighbour lists are rebuilt several times
        s = scenes.lattice_pack(500, seed=13, periodic=1, nw=1, wmode=1, vel_sigma=60.0,
                                angvel_sigma=100.0)
        return s, True, 40
    raise KeyError(name)


CASES = ["periodic_xy_wall_stress", "walls_all_sides", "periodic_x_wall_velocity",
         "contact_model_1", "contact_model_3_hertz", "youngs_modulus", "bonds", "bonds_breaking",
         "fixvel_modes", "shear_stress_wall", "adaptive_grid", "sinusoidal_stress",
         "fast_spheres", "capillary_cohesion"]

# Cases whose results go through a transcendental function that CUDA and the
# C library may round differently, with the tolerance (relative to each
# field's largest magnitude) of the GPU-vs-oracle comparison:
#  * sinusoidal_stress: the wall stress through sin() in FP64 (a last-bit
#    difference of the wall force);
#  * capillary_cohesion: the capillary force through the FP32 expf()
#    (cohesion.cuh:270), which may differ by an FP32 ulp or two between CUDA
#    and glibc, ~1e-7 of each capillary force; the tolerance, 1e-6 of each
#    field's scale after 20 steps, is 2e5 times smaller than the capillary
#    forces' share of the force field (0.23), so a capillary law that is
#    wrong or missing fails it.  The oracle itself equals the reference's
#    kernels bit for bit on this case (both call glibc's expf on the CPU).
APPROX = {"sinusoidal_stress": 1e-12, "capillary_cohesion": 1e-6}


def render_scene(name):
    """A parity scene with seeded non-zero pressures, velocities, spins,
    rotations and displacements, so that every colour method of the ray
    tracer has values to map."""
    s, _, _ = make(name)
    rng = numpy.random.default_rng(5)
    n = len(s.radius)
    s.vel[:] = rng.normal(0.0, 1.0, (n, 3))
    s.angvel[:] = rng.normal(0.0, 10.0, (n, 3))
    s.angpos[:] = rng.normal(0.0, 1.0, (n, 3))
    s.xyzsum[:] = rng.normal(0.0, 0.01, (n, 3))
    s.p[:] = rng.uniform(0.0, 2.0e3, n)
    return s


def render_values(s, method):
    """The value a colour method maps (src/raytracer.cuh:452-499), FP64."""
    if method == 1:
        return numpy.asarray(s.p, dtype=numpy.float64)
    if method == 4:
        return numpy.asarray(s.xyzsum[:, 0], dtype=numpy.float64)
    a = {2: s.vel, 3: s.angvel, 5: s.angpos}[method]
    return numpy.sqrt(a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1] + a[:, 2] * a[:, 2])


# (width, height) of the ray-tracer cases: square; wide, where the integer
# hw_ratio = height / width is 0 and the image plane is flat; tall, where the
# row index wraps modulo the width
RENDER_SHAPES = [(64, 64), (48, 32), (32, 72)]


def render_runs(s):
    """(method, maxval, lower_cutoff, width, height) of the ray-tracer
    cases of scene s: every method on every shape, the middle shape with
    the median as the cutoff."""
    out = []
    for method in range(6):
        vals = render_values(s, method) if method else numpy.zeros(1)
        maxval = float(numpy.quantile(vals, 0.9)) if method else 1e3
        cut = float(numpy.median(vals)) if method else 0.0
        for k, (w, h) in enumerate(RENDER_SHAPES):
            out.append((method, maxval if maxval > 0.0 else 1.0, cut if k == 1 else 0.0, w, h))
    return out


RENDER_SCENES = ["fixvel_modes", "walls_all_sides"]
