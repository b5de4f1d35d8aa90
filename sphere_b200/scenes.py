"""Seeded synthetic scenes: small parity cases and the benchmark workloads.

All generators return ``sim`` objects (sphere_b200.sim) built from a numpy
Generator seed, so every run of a test or benchmark sees the same inputs.
"""
import math

import numpy

from .sim import sim, V_sphere


def lattice_pack(n, seed=0, r_min=0.009, r_max=0.011, spacing=None, jitter=None, periodic=1,
                 contactmodel=2, nw=1, wmode=1, sigma0=1.0e4, wvel=0.0, k_n=1.16e9, gamma_n=1.0e2,
                 gamma_t=5.0e1, mu=0.5, E=0.0, g=(0.0, 0.0, -9.81), vel_sigma=0.05,
                 angvel_sigma=1.0, aspect=(1.0, 1.0), margin_cells=0, fixvel_layers=False,
                 dt_scale=0.17, sid="lattice"):
    """A jittered cubic lattice of n spheres, packed so that neighbours
    overlap slightly (many contacts from the first step), random velocities
    and spins, a top wall (nw=1) and periodic or wall sides."""
    rng = numpy.random.default_rng(seed)
    s = sim(np=n, nw=0, sid=sid)
    s.radius[:] = rng.uniform(r_min, r_max, n)
    if spacing is None:
        spacing = 1.96 * (0.5 * (r_min + r_max))
    if jitter is None:
        jitter = 0.03 * spacing
    ax, ay = aspect
    side = max(int(math.ceil((n / (ax * ay)) ** (1.0 / 3.0))), 1)
    nx_ = max(int(round(side * ax)), 1)
    ny_ = max(int(round(side * ay)), 1)
    nz_ = int(math.ceil(n / float(nx_ * ny_)))
    i = numpy.arange(n)
    gp = numpy.stack([i % nx_, (i // nx_) % ny_, i // (nx_ * ny_)], 1).astype(float)
    cell = 2.1 * r_max
    if periodic:
        Lx, Ly = nx_ * spacing, ny_ * spacing
        base = numpy.array([0.5 * spacing, 0.5 * spacing, r_max * 1.5])
    else:
        Lx, Ly = nx_ * spacing + 2 * r_max, ny_ * spacing + 2 * r_max
        base = numpy.array([r_max + 0.5 * spacing, r_max + 0.5 * spacing, r_max * 1.5])
    s.x[:] = gp * spacing + base + rng.uniform(-jitter, jitter, (n, 3))
    if periodic:
        s.x[:, 0] = numpy.mod(s.x[:, 0], Lx)
        s.x[:, 1] = numpy.mod(s.x[:, 1], Ly)
    s.x[:, 2] = numpy.maximum(s.x[:, 2], s.radius * 0.999)
    s.vel[:] = rng.normal(0.0, vel_sigma, (n, 3))
    s.angvel[:] = rng.normal(0.0, angvel_sigma, (n, 3))
    s.g[:] = g
    s.k_n[0] = k_n
    s.k_t[0] = k_n
    s.gamma_n[0] = gamma_n
    s.gamma_t[0] = gamma_t
    s.mu_s[0] = mu
    s.mu_d[0] = mu
    s.E[0] = E
    s.contactmodel[0] = contactmodel
    s.periodic[0] = periodic
    ztop = float(numpy.max(s.x[:, 2] + s.radius))
    Lz = ztop + (3 + margin_cells) * cell
    nxc = max(int(Lx / cell), 3)
    nyc = max(int(Ly / cell), 3)
    nzc = max(int(Lz / cell), 3)
    s.origo[:] = 0.0
    s.L[:] = [Lx, Ly, Lz]
    s.num[:] = [nxc, nyc, nzc]
    if nw:
        s.nw = numpy.ones(1, dtype=numpy.uint32)
        s.wmode = numpy.array([wmode], dtype=numpy.int32)
        s.w_n = numpy.array([[0.0, 0.0, -1.0]])
        s.w_x = numpy.array([ztop - 0.2 * r_min])
        s.w_m = numpy.array([s.totalMass()])
        s.w_vel = numpy.array([wvel])
        s.w_force = numpy.zeros(1)
        s.w_sigma0 = numpy.array([sigma0])
    if fixvel_layers:
        zlo = s.x[:, 2] < s.x[:, 2].min() + 1.5 * r_max
        zhi = s.x[:, 2] > s.x[:, 2].max() - 1.5 * r_max
        s.fixvel[zlo | zhi] = 1.0
        s.vel[zlo | zhi, :2] = 0.0
        s.vel[zhi, 0] = 0.01
        s.angvel[zlo | zhi] = 0.0
    m_min = s.rho[0] * V_sphere(r_min)
    k = k_n if E <= 0.001 else math.pi / 2.0 * E * r_max
    s.time_dt[0] = dt_scale * math.sqrt(m_min / k)
    s.time_total[0] = 1.0
    s.time_file_dt[0] = 1.0
    return s


def two_particles(radii=(1.0, 1.0), x0=(5.0, 5.0, 2.0), x1=(5.0, 5.0, 4.05), vel0=(0.0, 0.0, 1.0),
                  total=0.1, file_dt=0.01, sid="contactmodeltest"):
    """The two-sphere impact of the reference's tests/contactmodel.py."""
    s = sim(np=2, sid=sid)
    s.radius[:] = radii
    s.x[0, :] = x0
    s.x[1, :] = x1
    s.vel[0, :] = vel0
    s.defineWorldBoundaries(L=[10, 10, 10])
    s.initTemporal(total=total, file_dt=file_dt)
    return s


def darcy_pack(n, seed, periodic=1, nw=1, wmode=1, beta_f=1.0e-7, file_every=7.5, **kw):
    """A seeded sphere pack (lattice_pack) in a Darcy fluid (cfd_solver 1)
    at hydrostatic pressure below the top wall: water (mu = 8.9e-4,
    rho_f = 1e3), compressibility beta_f, the grain-size permeability
    prefactor (d^2 / 180), an output every file_every steps."""
    s = lattice_pack(n, seed=seed, periodic=periodic, nw=nw, wmode=wmode, **kw)
    s.initFluid(cfd_solver=1, mu=8.9e-4, rho=1.0e3, p=0.0, hydrostatic=True)
    s.setFluidCompressibility(beta_f)
    s.setPermeabilityGrainSize()
    s.time_file_dt[0] = s.time_dt[0] * file_every
    return s


def gravity_settling(n=10000, seed=0, steps=1000):
    """Plain FP64 gravity settling of n spheres: radii U[0.010, 0.012] m,
    rho 2600, jittered cubic lattice (spacing 2.5*r_max, jitter +-0.2*r_max)
    in a 0.5 x 0.5 m box, zero velocity, linear contacts k_n = k_t = 1.16e9,
    no damping, mu 0.5, fixed bottom, wall sides, dt = 0.17*sqrt(m_min/k_n).
    The lattice is 16 x 16 per layer, so 40 layers reach z ~ 1.2 m; the box
    height is 1.25 m instead of 1.0 m to hold them."""
    rng = numpy.random.default_rng(seed)
    r_min, r_max = 0.010, 0.012
    s = sim(np=n, nw=0, sid="settle")
    s.radius[:] = rng.uniform(r_min, r_max, n)
    sp = 2.5 * r_max
    per = int(0.5 / sp)
    i = numpy.arange(n)
    gp = numpy.stack([i % per, (i // per) % per, i // (per * per)], 1).astype(float)
    s.x[:] = gp * sp + sp * 0.5 + rng.uniform(-0.2 * r_max, 0.2 * r_max, (n, 3))
    s.g[:] = [0.0, 0.0, -9.81]
    s.k_n[0] = s.k_t[0] = 1.16e9
    s.gamma_n[0] = s.gamma_t[0] = 0.0
    s.mu_s[0] = s.mu_d[0] = 0.5
    s.periodic[0] = 0
    s.defineWorldBoundaries(L=[0.5, 0.5, 1.25])
    m_min = s.rho[0] * V_sphere(r_min)
    s.time_dt[0] = 0.17 * math.sqrt(m_min / s.k_n[0])
    s.time_total[0] = (steps - 0.5) * s.time_dt[0]
    s.time_file_dt[0] = s.time_total[0]
    return s


def _fcc_sites(nxc, nyc, nzc, a):
    """FCC lattice sites (4 per cube of side a), layer by layer in z."""
    base = numpy.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    iz, iy, ix = numpy.meshgrid(numpy.arange(nzc), numpy.arange(nyc), numpy.arange(nxc),
                                indexing="ij")
    cubes = numpy.stack([ix.ravel(), iy.ravel(), iz.ravel()], 1).astype(float)
    sites = (cubes[:, None, :] + base[None, :, :]).reshape(-1, 3)
    order = numpy.lexsort((sites[:, 0], sites[:, 1], sites[:, 2]))
    return sites[order] * a


def _fcc_start(n, rng, r, porosity, aspect_z, zlift, sid):
    """Spheres of radii r on an FCC lattice (jittered) filling an x-y
    periodic box of aspect 1 : 1 : aspect_z sized for the porosity, with a
    sorting grid of cells 2.1 r_max wide and room above.  Returns the sim and
    the packing height H."""
    v_solid = float(numpy.sum(4.0 / 3.0 * math.pi * r ** 3))
    v_box = v_solid / (1.0 - porosity)
    L = (v_box / aspect_z) ** (1.0 / 3.0)
    H = aspect_z * L
    a0 = (4.0 * L * L * H / n) ** (1.0 / 3.0)   # FCC cube side for n sites in the box
    nxc = max(int(round(L / a0)), 3)
    a = L / nxc
    nzc = int(math.ceil(n / (4.0 * nxc * nxc)))
    sites = _fcc_sites(nxc, nxc, nzc, a)[:n]
    sites[:, 2] *= (H - 2.0 * zlift) / max(sites[:, 2].max(), 1e-12)
    s = sim(np=n, nw=0, sid=sid)
    s.radius[:] = r
    s.x[:] = sites + numpy.array([0.25 * a, 0.25 * a, zlift]) + \
        rng.uniform(-0.05 * a, 0.05 * a, (n, 3))
    s.x[:, 0] = numpy.mod(s.x[:, 0], L)
    s.x[:, 1] = numpy.mod(s.x[:, 1], L)
    s.x[:, 2] = numpy.clip(s.x[:, 2], r, H - r)
    r_max = float(r.max())
    cell = 2.1 * r_max
    ncx = max(int(L / cell), 3)
    s.periodic[0] = 1
    s.origo[:] = 0.0
    Lz = H + 4.0 * cell
    s.L[:] = [L, L, Lz]
    s.num[:] = [ncx, ncx, max(int(Lz / cell), 3)]
    s.time_dt[0] = 1e-7
    s.time_total[0] = 1.0
    return s, H


def gpu_relax(s, sweeps, alpha, z_top, device=-1):
    """Overlap removal of one box on the GPU (sph_relax): moves s.x and
    returns the largest overlap of the last sweep."""
    from .runner import Stepper
    st = Stepper([s], device=device)
    st.upload()
    worst = st.relax(sweeps, alpha=alpha, z_top=z_top)
    hp, _ = st.download()
    st.close()
    s.x = hp.x[:, :3].copy()
    return worst


def dense_pack(n, seed=0, porosity=0.40, median=0.01, sigma_ln=0.2, r_clip=(0.005, 0.02),
               aspect_z=0.5, sweeps=3000, alpha=0.6, inflate=2.0e-7, device=-1, sid="dense",
               relax=None):
    """A dense x-y periodic pack of n log-normal spheres at the given
    porosity: FCC lattice start in a box of aspect 1 : 1 : aspect_z sized
    for the porosity, then geometric overlap removal between the floor and
    the box top (`relax(s, sweeps, alpha, z_top)`, by default sph_relax on
    GPU `device`; any function with the same sweeps gives the same pack),
    then radii grown by the factor (1 + inflate) so that touching spheres
    overlap by ~inflate * r and form contacts.  Returns the sim (no walls
    yet) and the largest residual overlap of the relaxation."""
    rng = numpy.random.default_rng(seed)
    r = numpy.clip(numpy.exp(rng.normal(math.log(median), sigma_ln, n)), *r_clip)
    s, H = _fcc_start(n, rng, r, porosity, aspect_z, median, sid)
    if relax is None:
        worst = gpu_relax(s, sweeps, alpha, H, device=device)
    else:
        worst = relax(s, sweeps, alpha, H)
    s.radius *= 1.0 + inflate
    s.time_current[0] = 0.0
    return s, worst


def bonded_pack(n=200000, nbonds=300000, seed=0, porosity=0.38, r_range=(0.008, 0.012),
                E=70.0e9, k_bond=1.0e9, sigma_b=1.0e6, wvel=-0.005, sweeps=3000, device=-1,
                sid="bonded"):
    """The bonded-pack workload: n spheres of radii U[r_range] packed on the
    GPU to the porosity (FCC start + overlap removal, radii grown so that
    neighbours touch), nbonds linear bonds between touching pairs (the
    first nbonds pairs of the overlap listing, i < j ascending), contact
    stiffness from Young's modulus E (k_n = pi/2 E r, contact model 2),
    bond stiffness k_n = k_t = k_bond, bond strength sigma_b (tau_b
    unlimited), and a top wall moving at wvel (uniaxialStrainRate, wmode 2);
    dt = 0.17 sqrt(m_min / k) with k = pi/2 E r_max."""
    from .runner import Stepper
    rng = numpy.random.default_rng(seed)
    r = rng.uniform(r_range[0], r_range[1], n)
    s, H = _fcc_start(n, rng, r, porosity, 0.5, float(numpy.mean(r)), sid)
    st = Stepper([s], device=device)
    st.upload()
    st.relax(sweeps, alpha=0.6, z_top=H)
    st.to_sims()
    s.radius *= 1.0 + 2.0e-7
    st.close()
    st = Stepper([s], device=device)
    st.upload()
    pairs, _ = st.overlaps()
    st.close()
    nb = min(int(nbonds), len(pairs))
    s.nb0[0] = nb
    s.bonds = numpy.array(pairs[:nb], dtype=numpy.uint32)
    s.bonds_delta_n = numpy.zeros(nb)
    s.bonds_delta_t = numpy.zeros((nb, 3))
    s.bonds_omega_n = numpy.zeros(nb)
    s.bonds_omega_t = numpy.zeros((nb, 3))
    s.lambda_bar[0] = 1.0
    s.sigma_b[0] = sigma_b
    s.tau_b[0] = numpy.inf
    s.g[:] = [0.0, 0.0, -9.81]
    s.E[0] = E
    s.k_n[0] = s.k_t[0] = k_bond
    s.gamma_n[0] = 0.0
    s.gamma_t[0] = 0.0
    s.mu_s[0] = s.mu_d[0] = 0.5
    s.contactmodel[0] = 2
    s.time_current[0] = 0.0
    s.uniaxialStrainRate(wvel=wvel)
    # adjustWall rounds the z cell count up; keep every cell 2.1 r_max wide
    s.num[2] = max(int(float(s.L[2]) / (2.1 * float(s.radius.max()))), 3)
    m_min = float(s.rho[0]) * V_sphere(float(r.min()))
    k = math.pi / 2.0 * E * float(s.radius.max())
    s.time_dt[0] = 0.17 * math.sqrt(m_min / k)
    s.time_total[0] = 10000 * s.time_dt[0]
    s.time_file_dt[0] = s.time_total[0]
    return s


def _shear_setup(s, sigma0, mu, k_n=1.16e9, gamma_n=1.0e3, top_vel=0.01, steps=5000):
    """Turn a relaxed pack into a shear box: gravity, linear contacts, a top
    wall at normal stress sigma0 (wmode 1, mass = total particle mass as in
    sim.consolidate), the top layer moving at +x top_vel and the bottom
    layer held (fixvel, as in sim.shear), dt = 0.17 sqrt(m_min / k_n)."""
    s.g[:] = [0.0, 0.0, -9.81]
    s.k_n[0] = s.k_t[0] = k_n
    s.gamma_n[0] = gamma_n
    s.gamma_t[0] = 0.0
    s.mu_s[0] = s.mu_d[0] = mu
    rr = s.radius
    r_max = float(rr.max())
    ztop = float((s.x[:, 2] + rr).max())
    zmin = float((s.x[:, 2] - rr).min())
    s.nw = numpy.ones(1, dtype=numpy.uint32)
    s.wmode = numpy.array([1], dtype=numpy.int32)
    s.w_n = numpy.array([[0.0, 0.0, -1.0]])
    s.w_x = numpy.array([ztop])
    s.w_m = numpy.array([s.totalMass()])
    s.w_vel = numpy.zeros(1)
    s.w_force = numpy.zeros(1)
    s.w_sigma0 = numpy.array([sigma0])
    top = s.x[:, 2] > ztop - 2.0 * r_max
    bot = s.x[:, 2] < zmin + 2.0 * r_max
    s.fixvel[top | bot] = 1.0
    s.vel[:] = 0.0
    s.vel[top, 0] = top_vel
    m_min = s.rho[0] * V_sphere(float(rr.min()))
    s.time_dt[0] = 0.17 * math.sqrt(m_min / s.k_n[0])
    s.time_current[0] = 0.0
    s.time_total[0] = steps * s.time_dt[0]
    s.time_file_dt[0] = s.time_total[0]
    return s


def shear_ensemble(nboxes=256, seed=0, device=-1, counts=(500, 20000), r_range=(0.009, 0.011),
                   porosity=0.40, sweeps=2000, inflate=2.0e-7, steps=2000, subset=None):
    """The batched ensemble: nboxes independent x-y periodic shear boxes
    with particle counts uniform in [counts], radii U[r_range], packed to
    ~porosity on the GPU in one handle (FCC start, sph_relax of all boxes
    at once, radii grown by 1 + inflate), each with its own normal stress
    U[10, 80] kPa and friction mu U[0.3, 0.6] (_shear_setup).  subset: the
    indexes of the boxes to make (the others are drawn but not packed); a
    box is the same whichever subset it is made in (boxes relax
    independently), so ranks can each make their own share."""
    from .runner import Stepper
    rng = numpy.random.default_rng(seed)
    starts = []
    for b in range(nboxes):
        n = int(rng.integers(counts[0], counts[1] + 1))
        r = rng.uniform(r_range[0], r_range[1], n)
        s, _H = _fcc_start(n, rng, r, porosity, 0.5, float(r.mean()), "box%03d" % b)
        starts.append(s)
    setup = [(float(rng.uniform(1.0e4, 8.0e4)), float(rng.uniform(0.3, 0.6))) for _ in range(nboxes)]
    keep = list(range(nboxes)) if subset is None else [int(b) for b in subset]
    sims = [starts[b] for b in keep]
    if sims:
        st = Stepper(sims, device=device)
        st.upload()
        st.relax(sweeps, alpha=0.6, z_top=1e300)
        st.to_sims()
        st.close()
    for b, s in zip(keep, sims):
        s.radius *= 1.0 + inflate
        _shear_setup(s, sigma0=setup[b][0], mu=setup[b][1], steps=steps)
    return sims


def ensemble_counts(nboxes=256, seed=0, counts=(500, 20000)):
    """The particle counts of shear_ensemble's boxes (the same draws, no
    packing), to partition the boxes before they are made."""
    rng = numpy.random.default_rng(seed)
    out = []
    for _ in range(nboxes):
        n = int(rng.integers(counts[0], counts[1] + 1))
        out.append(n)
        rng.uniform(0.0, 1.0, n)          # the radii
        rng.uniform(-1.0, 1.0, (n, 3))    # the FCC start's jitter
    return out


def sheared_dense_pack(n=1000000, seed=0, device=-1, sweeps=3000, relax=None):
    """The 1e6-sphere sheared dense pack: log-normal radii (median 0.01 m,
    sigma_ln 0.2, clipped to [0.005, 0.02]) packed to porosity ~0.40 in an
    x-y periodic box of aspect 1:1:0.5 (dense_pack, on the GPU), a top wall
    at 20 kPa normal stress (wmode 1, mass = total particle mass as in
    sim.consolidate), the top layer moving at +x 0.01 m/s and the bottom
    layer held (fixvel, as in sim.shear), linear contacts
    k_n = k_t = 1.16e9 N/m, gamma_n = 1e3, mu = 0.5, NC = 32 slots,
    dt = 0.17 * sqrt(m_min / k_n), 5,000 steps.  `relax`: as in dense_pack."""
    s, _worst = dense_pack(n, seed=seed, device=device, sweeps=sweeps, sid="shear1e6",
                           relax=relax)
    return _shear_setup(s, sigma0=2.0e4, mu=0.5, steps=5000)


def _relax_cpu(x, r, lo, hi, iters=4000, tol=1e-12):
    """Overlap removal on the host: Jacobi sweeps that push every
    overlapping pair apart by half its overlap each, positions clamped to
    [lo + r, hi - r].  Stops when the largest overlap is below tol * r."""
    from scipy.spatial import cKDTree
    rmax = float(r.max())
    for _ in range(iters):
        pairs = cKDTree(x).query_pairs(2.0 * rmax, output_type="ndarray")
        if len(pairs) == 0:
            break
        i, j = pairs[:, 0], pairs[:, 1]
        d = x[i] - x[j]
        dist = numpy.sqrt((d * d).sum(1))
        ov = r[i] + r[j] - dist
        hit = ov > 0.0
        if not hit.any() or ov[hit].max() < tol * rmax:
            break
        i, j, d, dist, ov = i[hit], j[hit], d[hit], dist[hit], ov[hit]
        u = d / numpy.maximum(dist, 1e-30)[:, None]
        push = (0.75 * ov)[:, None] * u
        dx = numpy.zeros_like(x)
        numpy.add.at(dx, i, push)
        numpy.add.at(dx, j, -push)
        x += dx
        x[:] = numpy.clip(x, lo + r[:, None], hi - r[:, None])
    return x


def loose_pack(n=50000, seed=0, porosity=0.5, r_range=(0.009, 0.011), vel_sigma=0.1,
               k_n=1.5e8, gamma_n=20.0, mu=0.5, g=(0.0, 0.0, -9.81), nsteps=2000, device=None,
               sweeps=4000, sid="loose"):
    """The differentiable settling/impact scene: n spheres, radii
    U[r_range], random loose pack at the given porosity in a cube with fixed
    walls on all sides (uniform random positions, then overlap removal: on
    the host, or with sph_relax on GPU `device` when one is given),
    initial velocities N(0, vel_sigma) per component, no spin, linear
    contacts with k_t = k_n, gamma_t = 0, mu_s = mu_d = mu, wall damping
    gamma_wn = gamma_n, dt = 0.17 * sqrt(m_min / k_n), nsteps steps."""
    rng = numpy.random.default_rng(seed)
    s = sim(np=n, nw=0, sid=sid)
    r = rng.uniform(r_range[0], r_range[1], n)
    s.radius[:] = r
    side = (float(numpy.sum(4.0 / 3.0 * math.pi * r ** 3)) / (1.0 - porosity)) ** (1.0 / 3.0)
    x = rng.uniform(0.0, side, (n, 3))
    x = numpy.clip(x, r[:, None], side - r[:, None])
    s.periodic[0] = 0
    s.defineWorldBoundaries(L=[side, side, side])
    if device is None:
        s.x[:] = _relax_cpu(x, r, 0.0, side)
    else:
        from .runner import Stepper
        s.x[:] = x
        s.time_dt[0] = 1e-7
        s.time_total[0] = 1.0
        st = Stepper([s], device=device)
        st.upload()
        st.relax(sweeps, alpha=1.0, z_top=side)
        st.to_sims()
        st.close()
        s.radius[:] = r
    s.vel[:] = rng.normal(0.0, vel_sigma, (n, 3))
    s.g[:] = g
    s.k_n[0] = s.k_t[0] = k_n
    s.gamma_n[0] = gamma_n
    s.gamma_t[0] = 0.0
    s.gamma_wn[0] = gamma_n
    s.gamma_wt[0] = 0.0
    s.mu_s[0] = s.mu_d[0] = mu
    m_min = s.rho[0] * V_sphere(r_range[0])
    s.time_dt[0] = 0.17 * math.sqrt(m_min / k_n)
    s.time_current[0] = 0.0
    s.time_total[0] = nsteps * s.time_dt[0]
    s.time_file_dt[0] = s.time_total[0]
    return s


def reparam(s, k_n=None, gamma_n=None, mu=None):
    """A copy of sim s with the contact parameters the adjoint
    differentiates replaced (mu sets mu_s and mu_d); k_t, the wall damping
    and the time step are kept."""
    import copy
    q = copy.deepcopy(s)
    if k_n is not None:
        q.k_n[0] = k_n
    if gamma_n is not None:
        q.gamma_n[0] = gamma_n
    if mu is not None:
        q.mu_s[0] = q.mu_d[0] = mu
    return q
