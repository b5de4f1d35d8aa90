"""CUDA step (through the C ABI) against the FP64 CPU oracle.

Every parity case is stepped on the GPU (libsphere_b200.so, via
sphere_b200.runner.Stepper -> sph_create/sph_upload/sph_step/...) and by the
oracle from the same initial state; all particle state, energies, contact
lists, tangential histories, periodic shifts, the cell sort and the walls
must agree bit for bit (FP64 form, reference length mode).  The cases
driven through a transcendental function (sin of the sinusoidal wall
stress, expf of the capillary force) are compared within the tolerances of
cases.APPROX, since CUDA and glibc may round those differently.
"""
import numpy
import pytest

import cases
import oracle as O
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

NC = 32


def _cmp(a, b, name, approx):
    """approx: None or False for bit-exact, else the tolerance relative to
    the field's largest magnitude."""
    if approx:
        scale = max(float(numpy.max(numpy.abs(b))), 1e-300)
        assert numpy.allclose(a, b, rtol=approx, atol=approx * scale), name
    else:
        assert numpy.array_equal(a, b), "%s differs (max |d| = %g)" % (
            name, float(numpy.max(numpy.abs(a.astype(float) - b.astype(float)))))


def check_same(st, cpu, s, approx=None):
    n = int(s.np[0])
    hp, hb = st.download()
    _cmp(hp.x, cpu.x, "x", approx)
    _cmp(hp.vel, cpu.vel, "vel", approx)
    for name in ("xyzsum", "force", "angpos", "angvel", "torque"):
        _cmp(getattr(hp, name), getattr(cpu, name)[:, :3], name, approx)
    for name in ("es_dot", "es", "ev_dot", "ev", "p"):
        _cmp(getattr(hp, name), getattr(cpu, name), name, approx)
    c, dt, dm = st.contacts()
    assert numpy.array_equal(c, cpu.contacts), "contact lists differ"
    _cmp(dt, cpu.delta_t, "delta_t", approx)
    live = c != n
    assert numpy.array_equal(dm[live], cpu.distmod[live]), "distmod differs"
    cid, perm, cs, ce = st.sort_products()
    assert numpy.array_equal(cid, cpu.cell_id[:n]), "cell ids differ"
    assert numpy.array_equal(perm, cpu.perm[:n]), "sorted permutation differs"
    assert numpy.array_equal(cs, cpu.cell_start), "cellStart differs"
    nonempty = cs != 0xffffffff
    assert numpy.array_equal(ce[nonempty], cpu.cell_end[nonempty]), "cellEnd differs"
    nb0 = int(s.nb0[0])
    if nb0:
        assert numpy.array_equal(hb.pairs, cpu.bonds[:nb0])
        _cmp(hb.delta_t, cpu.bonds_delta[:nb0, :3], "bonds_delta_t", approx)
        _cmp(hb.delta_n, cpu.bonds_delta[:nb0, 3], "bonds_delta_n", approx)
        _cmp(hb.omega_t, cpu.bonds_omega[:nb0, :3], "bonds_omega_t", approx)
        _cmp(hb.omega_n, cpu.bonds_omega[:nb0, 3], "bonds_omega_n", approx)
    b = st.boxes()[0]
    for w in range(int(s.nw[0])):
        _cmp(numpy.array(b.walls.nx[w][:]), numpy.array(cpu.box.walls.nx[w][:]), "wall nx", approx)
        _cmp(numpy.array(b.walls.mvfd[w][:]), numpy.array(cpu.box.walls.mvfd[w][:]), "wall mvfd",
             approx)
    assert b.grid.L[2] == cpu.box.grid.L[2]
    assert b.t_current == cpu.box.t_current


@pytest.mark.parametrize("lists", [48, 0, 3])
@pytest.mark.parametrize("length", ["reference", "fp64"])
@pytest.mark.parametrize("name", cases.CASES)
def test_gpu_matches_oracle(name, length, lists):
    """lists: neighbour-list capacity (48 = default, 0 = cell search only,
    3 = most spheres overflow their list and fall back to the cell search
    while others use theirs, in the same step)."""
    s, _ref_ok, steps = cases.make(name)
    cpu = O.CpuRun(s, "oracle", length_mode=0 if length == "reference" else 1)
    st = Stepper([s], precision="fp64", length=length)
    st.set_neighbor_lists(lists)
    st.upload()
    done = 0
    for chunk in (1, steps // 2 - 1, steps - steps // 2):
        st.step(chunk)
        cpu.step(chunk)
        done += chunk
        check_same(st, cpu, s, approx=cases.APPROX.get(name))
    assert st.kernel_launches() > 0
    st.close()


def test_gpu_deterministic():
    s, _, steps = cases.make("periodic_xy_wall_stress")
    out = []
    for _ in range(2):
        st = Stepper([s])
        st.upload()
        st.step(steps)
        hp, _ = st.download()
        c, dt, _dm = st.contacts()
        out.append((hp.x.copy(), hp.force.copy(), c.copy(), dt.copy()))
        st.close()
    for a, b in zip(out[0], out[1]):
        assert numpy.array_equal(a, b)


@pytest.mark.parametrize("length", ["reference", "fp64"])
@pytest.mark.parametrize("variant", [0, 2, 3])
@pytest.mark.parametrize("name", ["periodic_xy_wall_stress", "walls_all_sides", "fast_spheres",
                                  "shear_stress_wall", "contact_model_3_hertz", "youngs_modulus",
                                  "bonds_breaking", "adaptive_grid", "fixvel_modes"])
def test_launch_variants_match_oracle(name, variant, length):
    """Every launch variant of the interact stage gives the same bits: the
    fused kernel for register budgets 255 and 80 (128 is the default above)
    and the split step (variant 3; cases it does not cover, such as the
    shear-stress wall, fall back to the fused kernel)."""
    s, _ref_ok, steps = cases.make(name)
    cpu = O.CpuRun(s, "oracle", length_mode=0 if length == "reference" else 1)
    st = Stepper([s], precision="fp64", length=length)
    st.set_variant(variant)
    st.upload()
    st.step(steps)
    cpu.step(steps)
    check_same(st, cpu, s, approx=cases.APPROX.get(name))
    st.close()


def test_autotune_keeps_the_state_and_the_bits():
    s, _, steps = cases.make("fast_spheres")
    a = Stepper([s], precision="fp64")
    a.upload()
    a.step(3)
    before, _ = a.download()
    c_before = a.contacts()[0].copy()
    chosen, ms = a.autotune(steps=5)
    # variants 0-3 apply to the FP64 form; the list step (4) is the mixed
    # form's and is not tried (-1)
    assert chosen in (0, 1, 2, 3) and all(m > 0.0 for m in ms[:4]) and ms[4] == -1.0
    after, _ = a.download()
    assert numpy.array_equal(before.x, after.x) and numpy.array_equal(before.vel, after.vel)
    assert numpy.array_equal(c_before, a.contacts()[0])
    b = Stepper([s], precision="fp64")
    b.upload()
    b.step(3)
    a.step(steps)
    b.step(steps)
    ha, _ = a.download()
    hb, _ = b.download()
    assert numpy.array_equal(ha.x, hb.x) and numpy.array_equal(ha.force, hb.force)
    assert a.boxes()[0].t_current == b.boxes()[0].t_current
    a.close()
    b.close()
