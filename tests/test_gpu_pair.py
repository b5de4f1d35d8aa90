"""The list step of the FP32-mixed form (launch variant 4) against the FP64
form and against itself.

Its contact set is the FP64 form's (the same FP64 overlap test), its
tangential histories are kept per neighbour-list entry, its sums run in
list order, and its state is stored compactly (FP32 where the mixed form
allows), so it is held to the mixed form's stated error:

* one step from the same state (with the same contact histories, handed
  over from the FP64 contact rows): force relative L2 <= 1e-5, torque
  <= 1e-4, the same contact set per sphere;
* rebuilding the lists every step gives the same bits as rebuilding them
  when the skin asks for it (the histories are carried over exactly, and
  the sums do not depend on what else the lists hold);
* two runs give the same bits; handing the state to the split step and
  back keeps the error bound;
* ensembles: box by box within the bound.
"""
import copy

import numpy
import pytest

import cases
from sphere_b200 import _abi, scenes
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

PAIR = 4
FORCE_TOL = 1e-5
TORQUE_TOL = 1e-4


def rel_l2(a, b):
    return float(numpy.linalg.norm(a - b) / max(numpy.linalg.norm(b), 1e-300))


def contact_sets(c, n):
    """Per sphere, the sorted partner indexes of its contact row."""
    rows = c.reshape(-1, 32)
    return [tuple(sorted(int(v) for v in r if v != n)) for r in rows]


def history_by_partner(c, dt, n):
    out = {}
    rows = c.reshape(-1, 32)
    h = dt.reshape(-1, 32, 4)
    for i in range(rows.shape[0]):
        for s in range(32):
            if rows[i, s] != n:
                out[(i, int(rows[i, s]))] = h[i, s, :3].copy()
    return out


def _restart(st):
    """The state of handle st as a new sim (a copy, as an output file holds
    it) with its contact rows and histories."""
    sims = copy.deepcopy(st.sims)
    st.to_sims()
    state = copy.deepcopy(st.sims)
    st.sims[:] = sims
    c, dt, _ = st.contacts()
    return state, c, dt


def _one_step(state, c, dt, precision, variant, length="reference"):
    q = Stepper(copy.deepcopy(state), precision=precision, length=length)
    q.set_variant(variant)
    q.upload()
    q.set_contacts(c, dt)
    q.step(1)
    hp, _ = q.download()
    cc = q.contacts()
    boxes = q.boxes()
    q.close()
    return hp, cc, boxes


def _pair_one_step_vs_fp64(s, warm, length="reference"):
    """warm steps of the FP64 form, then from that state (contact rows and
    histories handed over with sph_set_contacts) one step in the FP64 form
    and one in the list step."""
    a = Stepper([copy.deepcopy(s)], precision="fp64", length=length)
    a.upload()
    a.step(warm)
    state, c, dt = _restart(a)
    a.close()
    pa, ca, _ = _one_step(state, c, dt, "fp64", 1, length)
    pb, cb, _ = _one_step(state, c, dt, "mixed", PAIR, length)
    return pa, pb, ca, cb


@pytest.mark.parametrize("name", ["periodic_xy_wall_stress", "walls_all_sides", "youngs_modulus",
                                  "contact_model_3_hertz", "fast_spheres",
                                  "periodic_x_wall_velocity", "fixvel_modes"])
@pytest.mark.parametrize("length", ["reference", "fp64"])
def test_pair_step_error_vs_fp64(name, length):
    s = cases.make(name)[0]
    n = int(s.np[0])
    for warm in (0, 7):
        pa, pb, ca, cb = _pair_one_step_vs_fp64(s, warm, length)
        assert rel_l2(pb.force, pa.force) < FORCE_TOL, (warm, rel_l2(pb.force, pa.force))
        assert rel_l2(pb.torque, pa.torque) < TORQUE_TOL
        assert contact_sets(ca[0], n) == contact_sets(cb[0], n)
        # the histories of the same pairs agree to the law's FP32 rounding
        ha = history_by_partner(ca[0], ca[1], n)
        hb = history_by_partner(cb[0], cb[1], n)
        assert ha.keys() == hb.keys()
        if ha:
            A = numpy.array([ha[k] for k in sorted(ha)])
            B = numpy.array([hb[k] for k in sorted(ha)])
            assert rel_l2(B, A) < 1e-5


def test_pair_rebuild_every_step_changes_no_bit():
    s = cases.make("fast_spheres")[0]
    runs = []
    for forced in (False, True):
        st = Stepper([s], precision="mixed")
        st.set_variant(PAIR)
        st.upload()
        for _ in range(40):
            if forced:
                st.set_neighbor_lists(48)   # asks for a rebuild before the next step
            st.step(1)
        hp, _ = st.download()
        c, dt, _ = st.contacts()
        builds = st.neighbor_stats()["builds"]
        runs.append((hp, c, dt, builds))
        st.close()
    (a, ca, ta, ba), (b, cb, tb, bb) = runs
    assert bb == 40 and ba < bb
    for name in ("x", "vel", "angvel", "force", "torque", "es", "ev", "p"):
        assert numpy.array_equal(getattr(a, name), getattr(b, name)), name
    assert numpy.array_equal(ca, cb) and numpy.array_equal(ta, tb)


def test_pair_deterministic_and_runs_equal_single_steps():
    s = cases.make("periodic_xy_wall_stress")[0]
    out = []
    for chunks in ((20,), (1,) * 20, (20,)):
        st = Stepper([s], precision="mixed")
        st.set_variant(PAIR)
        st.upload()
        for k in chunks:
            st.step(k)
        hp, _ = st.download()
        out.append((hp.x.copy(), hp.force.copy(), st.boxes()[0].walls.nx[0][3]))
        st.close()
    for o in out[1:]:
        assert numpy.array_equal(o[0], out[0][0]) and numpy.array_equal(o[1], out[0][1])
        assert o[2] == out[0][2]


def test_pair_hands_state_to_the_split_step_and_back():
    """20 list steps, 5 split steps (on the contact rows the list step
    wrote), 20 list steps: at the end of each stretch, one more step of it
    within the mixed bound of an FP64 step from the same state."""
    s = cases.make("periodic_xy_wall_stress")[0]
    st = Stepper([copy.deepcopy(s)], precision="mixed")
    st.upload()
    for variant, k in ((PAIR, 20), (3, 5), (PAIR, 20)):
        st.set_variant(variant)
        st.step(k)
        state, c, dt = _restart(st)
        pa, _, _ = _one_step(state, c, dt, "fp64", 1)
        pb, _, _ = _one_step(state, c, dt, "mixed", variant)
        assert rel_l2(pb.force, pa.force) < FORCE_TOL, (variant, rel_l2(pb.force, pa.force))
    st.close()


def test_pair_ensemble_box_by_box():
    sims = scenes.shear_ensemble(nboxes=6, seed=2, device=0, counts=(300, 3000), sweeps=400)
    a = Stepper(sims, precision="fp64")
    b = Stepper(sims, precision="mixed")
    b.set_variant(PAIR)
    a.upload()
    b.upload()
    a.step(1)
    b.step(1)
    pa, _ = a.download()
    pb, _ = b.download()
    o = 0
    for q in sims:
        k = int(q.np[0])
        assert rel_l2(pb.force[o:o + k], pa.force[o:o + k]) < FORCE_TOL
        o += k
    ta = [x.t_current for x in a.boxes()]
    tb = [x.t_current for x in b.boxes()]
    assert ta == tb
    a.step(30)
    b.step(30)
    xa, _ = a.download()
    xb, _ = b.download()
    dev = float(numpy.max(numpy.abs(xa.x[:, :3] - xb.x[:, :3]))) / 0.01
    assert dev < 1e-4, dev
    a.close()
    b.close()


def test_pair_shapes_same_bits_under_a_loaded_wall():
    """A 6,000-sphere sheared pack with its top wall lowered onto the pack:
    over a hundred spheres press on it, so the wall-force sums (per chunk of
    spheres, then per box) add many terms; the persistent shapes run them
    with their own block sizes and must add them in the same order as the
    chunk and box kernels."""
    s = scenes.sheared_dense_pack(n=6000, seed=4, device=0, sweeps=800)
    # the wall lowered onto the pack's top 2 % (held spheres, overlaps of
    # about 1e-4 m at most)
    s.w_x[0] = numpy.quantile(s.x[:, 2] + s.radius, 0.98)
    out = {}
    for shape in range(_abi.PAIR_SHAPES):
        st = Stepper([copy.deepcopy(s)], precision="mixed")
        st.set_variant(PAIR)
        st.set_launch_shape(shape)
        st.upload()
        st.step(20)
        hp, _ = st.download()
        out[shape] = (hp, st.boxes()[0])
        st.close()
    a, ba = out[0]
    # spheres in contact with the top wall (x[:, 3] is the radius)
    assert numpy.count_nonzero(a.x[:, 2] + a.x[:, 3] > ba.walls.nx[0][3]) > 100
    for shape, (b, bb) in out.items():
        assert list(ba.walls.mvfd[0]) == list(bb.walls.mvfd[0]), shape
        assert list(ba.walls.nx[0]) == list(bb.walls.nx[0]), shape
        for f in ("x", "vel", "force"):
            assert numpy.array_equal(getattr(a, f), getattr(b, f)), (shape, f)


@pytest.mark.parametrize("name", ["fast_spheres", "periodic_xy_wall_stress"])
def test_pair_shapes_give_the_same_bits(name):
    """Every launch shape of the list step (register budgets, staged
    gathers, the persistent kernel with its grid barriers, loads without
    look-ahead) runs the same arithmetic in the same order: the file is
    compiled without FMA contraction, so no register budget can change
    which multiply-adds are fused."""
    s = cases.make(name)[0]
    out = {}
    for shape in range(_abi.PAIR_SHAPES):
        st = Stepper([s], precision="mixed")
        st.set_variant(PAIR)
        st.set_launch_shape(shape)
        st.upload()
        st.step(30)
        hp, _ = st.download()
        out[shape] = (hp, st.boxes()[0])
        st.close()
    a, ba = out[0]
    for shape, (b, bb) in out.items():
        for f in ("x", "vel", "angvel", "force", "torque", "es", "ev"):
            assert numpy.array_equal(getattr(a, f), getattr(b, f)), (shape, f)
        assert ba.t_current == bb.t_current
        assert list(ba.walls.nx[0]) == list(bb.walls.nx[0])
