"""sph_snapshot / sph_snapshot_read: the state at the snapshot, read back
while later steps run, equals a synchronous download taken at the same
step; and run() through it writes the same files as before (tested in
test_gpu_run.py)."""
import numpy
import pytest

import cases
from sphere_b200.runner import SphereError, Stepper

pytestmark = pytest.mark.gpu


def test_snapshot_equals_download_at_the_same_step():
    s, _, _ = cases.make("fast_spheres")
    a = Stepper([s], precision="fp64")
    b = Stepper([s], precision="fp64")
    a.upload()
    b.upload()
    a.step_async(7)
    a.snapshot()
    a.step_async(11)            # later steps do not change the snapshot
    code, hp, _, boxes = a.snapshot_read()
    assert code == 0
    b.step(7)
    ref, _ = b.download()
    for name in ("x", "vel", "force", "torque", "angpos", "angvel", "xyzsum", "es", "ev", "p"):
        assert numpy.array_equal(getattr(hp, name), getattr(ref, name)), name
    assert boxes[0].t_current == b.boxes()[0].t_current
    a.sync()
    b.step(11)
    fin_a, _ = a.download()
    fin_b, _ = b.download()
    assert numpy.array_equal(fin_a.x, fin_b.x)
    a.close()
    b.close()


def test_snapshot_read_without_snapshot_is_refused():
    s, _, _ = cases.make("walls_all_sides")
    a = Stepper([s], precision="fp64")
    a.upload()
    with pytest.raises(SphereError):
        a.snapshot_read()
    a.snapshot()
    assert a.snapshot_read()[0] == 0
    with pytest.raises(SphereError):
        a.snapshot_read()            # one read per snapshot
    a.close()


def _box_fields(b):
    return ([b.grid.L[c] for c in range(3)], [list(b.walls.nx[w]) for w in range(b.walls.nw)],
            [list(b.walls.mvfd[w]) for w in range(b.walls.nw)], b.t_current)


@pytest.mark.parametrize("name,nsteps", [("periodic_xy_wall_stress", 9),
                                         ("periodic_x_wall_velocity", 6),
                                         ("shear_stress_wall", 5), ("adaptive_grid", 7),
                                         ("walls_all_sides", 1),
                                         # more steps than the 128-step ring
                                         ("fixvel_modes", 300)])
def test_step_states_equal_a_read_after_every_step(name, nsteps):
    # two boxes in one handle; the queued run (the wall stage beside the
    # next step where the handle allows it) against one synchronous read
    # per step
    s, _, _ = cases.make(name)
    s2, _, _ = cases.make("fixvel_modes")
    a = Stepper([s, s2], precision="fp64")
    b = Stepper([s, s2], precision="fp64")
    a.upload()
    b.upload()
    nb = a.box_state_bytes()
    assert nb > 0 and nb % 8 == 0
    states = numpy.zeros((nsteps, nb), dtype=numpy.uint8)
    a.step_async_states(nsteps, states)
    a.sync()
    bulk = a.boxes_from_states(states)
    assert len(bulk) == nsteps
    for k in range(nsteps):
        b.step(1)
        want = b.boxes()
        got = a.boxes_from_state(states[k])
        for bw, bg, bb in zip(want, got, bulk[k]):
            assert _box_fields(bg) == _box_fields(bw), (name, k)
            assert _box_fields(bb) == _box_fields(bw), (name, k)
    fa, _ = a.download()
    fb, _ = b.download()
    assert numpy.array_equal(fa.x, fb.x)
    one = numpy.zeros(nb, dtype=numpy.uint8)
    a.get_boxes_async(one)
    a.sync()
    assert [_box_fields(x) for x in a.boxes_from_state(one)] == \
        [_box_fields(x) for x in a.boxes()]
    a.close()
    b.close()


def test_step_states_buffer_too_small_is_refused():
    s, _, _ = cases.make("periodic_xy_wall_stress")
    a = Stepper([s], precision="fp64")
    a.upload()
    nb = a.box_state_bytes()
    with pytest.raises(SphereError):
        a.step_async_states(3, numpy.zeros(3 * nb - 1, dtype=numpy.uint8))
    with pytest.raises(SphereError):
        a.get_boxes_async(numpy.zeros(nb - 1, dtype=numpy.uint8))
    a.step(1)
    a.close()
