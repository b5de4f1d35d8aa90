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
