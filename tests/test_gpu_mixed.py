"""The FP32-mixed step against the FP64 step.

The mixed form keeps the overlap test in FP64, so its contact lists must be
identical to the FP64 form's; its forces, computed with FP32 contact-law
arithmetic, must agree per step within 1e-5 relative L2 (the tolerance of
the precision target), torques within 1e-4, and positions after 100 steps
within 1e-4 of the mean radius."""
import numpy
import pytest

import cases
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
TORQUE_TOL = 1e-4


def rel_l2(a, b):
    return float(numpy.linalg.norm(a - b) / max(numpy.linalg.norm(b), 1e-300))


def contact_sets(c, n):
    rows = c.reshape(-1, 32)
    return [tuple(sorted(int(v) for v in r if v != n)) for r in rows]


@pytest.mark.parametrize("variant", [1, 3, 4])
@pytest.mark.parametrize("name", ["periodic_xy_wall_stress", "walls_all_sides", "contact_model_1",
                                  "youngs_modulus", "bonds", "contact_model_3_hertz",
                                  "shear_stress_wall"])
def test_mixed_step_error(name, variant):
    """variant 1: fused kernel; 3: split step; 4: the list step (where
    they apply).  The list step keeps its contacts in list order, so its
    contact rows are compared as sets."""
    s = cases.make(name)[0]
    a = Stepper([s], precision="fp64")
    b = Stepper([s], precision="mixed")
    b.set_variant(variant)
    a.upload()
    b.upload()
    a.step(1)
    b.step(1)
    pa, _ = a.download()
    pb, _ = b.download()
    assert rel_l2(pb.force, pa.force) < FORCE_TOL
    assert rel_l2(pb.torque, pa.torque) < TORQUE_TOL
    ca = a.contacts()[0]
    cb = b.contacts()[0]
    if variant == 4:
        n = int(s.np[0])
        assert contact_sets(ca, n) == contact_sets(cb, n)
    else:
        assert numpy.array_equal(ca, cb)
    a.close()
    b.close()


def test_mixed_positions_after_100_steps():
    s = cases.make("periodic_xy_wall_stress")[0]
    a = Stepper([s], precision="fp64")
    b = Stepper([s], precision="mixed")
    a.upload()
    b.upload()
    a.step(100)
    b.step(100)
    pa, _ = a.download()
    pb, _ = b.download()
    # largest position difference after 100 steps, relative to the mean
    # radius (measured ~1e-6 on this strongly overlapping lattice)
    dev = float(numpy.max(numpy.abs(pa.x[:, :3] - pb.x[:, :3]))) / float(numpy.mean(s.radius))
    print("mixed vs fp64: max |dx| / r_mean after 100 steps = %.3e" % dev)
    assert dev < 1e-4
    a.close()
    b.close()


def test_mixed_wall_stress_and_porosity_over_a_long_run():
    """A 20,000-sphere sheared dense pack (the benchmark's scene at a
    smaller size: 20 kPa on the top wall, top layer sheared), 2,000 steps,
    in the mixed form's default variant and in the list step, against the
    FP64 form.  The flow is chaotic, so the bound is the floor two FP64
    runs show when one starts from positions moved by one part in 1e15:
    measured on this scene over four such moves, mean stress over the
    second half 1.7e-5 to 8.6e-5, RMS 1.9e-3 to 2.0e-3, positions 9.0e-4 r
    to 1.1e-3 r at the end; the mixed form within a few times that."""
    import json
    from sphere_b200 import scenes
    from sphere_b200.mixed_error import compare_precisions
    s = scenes.sheared_dense_pack(n=20000, seed=3, device=0, sweeps=1500)
    floor = [compare_precisions(s, nsteps=2000, slices=20, device=0, precision="fp64",
                                perturb=1e-15, seed=k) for k in (0, 1)]
    print(json.dumps(floor))
    top = {k: max(f[k] for f in floor) for k in floor[0] if isinstance(floor[0][k], float)}
    for variant in (None, 4):
        e = compare_precisions(s, nsteps=2000, slices=20, device=0, variant=variant)
        print(json.dumps(e))
        assert e["status"] == [0, 0]
        assert e["times_equal"]
        assert e["wall_stress_mean_rel_diff_second_half"] < 5e-4
        assert e["wall_stress_rms_diff_over_rms"] < 2.0 * top["wall_stress_rms_diff_over_rms"]
        assert e["positions_max_diff_over_rmean"] < 3.0 * top["positions_max_diff_over_rmean"]
        assert e["bulk_porosity_max_abs_diff"] < max(1e-7, 10.0 * top["bulk_porosity_max_abs_diff"])
        assert e["porosity_profile_max_abs_diff"] < max(1e-5, 10.0 * top["porosity_profile_max_abs_diff"])
