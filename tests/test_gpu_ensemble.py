"""Several independent boxes stepped by the same kernel launches (one
handle, segmented cell grids) must give, box by box, exactly what each box
gives alone: the CPU oracle run of that box."""
import numpy
import pytest

import cases
import oracle as O
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("names", [
    ["periodic_xy_wall_stress", "walls_all_sides", "bonds", "youngs_modulus", "contact_model_1"],
    ["shear_stress_wall", "periodic_x_wall_velocity", "bonds_breaking", "adaptive_grid"],
])
def test_ensemble_equals_each_box_alone(names):
    sims = [cases.make(n)[0] for n in names]
    steps = 12
    ens = Stepper(sims)
    ens.upload()
    ens.step(5)
    ens.step(steps - 5)
    hp, hb = ens.download()
    c, dt, dm = ens.contacts()
    boxes = ens.boxes()
    o = ob = 0
    for s, b in zip(sims, boxes):
        n, nb = int(s.np[0]), int(s.nb0[0])
        cpu = O.CpuRun(s, "oracle")
        cpu.step(steps)
        assert numpy.array_equal(hp.x[o:o + n], cpu.x)
        assert numpy.array_equal(hp.vel[o:o + n], cpu.vel)
        assert numpy.array_equal(hp.force[o:o + n], cpu.force[:, :3])
        assert numpy.array_equal(hp.torque[o:o + n], cpu.torque[:, :3])
        assert numpy.array_equal(hp.es[o:o + n], cpu.es)
        assert numpy.array_equal(c[o * 32:(o + n) * 32], cpu.contacts)
        assert numpy.array_equal(dt[o * 32:(o + n) * 32], cpu.delta_t)
        if nb:
            assert numpy.array_equal(hb.pairs[ob:ob + nb], cpu.bonds[:nb])
            assert numpy.array_equal(hb.delta_n[ob:ob + nb], cpu.bonds_delta[:nb, 3])
        for w in range(int(s.nw[0])):
            assert list(b.walls.nx[w]) == list(cpu.box.walls.nx[w])
        assert b.t_current == cpu.box.t_current
        o += n
        ob += nb
    ens.close()
