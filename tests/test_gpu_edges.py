"""Edge cases of the step on the GPU: a non-finite position or one outside
the grid is refused at upload (SPH_ERR_INPUT, the reference's checkValues);
a sphere that leaves the grid during the steps is reported
(SPH_ERR_OUT_OF_GRID, the reference's checks of device.cu:241-276); a
sphere with more than NC = 32
contacts is reported (SPH_ERR_NC_OVERFLOW) and the rest of the step equals
the oracle's; a box without spheres steps (its time advances, its walls
stay, as in the reference, which allows np = 0, src/sphere.cpp:169-172),
alone and inside a ragged ensemble; a single sphere falls as the oracle's
does."""
import math

import numpy
import pytest

import cases
import oracle as O
from sphere_b200 import _abi
from sphere_b200 import sim as simclass
from sphere_b200.runner import SphereError, Stepper
from test_gpu_parity import check_same

pytestmark = pytest.mark.gpu


def _status(name):
    return {v: k for k, v in _abi.STATUS_NAMES.items()}[name]


def _params(s, dt_scale=0.17):
    s.k_n[0] = s.k_t[0] = 1.16e9
    s.gamma_n[0] = 100.0
    s.gamma_t[0] = 50.0
    s.mu_s[0] = s.mu_d[0] = 0.5
    s.contactmodel[0] = 2
    m_min = s.rho[0] * 4.0 / 3.0 * math.pi * float(numpy.min(s.radius)) ** 3
    s.time_dt[0] = dt_scale * math.sqrt(m_min / s.k_n[0])
    s.time_total[0] = 1.0
    s.time_file_dt[0] = 1.0


def test_bad_positions_are_refused_at_upload():
    """The reference's checkValues (src/sphere.cpp:233-262) on the input."""
    for field, value in ((1, numpy.nan), (2, 1.5)):
        s, _, _ = cases.make("walls_all_sides")
        s.x[5, field] = value if field == 1 else value * float(s.L[2])
        st = Stepper([s], precision="fp64")
        with pytest.raises(SphereError) as e:
            st.upload()
        assert e.value.status == _status("SPH_ERR_INPUT")
        # the refused input leaves no state to step
        with pytest.raises(SphereError) as e:
            st.step(1)
        assert e.value.status == _status("SPH_ERR_STATE")
        st.close()


def test_first_bad_particle_is_named_in_a_large_box():
    # a box large enough for the check to be split over host threads: the
    # message names the first failing particle in index order
    from sphere_b200 import scenes
    s = scenes.lattice_pack(200000, seed=5, periodic=1, nw=0)
    n = int(s.np[0])
    late, later = n - 7, n - 3
    s.x[later, 0] = numpy.nan
    s.radius[late] = -1.0
    st = Stepper([s], precision="fp64")
    with pytest.raises(SphereError) as e:
        st.upload()
    assert e.value.status == _status("SPH_ERR_INPUT")
    assert "particle %d has a radius" % late in str(e.value)
    s.radius[late] = float(numpy.median(s.radius))
    with pytest.raises(SphereError) as e:
        st.upload()
    assert "particle %d has NaN values" % later in str(e.value)
    s.x[later, 0] = s.x[later - 1, 0]
    s.x[n // 3, 2] = 10.0 * float(s.L[2])
    with pytest.raises(SphereError) as e:
        st.upload()
    assert "particle %d is outside" % (n // 3) in str(e.value)
    st.close()


def test_sphere_leaving_the_grid_is_reported():
    """A sphere that crosses the top of the grid during the steps (walls on
    all sides are implicit in the reference only at L; z is never
    periodic): the next cell hash reports it (device.cu:241-276)."""
    s, _, _ = cases.make("walls_all_sides")
    k = int(numpy.argmax(s.x[:, 2]))
    s.vel[k] = [0.0, 0.0, 0.0]
    s.vel[k, 2] = (float(s.L[2]) - float(s.x[k, 2])) / (2.0 * float(s.time_dt[0]))
    s.g[:] = 0.0
    st = Stepper([s], precision="fp64")
    st.upload()
    with pytest.raises(SphereError) as e:
        st.step(5)
    assert e.value.status == _status("SPH_ERR_OUT_OF_GRID")
    st.close()


def _crowded():
    """One sphere of radius 0.05 m touched by 40 spheres of 0.01 m spread
    over its surface (Fibonacci lattice), each overlapping it by 1 mm."""
    n = 40
    s = simclass(np=n + 1, nw=0, sid="crowded")
    c = numpy.array([0.25, 0.25, 0.25])
    s.radius[0] = 0.05
    s.radius[1:] = 0.01
    s.x[0] = c
    k = numpy.arange(n) + 0.5
    phi = numpy.arccos(1.0 - 2.0 * k / n)
    theta = math.pi * (1.0 + 5.0 ** 0.5) * k
    d = numpy.stack([numpy.cos(theta) * numpy.sin(phi), numpy.sin(theta) * numpy.sin(phi),
                     numpy.cos(phi)], 1)
    s.x[1:] = c + (0.05 + 0.01 - 0.001) * d
    s.defineWorldBoundaries([0.5, 0.5, 0.5])
    s.g[:] = 0.0
    _params(s)
    return s


@pytest.mark.parametrize("variant", [1, 3])
def test_contact_row_overflow_is_reported_and_the_rest_matches(variant):
    s = _crowded()
    st = Stepper([s], precision="fp64")
    st.upload()
    st.set_variant(variant)
    with pytest.raises(SphereError) as e:
        st.step(1)
    assert e.value.status == _status("SPH_ERR_NC_OVERFLOW")
    cpu = O.CpuRun(s, "oracle")
    cpu.step(1)
    check_same(st, cpu, s)
    c, _, _ = st.contacts()
    assert int((c[:32] != s.np[0]).sum()) == 32   # the crowded row is full
    st.close()


def _empty_box():
    s = simclass(np=0, nw=1, sid="empty")
    s.defineWorldBoundaries([0.3, 0.3, 0.3], dx=0.05)
    s.wmode = numpy.array([1], dtype=numpy.int32)
    s.w_n = numpy.array([[0.0, 0.0, -1.0]])
    s.w_x = numpy.array([0.2])
    s.w_m = numpy.array([1.0])
    s.w_vel = numpy.array([0.0])
    s.w_force = numpy.zeros(1)
    s.w_sigma0 = numpy.array([100.0])
    s.time_dt[0] = 1.0e-5
    s.time_total[0] = 1.0
    s.time_file_dt[0] = 1.0
    return s


def test_empty_box_steps_time_and_wall():
    s = _empty_box()
    st = Stepper([s], precision="fp64")
    st.upload()
    st.step(10)
    b = st.boxes()[0]
    assert b.t_current == pytest.approx(10 * 1.0e-5, rel=1e-12)
    # the reference integrates walls only inside its np > 0 branch
    # (src/device.cu:1039-2532): the wall stays, the time advances
    assert b.walls.nx[0][3] == 0.2
    st.close()


def test_ragged_ensemble_with_an_empty_box():
    sims = [cases.make("walls_all_sides")[0], _empty_box(), cases.make("fast_spheres")[0]]
    ens = Stepper(sims, precision="fp64")
    ens.upload()
    ens.step(7)
    hp, _ = ens.download()
    boxes = ens.boxes()
    o = 0
    for s, b in zip(sims, boxes):
        n = int(s.np[0])
        if n:
            cpu = O.CpuRun(s, "oracle")
            cpu.step(7)
            assert numpy.array_equal(hp.x[o:o + n], cpu.x)
            assert numpy.array_equal(hp.force[o:o + n], cpu.force[:, :3])
            assert b.t_current == cpu.box.t_current
        o += n
    alone = Stepper([sims[1]], precision="fp64")
    alone.upload()
    alone.step(7)
    assert list(alone.boxes()[0].walls.nx[0]) == list(boxes[1].walls.nx[0])
    ens.close()
    alone.close()


def test_single_sphere_falls_as_the_oracle():
    s = simclass(np=1, nw=0, sid="one")
    s.radius[0] = 0.01
    s.x[0] = [0.05, 0.05, 0.08]
    s.vel[0] = [0.1, 0.0, 0.0]
    s.defineWorldBoundaries([0.1, 0.1, 0.1])
    _params(s)
    st = Stepper([s], precision="fp64")
    st.upload()
    st.step(200)
    cpu = O.CpuRun(s, "oracle")
    cpu.step(200)
    check_same(st, cpu, s)
    st.close()
