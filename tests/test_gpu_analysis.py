"""sph_porosity and sph_overlaps (sim.porosity, sim.findOverlaps) against
the oracle's restatement of the reference's analysis code, bit for bit, on
the parity scenes and after some steps; and the sim-level helpers on top."""
import numpy
import pytest

import cases
import oracle as O
from sphere_b200.runner import SphereError, Stepper

pytestmark = pytest.mark.gpu

NAMES = ["walls_all_sides", "periodic_xy_wall_stress", "fixvel_modes", "fast_spheres"]


@pytest.mark.parametrize("name", NAMES)
def test_porosity_and_overlaps_match_oracle(name):
    s, _, steps = cases.make(name)
    st = Stepper([s], precision="fp64")
    st.upload()
    st.step(steps)
    st.to_sims()               # the sim now holds the stepped state
    for slices in (2, 4):
        z, p = st.porosity(slices)
        ref = O.porosity(s, slices)
        assert numpy.array_equal(z, ref[0]) and numpy.array_equal(p, ref[1])
    pairs, d = st.overlaps()
    rp, rd = O.overlaps(s)
    assert len(pairs) > 0
    assert numpy.array_equal(pairs, rp) and numpy.array_equal(d, rd)
    with pytest.raises(SphereError):
        st.porosity(10000)
    st.close()


def test_sim_analysis_helpers():
    s, _, _ = cases.make("walls_all_sides")
    p, depth = s.porosity(slices=4)
    ref = O.porosity(s, 4)
    assert numpy.array_equal(p, ref[1]) and numpy.array_equal(depth, ref[0])
    s.findOverlaps()
    rp, rd = O.overlaps(s)
    assert numpy.array_equal(s.pairs.T, rp.astype(numpy.int32))
    assert numpy.array_equal(s.overlaps, rd)
    s.findCoordinationNumber()
    assert s.coordinationnumber.sum() == 2 * len(rd)
    s.findContactStresses()
    assert numpy.all(s.sigma_contacts > 0.0)
    loaded = s.findLoadedContacts(numpy.median(s.sigma_contacts))
    assert 0 < len(loaded[0]) <= len(rd)
