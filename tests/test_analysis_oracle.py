"""The oracle's restatement of the reference's analysis code
(src/sphere.cpp: DEM::porosity, DEM::findOverlaps) against that code itself,
compiled for the CPU from the reference sources (oracle/_ref/
sphere_analysis_ref, printing 17 significant digits), on the parity scenes.
Scenes with more bonds than spheres are left out: the reference's readbin
sizes its bond-history arrays by the sphere count (src/file_io.cpp:234-235)
and overruns them."""
import numpy
import pytest

import cases
import oracle as O

NAMES = ["walls_all_sides", "periodic_xy_wall_stress", "fixvel_modes", "youngs_modulus"]


def _need_ref():
    s, _, _ = cases.make("walls_all_sides")
    if O.reference_analysis(s, "contacts") is None:
        pytest.skip("the reference analysis program is not built here")


@pytest.mark.parametrize("name", NAMES)
def test_porosity_restatement_matches_reference(name):
    _need_ref()
    s, _, _ = cases.make(name)
    for slices in (2, 4):
        z_r, p_r = O.reference_analysis(s, "porosity", slices)
        z_o, p_o = O.porosity(s, slices)
        assert numpy.array_equal(z_r, z_o) and numpy.array_equal(p_r, p_o)


@pytest.mark.parametrize("name", NAMES)
def test_overlaps_restatement_matches_reference(name):
    _need_ref()
    s, _, _ = cases.make(name)
    pr, dr = O.reference_analysis(s, "contacts")
    po, do = O.overlaps(s)
    assert len(po) > 0
    assert numpy.array_equal(pr, po) and numpy.array_equal(dr, do)


def test_porosity_rejects_thin_slabs():
    s, _, _ = cases.make("walls_all_sides")
    assert O.porosity(s, 1000) is None
