"""The bounded grid barrier of the persistent list step (sph_barrier_check):
barriers among resident blocks open; a barrier that waits for more blocks
than were launched -- an arrival that never comes -- gives up after its time
limit with SPH_ERR_TIMEOUT, and the device stays usable."""
import time

import numpy
import pytest

import cases
from sphere_b200 import _abi
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

OK, INPUT, TIMEOUT = 0, 1, 9


def test_barriers_open_among_resident_blocks():
    lib = _abi.load_library()
    for blocks in (1, 7, 64):
        assert lib.sph_barrier_check(blocks, blocks, 200, 1.0) == OK


def test_a_barrier_missing_an_arrival_times_out_and_the_device_stays_usable():
    lib = _abi.load_library()
    t0 = time.perf_counter()
    rc = lib.sph_barrier_check(8, 9, 1, 0.25)
    dt = time.perf_counter() - t0
    assert rc == TIMEOUT
    assert 0.2 < dt < 10.0
    # the context is still good: a step runs and gives results
    s = cases.make("periodic_xy_wall_stress")[0]
    st = Stepper([s], precision="mixed")
    st.set_variant(4)
    st.upload()
    st.step(3)
    hp, _ = st.download()
    assert numpy.isfinite(hp.x).all()
    st.close()


def test_barrier_check_refuses_bad_arguments():
    lib = _abi.load_library()
    assert lib.sph_barrier_check(0, 1, 1, 1.0) == INPUT
    assert lib.sph_barrier_check(100000, 100000, 1, 1.0) == INPUT
    assert lib.sph_barrier_check(4, 4, 1, 0.0) == INPUT
    assert lib.sph_barrier_check(4, 4, 1, 100.0) == INPUT
