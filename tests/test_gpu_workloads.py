"""The other measured workloads at parity-test sizes, against the oracle bit
for bit: the bonded pack (bonds between touching pairs, more bonds than
spheres, Young's-modulus contacts, a top wall moving at constant velocity)
in both launch variants, stepped in one run (the overlapped wall stage) and
step by step."""
import pytest

import oracle as O
from sphere_b200 import scenes
from sphere_b200.runner import Stepper
from test_gpu_parity import check_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bonded():
    return scenes.bonded_pack(n=20000, nbonds=30000, seed=3, device=0, sweeps=1500)


@pytest.mark.parametrize("variant", [1, 3])
def test_bonded_pack_matches_oracle(bonded, variant):
    s = bonded
    assert int(s.nb0[0]) > int(s.np[0])
    st = Stepper([s], precision="fp64", length="reference")
    st.upload()
    st.set_variant(variant)
    cpu = O.CpuRun(s, "oracle")
    st.step(1)
    cpu.step(1)
    check_same(st, cpu, s)
    st.step(9)
    cpu.step(9)
    check_same(st, cpu, s)
    st.close()
