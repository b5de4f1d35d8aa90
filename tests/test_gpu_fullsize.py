"""Parity at the measured size: the 1e6-sphere sheared dense pack of the
benchmark (log-normal radii, porosity 0.40, x-y periodic, top wall at
20 kPa, top layer sheared).

* five FP64 steps on the GPU against the C oracle (OpenMP), bit for bit,
  in every field the small parity cases check (after steps 1 and 5);
* the fused interact kernel and the split step, 30 steps each from the same
  state, bit for bit;
* the FP32-mixed form's per-step force error against FP64 at this size
  (one step from the same state), within the 1e-5 relative L2 of the
  precision contract.
"""
import numpy
import pytest

import oracle as O
from sphere_b200 import scenes
from sphere_b200.runner import Stepper
from test_gpu_parity import check_same

pytestmark = pytest.mark.gpu

N = 1_000_000


@pytest.fixture(scope="module")
def pack():
    return scenes.sheared_dense_pack(n=N, seed=0, device=0, sweeps=3000)


def test_full_size_steps_match_oracle(pack):
    s = pack
    st = Stepper([s], precision="fp64", length="reference")
    st.upload()
    cpu = O.CpuRun(s, "oracle")
    for k in (1, 4):
        st.step(k)
        cpu.step(k)
        check_same(st, cpu, s)
    assert int((cpu.contacts != N).sum()) > 3 * N   # a dense pack: 4.4 contacts per sphere
    st.close()


def _state(st):
    hp, _ = st.download()
    c, dt, _ = st.contacts()
    return hp, c, dt


def test_full_size_fused_and_split_agree(pack):
    out = []
    for variant in (1, 3):
        st = Stepper([pack], precision="fp64", length="reference")
        st.upload()
        st.set_variant(variant)
        st.step(30)
        out.append(_state(st))
        st.close()
    (a, ca, ta), (b, cb, tb) = out
    for name in ("x", "vel", "angvel", "angpos", "xyzsum", "force", "torque", "es", "ev", "p"):
        assert numpy.array_equal(getattr(a, name), getattr(b, name)), name
    assert numpy.array_equal(ca, cb) and numpy.array_equal(ta, tb)


def test_full_size_mixed_force_error(pack):
    """One step from the same state in each form (trajectories of a dense
    pack diverge over many steps in any precision, so the contract is per
    step)."""
    res = []
    for prec in ("fp64", "mixed"):
        st = Stepper([pack], precision=prec, length="reference")
        st.upload()
        st.set_variant(3)
        st.step(1)
        hp, _ = st.download()
        res.append((hp, st.contacts()[0]))
        st.close()
    (a, ca), (b, cb) = res
    rel = numpy.linalg.norm(b.force - a.force) / numpy.linalg.norm(a.force)
    assert rel < 1e-5, rel
    assert numpy.array_equal(ca, cb)   # the same contacts in both forms
