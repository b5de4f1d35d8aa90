"""The packing sweeps of scene preparation (sph_relax: cell sort, then per
sphere the pushes of every overlapping neighbour in the 27 cells, walls and
floor, then the Jacobi move) against their C restatement (oracle.relax,
or_relax in oracle/sphere_oracle.c), bit for bit: every benchmark pack is
made by this chain, so a change in it would change the measured workloads.
Cases: a 2,000-sphere log-normal FCC start in an x-y periodic box (the dense
pack's construction), a loose random start with walls on every side, and
three boxes relaxed in one handle (as the ensemble is made) against each
box relaxed alone by the oracle."""
import math

import numpy
import pytest

import oracle as O
from sphere_b200 import scenes
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu


def _fcc(n, seed):
    rng = numpy.random.default_rng(seed)
    r = numpy.clip(numpy.exp(rng.normal(math.log(0.01), 0.2, n)), 0.005, 0.02)
    s, H = scenes._fcc_start(n, rng, r, 0.40, 0.5, 0.01, "relax")
    return s, H


def _gpu_chunks(sims, chunks, alpha, z_top):
    st = Stepper(sims)
    st.upload()
    out = []
    for k in chunks:
        worst = st.relax(k, alpha=alpha, z_top=z_top)
        hp, _ = st.download()
        out.append((hp.x[:, :3].copy(), worst))
    st.close()
    return out


@pytest.mark.parametrize("alpha", [0.6, 1.0])
def test_relax_dense_start_matches_oracle(alpha):
    s, H = _fcc(2000, 3)
    chunks = (1, 24, 275)
    g = _gpu_chunks([s], chunks, alpha, H)
    for k, (xg, wg) in zip(chunks, g):
        wc = O.relax(s, k, alpha=alpha, z_top=H)
        assert numpy.array_equal(xg, s.x), "positions differ after a chunk of %d sweeps" % k
        assert wg == wc
    assert g[-1][1] < g[0][1]   # the overlaps shrink


def test_relax_walled_box_matches_oracle():
    from sphere_b200.sim import sim
    n = 1500
    rng = numpy.random.default_rng(4)
    s = sim(np=n, nw=0, sid="walled")
    s.radius[:] = rng.uniform(0.009, 0.011, n)
    side = (float(numpy.sum(4.0 / 3.0 * math.pi * s.radius ** 3)) / 0.55) ** (1.0 / 3.0)
    s.x[:] = rng.uniform(0.0, side * 0.999, (n, 3))
    s.periodic[0] = 0
    s.defineWorldBoundaries(L=[side, side, side])
    s.time_dt[0] = 1e-7
    s.time_total[0] = 1.0
    chunks = (1, 40)
    g = _gpu_chunks([s], chunks, 1.0, side)
    for k, (xg, wg) in zip(chunks, g):
        wc = O.relax(s, k, alpha=1.0, z_top=side)
        assert numpy.array_equal(xg, s.x)
        assert wg == wc


def test_relax_boxes_in_one_handle_match_each_box_alone():
    sims = [_fcc(n, 10 + k)[0] for k, n in enumerate((700, 1200, 300))]
    g = _gpu_chunks(sims, (60,), 0.6, 1e300)
    x = g[0][0]
    o = 0
    for s in sims:
        n = int(s.np[0])
        O.relax(s, 60, alpha=0.6, z_top=1e300)
        assert numpy.array_equal(x[o:o + n], s.x)
        o += n
