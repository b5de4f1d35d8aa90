"""Ensemble sharding on the GPU path (world size 1 here; the multi-rank
host logic is covered by the gloo test): boxes made in a subset equal the
same boxes made with the whole ensemble, and run_rank with the real GPU
stepper as its engine gives the per-box summaries of stepping every box in
one handle."""
import copy
import os
import socket

import numpy
import pytest
import torch.distributed as dist

from sphere_b200 import ensemble, scenes
from sphere_b200.runner import Stepper

pytestmark = pytest.mark.gpu

KW = dict(nboxes=8, seed=4, device=0, counts=(200, 2000), sweeps=300)


def test_subset_boxes_equal_the_whole_ensembles():
    whole = scenes.shear_ensemble(**KW)
    part = scenes.shear_ensemble(subset=[6, 1, 3], **KW)
    for b, s in zip([6, 1, 3], part):
        w = whole[b]
        assert s.sid == w.sid
        assert numpy.array_equal(s.x, w.x) and numpy.array_equal(s.radius, w.radius)
        assert float(s.w_sigma0[0]) == float(w.w_sigma0[0]) and float(s.mu_s[0]) == float(w.mu_s[0])
    assert [int(s.np[0]) for s in whole] == scenes.ensemble_counts(8, seed=4, counts=(200, 2000))


def _gpu_steps(precision):
    def run(sims, steps):
        st = Stepper(copy.deepcopy(sims), precision=precision, device=0)
        st.upload()
        st.step(steps)
        out = st.to_sims()
        st.close()
        return out
    return run


def test_run_rank_with_the_gpu_stepper():
    sims = scenes.shear_ensemble(**KW)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1)
    try:
        got = ensemble.run_rank(sims, 20, 0, 1, _gpu_steps("fp64"))
    finally:
        dist.destroy_process_group()
    want = [ensemble.summary(q) for q in _gpu_steps("fp64")(sims, 20)]
    assert got == want
