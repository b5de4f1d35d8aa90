"""The reference's known-answer tests (momentum transfer, energy balances,
spin signs; see tests/physics_cases.py) run through the CPU oracle, with
linear and Young's-modulus stiffness.  This pins the oracle to the
reference's own tests; tests/test_gpu_run.py runs the same scenarios
through sim.run() on the GPU."""
import copy

import pytest

import oracle as O
import physics_cases as P

NAMES = sorted(P.scenarios().keys())


@pytest.mark.parametrize("young", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_oracle_known_answers(name, young):
    s, check = P.scenarios(young)[name]
    run = O.CpuRun(s, "oracle")
    run.step(P.n_steps(s))
    after = run.to_sim(copy.deepcopy(s))
    check(s, after)
