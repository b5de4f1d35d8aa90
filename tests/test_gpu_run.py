"""The drop-in surface on the GPU: the reference's known-answer scenarios
(tests/physics_cases.py) run exactly as the reference's tests drive them --
sim.run() writes <root>/input/<sid>.bin and the output files, readlast()
reads the last output -- plus output-file parity with the oracle."""
import copy
import os

import numpy
import pytest

import oracle as O
import physics_cases as P
import sphere_b200 as simmod
from sphere_b200 import binio

pytestmark = pytest.mark.gpu

NAMES = sorted(P.scenarios().keys())


@pytest.mark.parametrize("young", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_run_known_answers(name, young, tmp_path):
    s, check = P.scenarios(young)[name]
    root = str(tmp_path)
    assert s.run(verbose=False, root=root) == 0
    after = simmod.sim(np=int(s.np[0]), sid=s.sid)
    after.readlast(verbose=False, root=root)
    check(s, after)


def test_run_writes_reference_files_and_matches_oracle(tmp_path):
    s, _ = P.scenarios(False)["oblique_slip"]
    s.time_total[0] = 0.02
    s.time_file_dt[0] = 0.005
    root = str(tmp_path)
    x0 = s.x.copy()
    assert s.run(verbose=False, root=root) == 0
    assert numpy.array_equal(s.x, x0), "run() must not change the caller's object"
    last = simmod.status(s.sid, root=root)
    # the reference's output cadence (src/device.cu:1031, 2536-2537, 2569,
    # 2672): step while time <= total, write when the file clock reaches
    # file_dt, then restart the file clock at zero
    dt, cur, ftc, files, steps, at_last_file = float(s.time_dt[0]), float(s.time_current[0]), \
        0.0, 0, 0, 0
    while cur <= 0.02:
        cur += dt
        ftc += dt
        steps += 1
        if ftc >= 0.005:
            files += 1
            ftc = 0.0
            at_last_file = steps
    assert last == files
    for k in range(last + 1):
        assert os.path.exists(os.path.join(root, "output", "%s.output%05d.bin" % (s.sid, k)))
    # output 0 is the input state; the input file is the writebin of the sim
    first = simmod.sim(sid=s.sid)
    first.readfirst(verbose=False, root=root)
    assert open(os.path.join(root, "input", s.sid + ".bin"), "rb").read() == binio.encode_bin(first)
    # the last output equals the oracle stepped to the step of that output
    after = simmod.sim(sid=s.sid)
    after.readlast(verbose=False, root=root)
    run = O.CpuRun(s, "oracle")
    run.step(at_last_file)
    ref = run.to_sim(copy.deepcopy(s))
    for name in ("x", "vel", "angvel", "angpos", "force", "torque", "es", "ev", "xyzsum"):
        assert numpy.array_equal(getattr(after, name), getattr(ref, name)), name
    assert after.time_current[0] == ref.time_current[0]


def test_dry_run_reports(tmp_path, capsys):
    s, _ = P.scenarios(False)["elastic_equal"]
    assert s.run(dry=True, root=str(tmp_path)) == 0
    out = capsys.readouterr().out
    assert "Number of particles:  np = 2" in out


def test_run_rejects_bad_input(tmp_path, capsys):
    s, _ = P.scenarios(False)["elastic_equal"]
    s.x[0, 0] = 11.0      # outside the 10 m grid
    assert s.run(verbose=False, root=str(tmp_path)) == 1
    assert "outside" in capsys.readouterr().out
