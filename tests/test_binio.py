"""The .bin v2.15 format against golden files written by the reference's own
python/sphere.py (tests/golden/bin_*.bin, see tests/golden/make_golden.py):
the same seeded scenes built with sphere_b200.sim must encode to the same
bytes, and every golden file must read back and re-encode unchanged.  The
darcy scene carries the Darcy fluid block (cfd_solver 1), the ns scene the
Navier-Stokes fluid block (cfd_solver 0: read and written, not stepped)."""
import os

import numpy
import pytest

import oracle as O
from sphere_b200 import binio
from sphere_b200.sim import sim

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _scenes():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.bin_scenes(sim)


@pytest.mark.parametrize("name", ["grid", "consolidate", "shear", "bonds", "darcy", "ns"])
def test_setup_and_writer_match_reference_bytes(name):
    ours = _scenes()[name]
    golden = open(os.path.join(GOLDEN, "bin_%s.bin" % name), "rb").read()
    assert binio.encode_bin(ours) == golden


@pytest.mark.parametrize("name", ["grid", "consolidate", "shear", "bonds", "darcy", "ns"])
def test_reader_round_trip(name, tmp_path):
    path = os.path.join(GOLDEN, "bin_%s.bin" % name)
    # as in the reference, the sim says whether the file has a fluid block
    s = sim(fluid=(name in ("darcy", "ns")))
    s.readbin(path, verbose=False)
    if name in ("darcy", "ns"):
        # the reader divides dphi by time_dt * ndem with the ndem the sim
        # held before the read (1), the writer multiplies by the file's (3),
        # as the reference's own reader and writer do: every other byte
        # round-trips, and dphi does with the scale the writer applies
        s.dphi = s.dphi / s.ndem
    assert binio.encode_bin(s) == open(path, "rb").read()
    s.writebin(folder=str(tmp_path), verbose=False)
    assert open(os.path.join(str(tmp_path), s.sid + ".bin"), "rb").read() == open(path, "rb").read()


def test_truncated_file_is_an_error(tmp_path):
    data = open(os.path.join(GOLDEN, "bin_grid.bin"), "rb").read()
    p = tmp_path / "t.bin"
    p.write_bytes(data[:len(data) // 2])
    with pytest.raises(ValueError, match="truncated"):
        sim().readbin(str(p), verbose=False)


@pytest.mark.skipif(O.reference_root() is None,
                    reason="reference fixtures not present")
@pytest.mark.parametrize("fname,n", [("cube-init.output00029.bin", 1000),
                                     ("init-1e4.output00199.bin", 10000)])
def test_reads_reference_output_files(fname, n):
    s = sim()
    s.readbin(os.path.join(O.reference_root(), "output", fname), verbose=False)
    assert int(s.np[0]) == n
    assert s.x.shape == (n, 3) and (s.radius > 0).all()
    assert numpy.isfinite(s.x).all()
    assert s.version[0] == binio.VERSION


def test_darcy_reader_scales_dphi_and_fields(tmp_path):
    """The fluid fields of the Darcy golden scene read back in the sim's
    [x, y, z] layout, dphi divided by time_dt * ndem as the reference's
    reader divides (with the ndem the sim held before the read)."""
    ours = _scenes()["darcy"]
    s = sim(fluid=True)
    s.readbin(os.path.join(GOLDEN, "bin_darcy.bin"), verbose=False)
    assert numpy.array_equal(s.p_f, ours.p_f) and numpy.array_equal(s.v_f, ours.v_f)
    assert numpy.array_equal(s.p_f_constant, ours.p_f_constant)
    raw = ours.dphi * ours.time_dt * ours.ndem
    assert numpy.array_equal(s.dphi, raw / (s.time_dt * 1))
    assert int(numpy.ravel(s.ndem)[0]) == 3 and int(numpy.ravel(s.maxiter)[0]) == 500
    assert int(s.bc_bot[0]) == 1
    assert numpy.array_equal(s.f_p, ours.f_p)


def test_navier_stokes_fields_read_back():
    """The Navier-Stokes block's solver parameters and per-sphere fluid
    forces, as the reference's writer stored them."""
    ours = _scenes()["ns"]
    s = sim(fluid=True)
    s.readbin(os.path.join(GOLDEN, "bin_ns.bin"), verbose=False)
    assert int(s.cfd_solver[0]) == 0 and not hasattr(s, "bc_xn")
    for name in ("gamma", "theta", "beta", "tolerance", "c_phi", "c_v", "dt_dem_fac"):
        assert float(numpy.ravel(getattr(s, name))[0]) == float(numpy.ravel(getattr(ours, name))[0]), name
    assert int(numpy.ravel(s.maxiter)[0]) == 800 and int(numpy.ravel(s.ndem)[0]) == 2
    for name in ("f_d", "f_p", "f_v", "f_sum"):
        assert numpy.array_equal(getattr(s, name), getattr(ours, name)), name
    assert numpy.array_equal(s.p_f, ours.p_f) and numpy.array_equal(s.v_f, ours.v_f)


def test_navier_stokes_fluid_is_not_stepped(tmp_path):
    """The Navier-Stokes solver is not built: run() refuses such a sim
    before it touches a device."""
    from sphere_b200 import runner
    s = _scenes()["ns"]
    with pytest.raises(NotImplementedError):
        runner.run_sim(s, root=str(tmp_path), verbose=False)