"""The .bin v2.15 format against golden files written by the reference's own
python/sphere.py (tests/golden/bin_*.bin, see tests/golden/make_golden.py):
the same seeded scenes built with sphere_b200.sim must encode to the same
bytes, and every golden file must read back and re-encode unchanged."""
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


@pytest.mark.parametrize("name", ["grid", "consolidate", "shear", "bonds"])
def test_setup_and_writer_match_reference_bytes(name):
    ours = _scenes()[name]
    golden = open(os.path.join(GOLDEN, "bin_%s.bin" % name), "rb").read()
    assert binio.encode_bin(ours) == golden


@pytest.mark.parametrize("name", ["grid", "consolidate", "shear", "bonds"])
def test_reader_round_trip(name, tmp_path):
    path = os.path.join(GOLDEN, "bin_%s.bin" % name)
    s = sim()
    s.readbin(path, verbose=False)
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
