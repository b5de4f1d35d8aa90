"""The C-ABI library: it loads, exports every entry point declared in
include/sphere_b200.h, and its struct layouts match the ctypes mirror.
No compute calls (these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

from sphere_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sphere_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("sph_create", "sph_upload", "sph_step", "sph_advance", "sph_download",
                 "sph_get_contacts", "sph_get_sort", "sph_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_sizes_match_ctypes():
    lib = _abi.load_library()
    sizes = (C.c_uint64 * 6)()
    assert lib.sph_struct_sizes(sizes) == 0
    mirror = [_abi.SphParams, _abi.SphGrid, _abi.SphWalls, _abi.SphBox, _abi.SphParticles,
              _abi.SphBonds]
    assert list(sizes) == [C.sizeof(t) for t in mirror]


def test_status_strings_and_null_handle():
    lib = _abi.load_library()
    for code in range(9):
        assert lib.sph_status_string(code)
    assert lib.sph_step(None, 1) == _abi.SPH_ERR_INPUT
    assert lib.sph_download(None, None, None) == _abi.SPH_ERR_INPUT
    buf = C.create_string_buffer(64)
    assert lib.sph_last_error(None, buf, 64) > 0
    lib.sph_destroy(None)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_abi, "_LIB", None)
    monkeypatch.setattr(_abi, "lib_path", lambda: str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError, match="missing"):
        _abi.load_library()


def test_header_constants_match_the_mirror():
    text = open(os.path.join(ROOT, "include", "sphere_b200.h")).read()
    defs = dict(re.findall(r"#define\s+(SPH_[A-Z_]+)\s+(\d+)", text))
    assert int(defs["SPH_TUNE_VARIANTS"]) == _abi.TUNE_VARIANTS
    assert int(defs["SPH_PAIR_SHAPES"]) == _abi.PAIR_SHAPES


def test_darcy_struct_size_matches_ctypes():
    lib = _abi.load_library()
    n = C.c_uint64(0)
    assert lib.sph_darcy_struct_size(C.byref(n)) == 0
    assert n.value == C.sizeof(_abi.SphDarcy)
