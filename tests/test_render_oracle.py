"""The oracle's ray tracer (or_render, a restatement of src/raytracer.cuh)
pinned pixel for pixel to the reference's own ray-tracer kernels and camera
compiled for the CPU (oracle/_ref/sphere_render_ref, where the reference
sources are present) and to golden images made by that program
(tests/golden/render_*.npz, tests/golden/make_render_golden.py); against a
second, independent restatement in numpy float32 arithmetic (one IEEE
operation per ufunc call, so no contraction); known answers for the camera
and the colours; the PPM and PNG writers."""
import importlib
import os
import struct
import sys
import zlib

import numpy
import pytest

import cases
import oracle as O
from sphere_b200 import sim as simmod
from sphere_b200 import scenes

f32 = numpy.float32
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _scale(s, a):
    return (s * a[0], s * a[1], s * a[2])


def _camera(s, width, height):
    """cameraInit (src/raytracer.cuh:291-333) as render() calls it (:399-419)."""
    L = [float(v) for v in s.L]
    mx = [max(0.0, float(numpy.max(s.x[:, a]))) for a in range(3)]
    imgw = f32(L[0] * float(f32(1.35)))
    lookat = tuple(f32(m) / f32(2.0) for m in mx)
    eye = (f32(L[0] * float(f32(2.3))), f32(L[1] * float(f32(-5.0))), f32(L[2] * float(f32(1.3))))
    hw = f32(height // width)
    plane = (f32(-0.5) * imgw, f32(0.5) * imgw, f32(-0.5) * imgw * hw, f32(0.5) * imgw * hw)
    view = tuple(e - l for e, l in zip(eye, lookat))
    up = (f32(0), f32(0), f32(1))
    lv = numpy.sqrt(_dot(view, view))
    w = tuple(-c / lv for c in view)
    cw = _cross(up, w)
    lcw = numpy.sqrt(_dot(cw, cw))
    u = tuple(c / lcw for c in cw)
    v = _cross(w, u)
    d = lv * f32(0.8)
    le = _scale(f32(-1.0), eye)
    lt = (le[0] * f32(1.0), le[1] * f32(0.2), le[2] * f32(0.6))
    light = _scale(f32(1.0) / numpy.sqrt(_dot(lt, lt)), lt)
    return eye, plane, u, v, w, d, light


_values = cases.render_values


def _render_numpy(s, method, maxval, cutoff, width, height):
    """Every pixel against every sphere, vectorised over (pixel, sphere)."""
    eye, (pl, pr, pb, pt), u, v, w, dfoc, light = _camera(s, width, height)
    mem = numpy.arange(width * height, dtype=numpy.uint32)
    i = mem % numpy.uint32(width)
    j = (numpy.floor(mem.astype(f32) / f32(width)).astype(numpy.int64) % width).astype(f32)
    pu = pl + (pr - pl) * (i.astype(f32) + f32(0.5)) / f32(width)
    pv = pb + (pt - pb) * (j + f32(0.5)) / f32(height)
    d = [(f32(-dfoc) * w[a] + pu * u[a]) + pv * v[a] for a in range(3)]
    c = [s.x[:, a].astype(f32) for a in range(3)]
    R = s.radius.astype(f32)
    ec = [eye[a] - c[a][None, :] for a in range(3)]
    D = [da[:, None] for da in d]
    dec = _dot(D, ec)
    dd = _dot(D, D)
    ecec = _dot(ec, ec)
    Delta = (f32(2.0) * dec) * (f32(2.0) * dec) - f32(4.0) * dd * (ecec - R * R)
    with numpy.errstate(invalid="ignore"):
        ndec = _dot([-x for x in D], ec)
        t = (ndec - numpy.sqrt(dec * dec - dd * (ecec - R * R))) / dd
        at = numpy.abs(t)
        take = (Delta > f32(0.0)) & (at < f32(1e10))
    if method != 0 and cutoff > 0.0:
        val = _values(s, method).astype(f32)
        fix = s.fixvel.astype(f32)
        take &= ((val > f32(cutoff)) & (fix == f32(0.0)))[None, :]
    at = numpy.where(take, at, numpy.inf)
    hit = numpy.argmin(at, axis=1)
    anyhit = numpy.isfinite(at[numpy.arange(len(mem)), hit])
    img = numpy.full((width * height, 3), 255, dtype=numpy.uint8)
    for m in numpy.nonzero(anyhit)[0]:
        k = hit[m]
        tm = t[m, k]
        p = [eye[a] + tm * d[a][m] for a in range(3)]
        n2 = [f32(2.0) * (p[a] - c[a][k]) for a in range(3)]
        n = _scale(f32(1.0) / numpy.sqrt(_dot(n2, n2)), n2)
        dot = max(f32(0.0), _dot(n, light))
        shade = f32(5.0) * f32(40.0) * dot + f32(10.0) * f32(5.0)
        if method == 0:
            cols = (f32(0.48), f32(0.41), f32(0.27))
        else:
            ratio = f32(_values(s, method)[k] / float(f32(maxval)))
            ratio = min(max(ratio, f32(0.01)), f32(0.99))
            r = ratio
            cols = (min(f32(1.0), f32(0.209) * r * r * r - f32(2.49) * r * r + f32(3.0) * r + f32(0.0109)),
                    min(f32(1.0), f32(-2.44) * r * r + f32(2.15) * r + f32(0.369)),
                    min(f32(1.0), f32(-2.21) * r * r + f32(1.61) * r + f32(0.573)))
            if f32(s.fixvel[k]) > f32(0.0):
                cols = (f32(0.5),) * 3
        img[m] = [numpy.uint8(int(shade * cc)) for cc in cols]
    return img.reshape(height, width, 3)


def _scene(name):
    return cases.render_scene(name)


def _golden(name):
    g = numpy.load(os.path.join(GOLDEN, "render_%s.npz" % name))
    import make_render_golden
    s = _scene(name)
    assert str(g["digest"]) == make_render_golden.scene_digest(s), "scene drifted"
    return s, g


@pytest.mark.parametrize("name", cases.RENDER_SCENES)
def test_oracle_matches_golden_images(name):
    s, g = _golden(name)
    for k, (method, maxval, cut, w, h) in enumerate(g["runs"]):
        img = O.render(s, int(method), maxval, cut, int(w), int(h))
        assert numpy.array_equal(img, g["img_%d" % k]), (name, k)
        assert (img != 255).any()


@pytest.mark.parametrize("name", cases.RENDER_SCENES + ["periodic_xy_wall_stress"])
def test_oracle_matches_reference_program(name):
    s = _scene(name)
    if O.reference_render(s, 0, 1e3, 0.0, 8, 8) is None:
        pytest.skip("the reference ray-tracer program is not built here")
    for method, maxval, cut, w, h in cases.render_runs(s):
        ref = O.reference_render(s, method, maxval, cut, w, h)
        assert numpy.array_equal(O.render(s, method, maxval, cut, w, h), ref), (method, w, h)
    ref = O.reference_render(s, 1, 1.5e3, 0.0, 800, 800)   # DEM::render's default size
    assert numpy.array_equal(O.render(s, 1, 1.5e3, 0.0, 800, 800), ref)


@pytest.mark.parametrize("method", [0, 1, 2, 3, 4, 5])
def test_oracle_render_matches_numpy_restatement(method):
    s = _scene("fixvel_modes")
    vals = _values(s, method) if method else numpy.zeros(1)
    maxval = float(numpy.quantile(vals, 0.9)) if method else 1e3
    for cutoff, (w, h) in ((0.0, (40, 40)), (float(numpy.median(vals)) if method else 0.0, (36, 24)),
                           (0.0, (20, 44))):
        ref = _render_numpy(s, method, maxval, cutoff, w, h)
        got = O.render(s, method, maxval, cutoff, w, h)
        assert numpy.array_equal(got, ref), (method, cutoff, w, h)
        assert (got != 255).any()


def test_render_known_answers():
    s = simmod(np=1, nw=0, sid="one")
    s.radius[:] = 0.25
    s.x[0] = [1.0, 1.0, 1.0]
    s.defineWorldBoundaries([2.0, 2.0, 2.0])
    img = O.render(s, 0, 1e3, 0.0, 64, 64)
    # background where no sphere is hit (imageInit)
    assert (img[0, 0] == 255).all() and (img[-1, -1] == 255).all()
    hit = (img != 255).any(axis=2)
    assert 0 < hit.sum() < 64 * 64
    # uniform colour in the proportions 0.48 : 0.41 : 0.27 of the shade
    px = img[hit]
    assert (px[:, 0] >= px[:, 1]).all() and (px[:, 1] >= px[:, 2]).all()
    assert px[:, 0].max() <= int(250 * 0.48) and px[:, 0].min() >= int(50 * 0.48)
    # the ambient floor: 50 * 0.48 = 24 on the side away from the light
    assert px[:, 0].min() == 24
    # hw_ratio = height / width in integers: a wide image has a flat plane
    # (every row the same ray set)
    flat = O.render(s, 0, 1e3, 0.0, 32, 16)
    assert (flat == flat[:1]).all()


def test_render_cutoff_hides_spheres():
    s = _scene("walls_all_sides")
    full = O.render(s, 1, 2e3, 0.0, 48, 48)
    hidden = O.render(s, 1, 2e3, 5e3, 48, 48)     # above every pressure
    assert (full != 255).any() and (hidden == 255).all()
    s.fixvel[:] = 1.0
    grey = O.render(s, 1, 2e3, 0.0, 48, 48)
    px = grey[(grey != 255).any(axis=2)]
    assert (px[:, 0] == px[:, 1]).all() and (px[:, 1] == px[:, 2]).all()


def test_ppm_and_png_writers(tmp_path):
    rng = numpy.random.default_rng(0)
    img = rng.integers(0, 256, (7, 5, 3), dtype=numpy.uint8)
    p = os.path.join(tmp_path, "a.ppm")
    simmod_mod = importlib.import_module("sphere_b200.sim")
    simmod_mod.write_ppm(p, img)
    with open(p, "rb") as fh:
        assert fh.read(11) == b"P6 5 7 255\n"
    assert numpy.array_equal(simmod_mod.read_ppm(p), img)
    simmod_mod.convert("png", folder=str(tmp_path))
    assert not os.path.exists(p)
    with open(os.path.join(tmp_path, "a.png"), "rb") as fh:
        data = fh.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(kind + body)
        if kind == b"IHDR":
            assert struct.unpack(">IIBBBBB", body) == (5, 7, 8, 2, 0, 0, 0)
        if kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = numpy.frombuffer(zlib.decompress(idat), dtype=numpy.uint8).reshape(7, 1 + 15)
    assert (raw[:, 0] == 0).all()
    assert numpy.array_equal(raw[:, 1:].reshape(7, 5, 3), img)


def test_render_method_names():
    s = scenes.lattice_pack(8, seed=0)
    with pytest.raises(ValueError):
        s.renderImage(method="temperature")
