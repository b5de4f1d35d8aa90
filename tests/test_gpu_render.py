"""sph_render (Stepper.render, sim.renderImage, sphere_b200.render) against
the oracle's restatement of the reference's ray tracer (every sphere tested
for every pixel), byte for byte: the parity scenes after some steps with
every colour method, cutoffs and image shapes (square, wide with the flat
image plane of hw_ratio = 0, tall with the row index wrapped modulo the
width); the golden images of the reference's own kernels; spheres of
about a pixel; the file path of `sphere --render`."""
import os

import numpy
import pytest

import cases
import oracle as O
import sphere_b200
from sphere_b200 import scenes
from sphere_b200.runner import SphereError, Stepper
from test_render_oracle import _golden

_values = cases.render_values

pytestmark = pytest.mark.gpu

NAMES = ["walls_all_sides", "periodic_xy_wall_stress", "fixvel_modes", "fast_spheres"]
SHAPES = [(96, 96), (80, 48), (48, 100)]


def _maxval(s, method):
    if method == 0:
        return 1e3
    m = float(numpy.quantile(_values(s, method), 0.9))
    return m if m > 0.0 else 1.0


@pytest.mark.parametrize("name", NAMES)
def test_render_matches_oracle(name):
    s, _, steps = cases.make(name)
    st = Stepper([s], precision="fp64")
    st.upload()
    st.step(steps)
    st.to_sims()
    for method in range(6):
        maxval = _maxval(s, method)
        cut = float(numpy.median(_values(s, method))) if method else 0.0
        for cutoff, (w, h) in zip((0.0, cut, 0.0), SHAPES):
            got = st.render(method=method, maxval=maxval, lower_cutoff=cutoff, width=w, height=h)
            ref = O.render(s, method, maxval, cutoff, w, h)
            assert numpy.array_equal(got, ref), (name, method, cutoff, w, h)
            assert (got != 255).any()
    st.close()


def test_render_pixel_sized_spheres():
    s = scenes.lattice_pack(27000, seed=21, periodic=1, nw=0)
    rng = numpy.random.default_rng(21)
    s.p[:] = rng.uniform(0.0, 1.0, len(s.radius))
    st = Stepper([s], precision="fp64")
    st.upload()
    for method, (w, h) in ((0, (128, 128)), (1, (200, 120))):
        got = st.render(method=method, maxval=0.8, width=w, height=h)
        ref = O.render(s, method, 0.8, 0.0, w, h)
        assert numpy.array_equal(got, ref), (method, w, h)
    st.close()


def test_render_default_image_size():
    s, _, _ = cases.make("walls_all_sides")
    img = s.renderImage(method="normal")
    assert img.shape == (800, 800, 3)
    assert numpy.array_equal(img, O.render(s, 0, 1e3, 0.0, 800, 800))


@pytest.mark.parametrize("name", cases.RENDER_SCENES)
def test_render_matches_golden_images(name):
    """Against the images of the reference's own kernels run on the CPU."""
    s, g = _golden(name)
    st = Stepper([s], precision="fp64")
    st.upload()
    for k, (method, maxval, cut, w, h) in enumerate(g["runs"]):
        img = st.render(method=int(method), maxval=maxval, lower_cutoff=cut, width=int(w),
                        height=int(h))
        assert numpy.array_equal(img, g["img_%d" % k]), (name, k)
    st.close()


def test_render_refuses_bad_arguments():
    s, _, _ = cases.make("walls_all_sides")
    st = Stepper([s], precision="fp64")
    st.upload()
    with pytest.raises(SphereError):
        st.render(method=6)
    with pytest.raises(SphereError):
        st.render(width=0)
    with pytest.raises(SphereError):
        st.render(box=1)
    st.close()


def test_render_files(tmp_path):
    """sphere_b200.render(binary) writes img_out/<name>.ppm as `sphere
    --render` does; sim.render renders every output file of the sid."""
    root = str(tmp_path)
    s, _, _ = cases.make("fixvel_modes")
    rng = numpy.random.default_rng(3)
    s.p[:] = rng.uniform(0.0, 2e3, len(s.radius))
    s.sid = "rt"
    os.makedirs(os.path.join(root, "output"))
    for k in range(2):
        s.x[:, 2] += 0.001 * k
        s.sid = "rt.output{:05d}".format(k)
        s.writebin(folder=os.path.join(root, "output"), verbose=False)
    path = sphere_b200.render(os.path.join(root, "output", "rt.output00001.bin"), method="pres",
                              max_val=1.5e3, graphics_format="ppm", verbose=False, root=root)
    assert path == os.path.join(root, "img_out", "rt.output00001.ppm")
    from sphere_b200.sim import read_ppm
    assert numpy.array_equal(read_ppm(path), O.render(s, 1, 1.5e3, 0.0, 800, 800))
    s.sid = "rt"
    pngs = s.render(method="pres", max_val=1.5e3, verbose=False, root=root)
    assert [os.path.basename(p) for p in pngs] == ["rt.output00000.png", "rt.output00001.png"]
    assert all(os.path.getsize(p) > 0 for p in pngs)
    assert not os.path.exists(path)
