"""Generate tests/golden/render_<scene>.npz: images made by the reference's
own ray-tracer kernels and camera compiled for the CPU
(oracle/_ref/sphere_render_ref, built by oracle/Makefile where the reference
sources are present) for the scenes and runs of cases.render_runs.

    python tests/golden/make_render_golden.py

Each file holds img_<k> for run k (method, maxval, cutoff, width, height in
runs[k]) and a digest of the scene's inputs, which the tests recompute to
make sure they rebuild the same scene.
"""
import hashlib
import os
import sys

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def scene_digest(s):
    h = hashlib.sha256()
    for a in (s.x, s.radius, s.vel, s.fixvel, s.angvel, s.angpos, s.xyzsum, s.p, s.L):
        h.update(numpy.ascontiguousarray(a, dtype=numpy.float64).tobytes())
    return h.hexdigest()


def main():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import oracle as O
    O.build()
    for name in cases.RENDER_SCENES:
        s = cases.render_scene(name)
        runs = cases.render_runs(s)
        rec = {"runs": numpy.array(runs, dtype=numpy.float64), "digest": scene_digest(s)}
        for k, (method, maxval, cut, w, h) in enumerate(runs):
            img = O.reference_render(s, method, maxval, cut, w, h)
            if img is None:
                raise SystemExit("oracle/_ref/sphere_render_ref is not built")
            rec["img_%d" % k] = img
        numpy.savez_compressed(os.path.join(HERE, "render_%s.npz" % name), **rec)


if __name__ == "__main__":
    main()
