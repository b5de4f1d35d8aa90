"""Build the CUDA library in place: sphere_b200/libsphere_b200.so (sm_100a).

    python -m sphere_b200.build [--verbose]

Each .cu file is compiled separately: the FP64 step (sph_kernels.cu) and the
C ABI without FMA contraction (-fmad=false) so that FP64 results reproduce
the reference's arithmetic bit for bit, the FP32-mixed split step
(sph_mixed.cu) with contraction, the list step (sph_pair.cu) without it, so
that its launch shapes, compiled under different register budgets, give the
same bits.  ptxas resource usage is written to
sphere_b200/_build/ptxas.log.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libsphere_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]
SOURCES = [
    ("sph_kernels.cu", ["-fmad=false"]),
    ("sph_capi.cu", ["-fmad=false"]),
    ("sph_mixed.cu", ["-fmad=true"]),
    ("sph_pair.cu", ["-fmad=false", "-ftz=true"]),
    ("sph_darcy.cu", ["-fmad=false"]),
    ("sph_adjoint.cu", ["-fmad=false"]),
    ("sph_noalloc.cu", []),
    ("sph_render.cu", ["-fmad=false"]),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    log = []
    # the sources, the public header, and this file (its flags)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(ROOT, "include", "sphere_b200.h"), os.path.abspath(__file__)]
    newest_dep = max(os.path.getmtime(d) for d in deps)
    for src, flags in SOURCES:
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
            continue
        cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        log.append("$ " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed on " + src)
    if log:
        with open(os.path.join(BUILD, "ptxas.log"), "w") as fh:
            fh.write("\n".join(log))
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "--cudart", "static", "-o", OUT] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
