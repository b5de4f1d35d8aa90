#!/usr/bin/env python
"""DEM step throughput in particle-steps/s on the 1e6-sphere sheared dense
pack (log-normal radii, porosity ~0.40, x-y periodic, 20 kPa top wall, top
layer sheared at 0.01 m/s, k_n = k_t = 1.16e9, gamma_n = 1e3, mu = 0.5,
NC = 32), one pack per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                    [--impl ours|reference] [--n SPHERES] [--no-adjoint]

Our arm: W untimed steps, then K steps timed with CUDA events on the stream
the library launches on (a torch stream made current and handed to the
library with sph_set_stream), bracketed by a barrier and torch.cuda.synchronize(); the
max over ranks is reported.  The working set (~2.5 GB at 1e6 spheres) is
far larger than L2, so no L2 flush is needed.  Per-kernel durations come
from CUDA events recorded inside 8 step graphs run after the timed region
(sph_profile).  Then: live-contact count for the byte count, the roofline
of the dominant kernel, the end-to-end time through the C ABI with host
buffers, and (rank 0, N = 1) the CPU baseline: the reference's own step
kernels compiled for the CPU (oracle/_ref) on a bounded sample.  Rank 0
also reports the cost of the adjoint (time_adjoint) under "adjoint", the
batched-ensemble throughput and per-box error (time_ensemble) under
"ensemble", the bonded-pack throughput (time_bonded) under "bonded", the
FP64 gravity settling (time_settling) under "settling" and the
Darcy-coupled pack with the reference's CPU kernels beside it (time_darcy)
under "darcy".

--impl reference times that CPU reference alone (rank 0; other ranks exit).

One JSON line is printed by rank 0.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s @1e6 spheres, FP32-mixed vs FP64 on B200; adjoint/forward cost"
UNIT = "particle-steps/s"
PROFILE_RING = 8  # step graphs with event-record nodes held by the C ABI (SphHandle::PR)
WORKLOAD = ("sheared dense pack, 1e6 spheres: log-normal radii median 0.01 m sigma_ln 0.2 "
            "clipped [0.005, 0.02], porosity 0.40, x-y periodic 1:1:0.5, top wall 20 kPa, "
            "top layer +x 0.01 m/s, k_n=k_t=1.16e9, gamma_n=1e3, mu=0.5, NC=32")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler(object):
    """nvidia-smi clocks and throttle reasons, sampled during the timed
    region (100 ms period)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def make_scene(n, seed, device, sweeps=3000):
    from sphere_b200 import scenes
    return scenes.sheared_dense_pack(n=n, seed=seed, device=device, sweeps=sweeps)


def interact_bytes(n, c, precision):
    """Algorithmic bytes of one launch of the fused interact+integrate
    kernel: per sphere, the compulsory state read and written once
    (S_r = 184 B: x+r, vel+fixvel, angvel, angpos, xyzsum, acc0, angacc0;
    S_w = 168 B: the same seven 3-vectors), per live directed contact its
    partner id (4 B) and tangential history read and written (2 x 24 B)."""
    if precision == "mixed":
        return 220 * n + 52 * c
    return 352 * n + 52 * c


def step_bytes(n, c, precision):
    """Whole-step algorithmic bytes: interact bytes + the cell sort
    (16 B x 3 radix-equivalent passes per sphere)."""
    return interact_bytes(n, c, precision) + 48 * n


def cpu_reference_rate(s, nsteps, budget_s=25.0, warmup=0):
    """Time the reference's own kernels on the CPU (oracle/_ref) on a
    bounded sample: after `warmup` untimed whole steps (at most budget_s / 2
    seconds of them), whole steps of the same scene, up to nsteps or
    budget_s seconds.  Returns (particle-steps/s, steps timed, seconds,
    threads, kind, warm-up steps run)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kind = "reference" if O.available("ref") else "port"
    which = "ref" if kind == "reference" else "oracle"
    threads = os.cpu_count() or 1
    run = O.CpuRun(s, which, nthreads=threads)
    n = int(s.np[0])
    w0 = time.perf_counter()
    warm = 0
    while warm < warmup and time.perf_counter() - w0 < 0.5 * budget_s:
        run.step(1)
        warm += 1
    t0 = time.perf_counter()
    run.step(1)
    done = 1
    while done < nsteps and time.perf_counter() - t0 < budget_s:
        run.step(1)
        done += 1
    dt = time.perf_counter() - t0
    return n * done / dt, done, dt, threads, kind, warm


def time_adjoint(device, stream, n=50000, steps=2000, ckpt=100):
    """Cost of the adjoint on the differentiable settling/impact scene
    (50,000 spheres, radii U[0.009, 0.011] m, loose pack porosity 0.5,
    v0 ~ N(0, 0.1) m/s, k_n = 1.5e8, gamma_n = 20, mu = 0.5, 2,000 steps,
    checkpoint every 100 steps): device time of the plain forward (graph
    steps), of the checkpointed forward and of the backward pass
    (recompute + reverse) for loss = mean |x_T - x_target|^2, the target
    being the same scene run with k_n = 1e8, gamma_n = 50, mu = 0.4."""
    import numpy
    import torch
    from sphere_b200 import scenes
    from sphere_b200.runner import Stepper
    s = scenes.loose_pack(n, seed=0, device=device)
    st = Stepper([s], precision="fp64", length="fp64", device=device)
    st.set_stream(stream.cuda_stream)
    st.upload()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    st.step(3)          # graph build and first launches, untimed
    st.upload()
    start.record(stream)
    st.step_async(steps)
    end.record(stream)
    end.synchronize()
    st.sync()
    plain_ms = start.elapsed_time(end)
    st.upload()
    fwd_ms = st.adjoint_forward(steps, ckpt)
    hp, _ = st.download()
    tgt = Stepper([scenes.reparam(s, k_n=1e8, gamma_n=50.0, mu=0.4)], precision="fp64",
                  length="fp64", device=device)
    tgt.upload()
    tgt.step(steps)
    ht, _ = tgt.download()
    tgt.close()
    dx = 2.0 * (hp.x[:, :3] - ht.x[:, :3]) / n      # d/dx_T of mean |x_T - x_target|^2
    g, gv, adj_ms = st.adjoint_backward(dx)
    st.close()
    return {"workload": "differentiable settling/impact, 50,000 spheres U[0.009, 0.011] m, "
                        "loose pack porosity 0.5, v0 ~ N(0, 0.1) m/s, linear contacts "
                        "k_n=1.5e8 gamma_n=20 mu=0.5, FP64, 2,000 steps, checkpoint every 100",
            "forward_ms": plain_ms, "forward_checkpointed_ms": fwd_ms, "backward_ms": adj_ms,
            "backward_over_forward": adj_ms / plain_ms,
            "forward_and_backward_over_forward": (fwd_ms + adj_ms) / plain_ms,
            "grad_params": [g["k_n"], g["gamma_n"], g["mu"]],
            "grad_v0_norm": float(numpy.linalg.norm(gv))}


def time_ensemble(device, stream, nboxes=256, steps=200, err_steps=100, rank=0, world=1,
                  barrier=None, max_over_ranks=None):
    """The batched ensemble (256 independent x-y periodic shear boxes with
    uniform particle counts in [500, 20000], radii U[0.009, 0.011] m,
    per-box normal stress U[10, 80] kPa and mu U[0.3, 0.6]), its boxes
    shared out over the ranks by particle count (ensemble.partition, no
    data-path exchange): each rank makes and steps its own boxes in one
    handle, every step one CUDA graph whose launches cover all of them.
    Reports the FP32-mixed ensemble throughput (all ranks' spheres over the
    slowest rank's time; launch variant and shape picked by sph_autotune)
    and, per box, the mixed form's error against the FP64 form: force
    relative L2 after one step and the largest position difference after
    err_steps steps, relative to the mean radius (the largest over ranks)."""
    import numpy
    import torch
    from sphere_b200 import ensemble, scenes
    from sphere_b200.runner import Stepper
    all_counts = scenes.ensemble_counts(nboxes=nboxes, seed=0)
    mine = ensemble.partition(all_counts, world)[rank]
    sims = scenes.shear_ensemble(nboxes=nboxes, seed=0, device=device, subset=mine)
    counts = [int(q.np[0]) for q in sims]
    n = sum(counts)
    st = Stepper(sims, precision="mixed", length="reference", device=device)
    st.set_stream(stream.cuda_stream)
    st.upload()
    variant, variant_ms = st.autotune(steps=10)
    tuning = st.tuning()
    st.step(5)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if barrier:
        barrier()
    start.record(stream)
    st.step_async(steps)
    end.record(stream)
    end.synchronize()
    code = st.sync(raise_on_error=False)
    ms = start.elapsed_time(end)
    if barrier:
        barrier()
    if max_over_ranks:
        ms = max_over_ranks(ms)
    st.close()
    # per-box error of the mixed form against the FP64 form
    a = Stepper(sims, precision="fp64", length="reference", device=device)
    b = Stepper(sims, precision="mixed", length="reference", device=device)
    a.upload()
    b.upload()
    a.step(1)
    b.step(1)
    fa, _ = a.download()
    fb, _ = b.download()
    a.step(err_steps - 1)
    b.step(err_steps - 1)
    xa, _ = a.download()
    xb, _ = b.download()
    a.close()
    b.close()
    ferr, xerr = [], []
    o = 0
    for q, k in zip(sims, counts):
        da = fa.force[o:o + k]
        db = fb.force[o:o + k]
        ferr.append(float(numpy.linalg.norm(db - da) / max(numpy.linalg.norm(da), 1e-300)))
        xerr.append(float(numpy.max(numpy.abs(xa.x[o:o + k, :3] - xb.x[o:o + k, :3]))) /
                    float(numpy.mean(q.radius)))
        o += k
    fmax, xmax = max(ferr), max(xerr)
    if max_over_ranks:
        fmax, xmax = max_over_ranks(fmax), max_over_ranks(xmax)
    total = sum(all_counts)
    return {"workload": "%d independent x-y periodic shear boxes, %d..%d spheres each "
                        "(%d in total), radii U[0.009, 0.011] m, porosity ~0.40, normal "
                        "stress U[10, 80] kPa, mu U[0.3, 0.6], FP32-mixed, one handle per rank"
                        % (nboxes, min(all_counts), max(all_counts), total),
            "value": total * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "spheres": total, "ranks": world,
            "scaling": "strong" if world > 1 else None,
            "boxes_on_rank0": len(mine), "spheres_on_rank0": n,
            "variant": variant, "variant_ms_per_step": variant_ms,
            "tuning": {"variant": tuning[0], "list_step_shape": tuning[1]},
            "device_status": code,
            "per_box_force_rel_l2_max": fmax, "per_box_force_rel_l2_median_rank0":
                float(numpy.median(ferr)),
            "per_box_dx_over_rmean_max_after_%d_steps" % err_steps: xmax}


def time_bonded(device, stream, n=200000, nbonds=300000, steps=200):
    """The bonded-pack workload: 2e5 spheres U[0.008, 0.012] m at porosity
    0.38, 3e5 linear bonds between touching pairs (k = 1e9, sigma_b = 1 MPa),
    Young's-modulus contacts (E = 70 GPa), top wall at -0.005 m/s
    (uniaxialStrainRate), FP32-mixed; launch variant picked by sph_autotune."""
    import torch
    from sphere_b200 import scenes
    from sphere_b200.runner import Stepper
    s = scenes.bonded_pack(n=n, nbonds=nbonds, seed=0, device=device)
    nb = int(s.nb0[0])
    st = Stepper([s], precision="mixed", length="reference", device=device)
    st.set_stream(stream.cuda_stream)
    st.upload()
    variant, variant_ms = st.autotune(steps=10)
    st.step(5)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(stream)
    st.step_async(steps)
    end.record(stream)
    end.synchronize()
    code = st.sync(raise_on_error=False)
    ms = start.elapsed_time(end)
    st.close()
    return {"workload": "bonded pack: %d spheres U[0.008, 0.012] m, porosity 0.38, %d linear "
                        "bonds between touching pairs (k_n = k_t = 1e9, sigma_b = 1 MPa), "
                        "E = 70 GPa contacts, top wall at -0.005 m/s, FP32-mixed" % (n, nb),
            "value": n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "spheres": n, "bonds": nb, "variant": variant,
            "variant_ms_per_step": variant_ms, "device_status": code}


def time_settling(device, stream, n=10000, steps=1000):
    """The FP64 gravity-settling workload (scenes.gravity_settling: 10,000
    spheres U[0.010, 0.012] m on a jittered cubic lattice, 0.5 x 0.5 m box
    with wall sides, k_n = k_t = 1.16e9, no damping, mu = 0.5,
    dt = 0.17 sqrt(m_min / k_n)), its whole run of 1,000 steps queued at once
    and timed with CUDA events on the launching stream: a small box whose
    step time is set by launch latency and the few dependent kernels of a
    step, not by bandwidth."""
    import torch
    from sphere_b200 import scenes
    from sphere_b200.runner import Stepper
    s = scenes.gravity_settling(n=n, seed=0, steps=steps)
    st = Stepper([s], precision="fp64", length="reference", device=device)
    st.set_stream(stream.cuda_stream)
    st.upload()
    variant, variant_ms = st.autotune(steps=20)
    st.step(5)
    st.upload()    # the timed run starts from the workload's initial state
    st.step(3)     # graphs of the overlapped steps instantiated, untimed
    st.upload()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    launches0 = st.kernel_launches()
    start.record(stream)
    st.step_async(steps)
    end.record(stream)
    end.synchronize()
    code = st.sync(raise_on_error=False)
    ms = start.elapsed_time(end)
    launches = st.kernel_launches() - launches0
    st.close()
    return {"workload": "FP64 gravity settling, %d spheres U[0.010, 0.012] m, jittered cubic "
                        "lattice (spacing 2.5 r_max), 0.5 x 0.5 x 1.25 m box with wall sides, "
                        "k_n=k_t=1.16e9, gamma=0, mu=0.5, dt=0.17 sqrt(m_min/k_n), %d steps "
                        "(the whole run)" % (n, steps),
            "value": n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "spheres": n, "variant": variant,
            "variant_ms_per_step": variant_ms, "gpu_launches": launches,
            "device_status": code}


def time_darcy(device, stream, n=100000, steps=100, ref_n=5000):
    """The Darcy-coupled pack (scenes.darcy_pack: a lattice pack of n
    spheres U[0.009, 0.011] m under a 10 kPa top wall, periodic x-y, in
    water at hydrostatic pressure, beta_f = 1e-7 1/Pa, grain-size
    permeability; the fluid on the cell grid), FP64 with the fluid updated
    every step: steps queued at once and timed with CUDA events on the
    launching stream, the Jacobi iterations of each step from its log, the
    per-kernel-group times from the profiled step graphs.  Beside it the
    reference's own DEM and Darcy kernels on the CPU (oracle/_ref), all host
    threads, on the same construction at ref_n spheres."""
    import numpy
    import torch
    from sphere_b200 import scenes
    from sphere_b200.runner import Stepper
    s = scenes.darcy_pack(n, seed=31)
    s.time_file_dt[0] = 1.0   # no output inside the timed steps
    st = Stepper([s], precision="fp64", length="reference", device=device)
    st.set_stream(stream.cuda_stream)
    st.upload()
    st.step(3)     # graphs instantiated, untimed
    st.upload()    # the timed run starts from the workload's initial state
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    launches0 = st.kernel_launches()
    start.record(stream)
    st.step_async(steps)
    end.record(stream)
    end.synchronize()
    code = st.sync(raise_on_error=False)
    ms = start.elapsed_time(end)
    launches = st.kernel_launches() - launches0
    _, iters, ok = st.darcy_log()
    try:
        st.profile(True)
        st.step_async(PROFILE_RING)
        st.sync(raise_on_error=False)
        st.step_async(PROFILE_RING)
        st.sync(raise_on_error=False)
        kernels = st.profile_read()
    except Exception as e:
        kernels = {"error": str(e)}
    st.profile(False)
    st.close()
    cells = int(s.num[0]) * int(s.num[1]) * int(s.num[2])
    it = float(numpy.mean(iters)) if len(iters) else 0.0
    sr = scenes.darcy_pack(ref_n, seed=31)
    sr.time_file_dt[0] = 1.0
    rate, done, secs, threads, kind, _ = cpu_reference_rate(sr, 20, 10.0)
    return {"workload": "Darcy-coupled pack: %d spheres U[0.009, 0.011] m (jittered lattice, "
                        "periodic x-y, 10 kPa top wall) in water (mu = 8.9e-4 Pa s) at "
                        "hydrostatic pressure, beta_f = 1e-7 1/Pa, k_c = d^2/180, fluid on the "
                        "%d x %d x %d cell grid updated every step, FP64, %d steps"
                        % (n, int(s.num[0]), int(s.num[1]), int(s.num[2]), steps),
            "value": n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "spheres": n, "fluid_cells": cells,
            "jacobi_iterations_per_step": it, "solves_converged": int(numpy.sum(ok)),
            "jacobi_cell_iterations_per_s": cells * it * steps / (ms / 1e3),
            "kernel_ms": kernels, "gpu_launches": launches, "device_status": code,
            "cpu_reference": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                              "sample": "%d whole steps of the same construction at %d spheres "
                                        "(%.1f s)" % (done, ref_n, secs)}}


def bench_config(args):
    """The `config` object of the JSON line, the same in both arms."""
    return {"workload": WORKLOAD, "spheres_per_gpu": args.n, "length_mode": "reference",
            "l2": "working set > L2 (no flush needed)",
            "parallelism": "replicas only (one independent pack per GPU)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1000000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pack-sweeps", type=int, default=3000)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-bonded", action="store_true")
    ap.add_argument("--no-settling", action="store_true")
    ap.add_argument("--no-darcy", action="store_true")
    ap.add_argument("--darcy-only", action="store_true",
                    help="run only the Darcy-coupled workload (time_darcy) and print its JSON")
    ap.add_argument("--darcy-n", type=int, default=100000,
                    help="spheres of the Darcy-coupled workload")
    ap.add_argument("--darcy-steps", type=int, default=100)
    ap.add_argument("--ref-n", type=int, default=100000,
                    help="spheres of the reference arm's sample of the workload (the same "
                         "construction, packed on the CPU)")
    ap.add_argument("--no-long-run", action="store_true",
                    help="skip the mixed-vs-FP64 comparison over the whole run")
    ap.add_argument("--kernel-tour", action="store_true",
                    help="run every kernel family once inside the NVTX range 'k' (for profiling) "
                         "and exit")
    ap.add_argument("--variant", type=int, default=-1,
                    help="interact launch variant (0-4); default: picked by sph_autotune")
    ap.add_argument("--shape", type=int, default=0,
                    help="launch shape of the list step (variant 4) when --variant is given")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.darcy_only:
        import torch
        torch.cuda.set_device(local)
        out = time_darcy(local, torch.cuda.Stream(), n=args.darcy_n, steps=args.darcy_steps,
                         ref_n=min(5000, args.darcy_n))
        if rank == 0:
            print(json.dumps(out))
        return 0

    if args.impl == "reference":
        # The reference's own step kernels compiled for the CPU
        # (oracle/_ref), all host threads, on a bounded sample of the
        # workload: the same construction (log-normal FCC start, the packing
        # sweeps, radii grown, shear set-up) at args.ref_n spheres, packed
        # on the CPU by the C restatement of the packing sweeps, which gives
        # the GPU's pack bit for bit.  Nothing of this arm runs on a GPU or
        # loads this project's CUDA library.
        if rank != 0:
            return 0
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        from sphere_b200 import scenes
        nref = min(args.ref_n, args.n)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        s = scenes.sheared_dense_pack(
            n=nref, seed=0, sweeps=args.pack_sweeps,
            relax=lambda q, k, a, z: O.relax(q, k, alpha=a, z_top=z, nthreads=threads))
        t_pack = time.perf_counter() - t0
        rate, done, secs, threads, kind, warm = cpu_reference_rate(s, args.steps, 120.0,
                                                                   warmup=args.warmup)
        sample = ("%d whole steps after %d untimed ones, of the workload's construction at "
                  "%d spheres (packed on the CPU in %.0f s by the packing sweeps' C "
                  "restatement)" % (done, warm, nref, t_pack))
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT,
                "n_gpus": args.gpus, "steps": done, "warmup": warm,
                "ms_per_step": secs / done * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": bench_config(args),
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                                 "sample": sample},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    import torch.distributed as dist
    from sphere_b200.runner import Stepper, HostParticles

    if args.kernel_tour:
        # every kernel family once, inside one NVTX range: split steps in
        # both forms, fused steps, a render, a porosity profile, an overlap
        # listing, packing sweeps, the contact count and the download, the
        # unfused step of a shear-stress wall, bonded steps (split and
        # fused), an adjoint forward + backward pass and the cell-offset
        # scan with caller-owned memory
        import copy
        import numpy
        from sphere_b200 import scenes
        torch.cuda.set_device(local)
        s = make_scene(args.n, 0, local, args.pack_sweeps)
        # the same pack under a shear-stress top wall (wmode 3: the unfused
        # step), a bonded pack and the adjoint's loose pack, made before the
        # range
        s3 = copy.deepcopy(s)
        s3.wmode[0] = 3
        s3.w_tau_x[0] = 500.0
        nbd = min(args.n, 200000)
        sb = scenes.bonded_pack(n=nbd, nbonds=3 * nbd // 2, seed=0, device=local)
        sa = scenes.loose_pack(50000, seed=0, device=local)
        import ctypes as C
        from sphere_b200 import _abi
        lib = _abi.load_library()
        ncell = 4_000_000
        d_counts = torch.randint(0, 8, (ncell,), dtype=torch.int32, device="cuda")
        d_off = torch.empty(ncell + 1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("k")
        for prec in ("mixed", "fp64"):
            st = Stepper([s], precision=prec, length="reference", device=local)
            st.upload()
            st.set_variant(3)
            st.step(3)
            if prec == "mixed":
                # the list step (its first step rebuilds the lists)
                st.set_variant(4)
                st.step(3)
            if prec == "fp64":
                st.set_variant(1)
                st.step(2)
                st.render(method=1, maxval=1e3, width=800, height=800)
                st.porosity(10)
                st.overlaps()
                st.relax(2, alpha=0.5, z_top=float(s.L[2]))
                st.count_contacts()
                st.download()
            st.close()
        st = Stepper([s3], precision="fp64", length="reference", device=local)
        st.upload()
        st.step(2)
        st.close()
        st = Stepper([sb], precision="mixed", length="reference", device=local)
        st.upload()
        st.set_variant(3)
        st.step(2)
        st.set_variant(1)
        st.step(1)
        st.close()
        st = Stepper([sa], precision="fp64", length="fp64", device=local)
        st.upload()
        st.adjoint_forward(4, 2)
        hp, _ = st.download()
        st.adjoint_backward(numpy.ascontiguousarray(hp.x[:, :3]) * 1e-3)
        st.close()
        # the cell-offset scan with caller-owned memory (4e6 cells)
        rc = lib.sph_cell_offsets_static(
            C.c_void_p(d_counts.data_ptr()), C.c_uint64(ncell), C.c_void_p(d_off.data_ptr()),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("sph_cell_offsets_static: status %d" % rc)
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"kernel_tour": "done", "spheres": args.n}))
        return 0

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    s = make_scene(args.n, rank, local, args.pack_sweeps)
    n = int(s.np[0])
    # a stream of our own (never the legacy default stream, whose handle is
    # 0 and would send the library to its internal stream): the library
    # launches on it (sph_set_stream) and the timing events are recorded on it
    stream = torch.cuda.Stream(device=local)
    assert stream.cuda_stream != 0
    torch.cuda.set_stream(stream)
    hbm, peak_kind = peaks()

    def max_over_ranks(v):
        if world > 1:
            t = torch.tensor([v], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return v

    def time_form(precision):
        """W warm-up steps, then K steps timed with CUDA events on the
        launching stream; per-kernel times from the profiled step graphs."""
        st = Stepper([s], precision=precision, length="reference", device=local)
        st.set_stream(stream.cuda_stream)
        st.upload()
        # launch variant of the interact kernel picked on this scene (the
        # state is put back afterwards), then the warm-up steps
        if args.variant >= 0:
            st.set_variant(args.variant)
            st.set_launch_shape(args.shape)
            variant, variant_ms = args.variant, None
        else:
            variant, variant_ms = st.autotune(steps=20)
        st.step(args.warmup)
        clocks = ClockSampler(local)
        barrier()
        torch.cuda.synchronize()
        clocks.start()
        time.sleep(0.3)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        launches0 = st.kernel_launches()
        torch.cuda.nvtx.range_push("timed")
        start.record(stream)
        st.step_async(args.steps)
        end.record(stream)
        end.synchronize()
        torch.cuda.nvtx.range_pop()
        code = st.sync(raise_on_error=False)
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        launches = st.kernel_launches() - launches0
        ms_max = max_over_ranks(start.elapsed_time(end))
        # per-kernel breakdown, after the timed region: the ring of step
        # graphs with event-record nodes; every ring graph runs once untimed
        # before the steps whose events are read
        try:
            st.profile(True)
            st.step_async(PROFILE_RING)
            st.sync(raise_on_error=False)
            st.step_async(PROFILE_RING)
            st.sync(raise_on_error=False)
            kernels = st.profile_read()
        except Exception as e:  # the timing above stands without the breakdown
            kernels = {"error": str(e)}
        st.profile(False)
        contacts = st.count_contacts()
        nstats = st.neighbor_stats()
        # the interact stage: the fused kernel, the three kernels of the
        # split step or the list step's kernel (same work, same algorithmic
        # bytes)
        if "k_pair_step" in kernels:
            stage = ["k_pair_step"]
        elif "k_interact" in kernels:
            stage = ["k_interact"]
        else:
            stage = ["k_search", "k_contacts", "k_finish"]
        parts = [kernels.get(k) for k in stage]
        t_int = sum(parts) if all(isinstance(v, float) for v in parts) else None
        b_int = interact_bytes(n, contacts, precision)
        achieved = b_int / (t_int / 1e3) / 1e9 if t_int else None
        roofline = {"bound": "hbm", "kernel": "+".join(stage), "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                    "peak_source": peak_kind, "traffic": None,
                    "algorithmic_bytes_per_launch": b_int, "kernel_ms": t_int}
        try:
            with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
                tr = json.load(fh)
            key = "mixed_list" if stage == ["k_pair_step"] else precision
            if tr[key]["kernels"] == "+".join(stage):
                roofline["traffic"] = tr[key]["bytes_per_sphere"] * n
                roofline["traffic_source"] = tr["source"] + "; " + tr[key]["capture"]
        except Exception:
            pass
        tuning = st.tuning()
        shape_ms = [round(float(v), 4) for v in st.shape_times()] if variant_ms is not None else []
        st.close()
        ms_step = ms_max / args.steps
        return {"value": world * n * args.steps / (ms_max / 1e3), "ms_per_step": ms_step,
                "variant": variant, "variant_ms_per_step": variant_ms,
                "tuning": {"variant": tuning[0], "list_step_shape": tuning[1],
                           "list_step_shape_ms": shape_ms},
                "neighbor_lists": nstats,
                "roofline": roofline, "kernel_ms": kernels, "live_contacts": contacts,
                "gpu_launches": launches, "clocks": clk, "device_status": code,
                "step_gbs": step_bytes(n, contacts, precision) / (ms_step / 1e3) / 1e9}

    forms = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    res = {f: time_form(f) for f in forms}
    head = "mixed" if "mixed" in res else forms[0]
    H = res[head]

    # end to end through the C ABI with host buffers: upload from pinned
    # host memory, K steps each followed by a read of the box state (wall
    # force/position, time), download of the final state
    e2e = None
    if rank == 0 or world > 1:
        st2 = Stepper([s], precision=head, length="reference", device=local)
        st2.set_stream(stream.cuda_stream)
        st2.set_variant(H["tuning"]["variant"])
        st2.set_launch_shape(H["tuning"]["list_step_shape"])
        hp = HostParticles.from_sims([s])
        for name in ("x", "xyzsum", "vel", "force", "angpos", "angvel", "torque", "es_dot", "es",
                     "ev_dot", "ev", "p"):
            a = getattr(hp, name)
            pin = torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
            pin[...] = a
            setattr(hp, name, pin)
        st2.hp = hp
        import ctypes as C
        h2d = sum(getattr(hp, k).nbytes for k in ("x", "xyzsum", "vel", "force", "angpos",
                                                   "angvel", "torque", "es_dot", "es", "ev_dot",
                                                   "ev", "p"))
        nbs = st2.box_state_bytes()
        states = torch.empty((max(args.steps, args.warmup), nbs), dtype=torch.uint8,
                             pin_memory=True).numpy()
        # warm-up: the same calls untimed (graphs instantiated, pages touched);
        # the timed upload below starts the scene again from the host arrays
        ps = hp.struct()
        st2._check(st2.lib.sph_upload(st2.h, C.byref(ps), None), "sph_upload")
        st2.step_async_states(args.warmup, states)
        st2._check(st2.lib.sph_sync(st2.h), "sph_sync")
        # the final state goes to pinned host arrays as well
        out = HostParticles(n)
        for name in ("x", "xyzsum", "vel", "force", "angpos", "angvel", "torque", "es_dot", "es",
                     "ev_dot", "ev", "p"):
            a = getattr(out, name)
            setattr(out, name, torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy())
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        ps = hp.struct()
        st2._check(st2.lib.sph_upload(st2.h, C.byref(ps), None), "sph_upload")
        t1 = time.perf_counter()
        # every step's result (time, wall force and position) copied into
        # pinned host memory as the step ends, the steps queued back to
        # back; device errors collected once, then each state decoded
        st2.step_async_states(args.steps, states[:args.steps])
        st2._check(st2.lib.sph_sync(st2.h), "sph_sync")
        t2 = time.perf_counter()
        per_step = st2.boxes_from_states(states, args.steps)
        t3 = time.perf_counter()
        po = out.struct()
        st2._check(st2.lib.sph_download(st2.h, C.byref(po), None), "sph_download")
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        parts = {"upload_s": t1 - t0, "steps_and_sync_s": t2 - t1, "decode_s": t3 - t2,
                 "download_s": t_e2e - (t3 - t0)}
        barrier()
        if world > 1:
            t = torch.tensor([t_e2e], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        d2h = h2d + nbs * args.steps
        assert per_step[-1][0].t_current > per_step[0][0].t_current or args.steps == 1
        e2e = {"value": world * n * args.steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "seconds": t_e2e, "parts": parts,
               "what": "sph_upload from pinned host arrays + sph_step_async_states (K steps, "
                       "the box state after each copied to pinned host memory) + sph_sync + "
                       "decoding of the K states + sph_download into pinned host arrays"}
        st2.close()

    adj = None
    if rank == 0 and not args.no_adjoint:
        adj = time_adjoint(local, stream)
    ens = None
    if not args.no_ensemble:
        # every rank steps its share of the boxes (all ranks take part)
        ens = time_ensemble(local, stream, rank=rank, world=world, barrier=barrier,
                            max_over_ranks=max_over_ranks)
    bonded = None
    if rank == 0 and not args.no_bonded:
        bonded = time_bonded(local, stream)
    settling = None
    if rank == 0 and not args.no_settling:
        settling = time_settling(local, stream)
    darcy = None
    if rank == 0 and not args.no_darcy:
        darcy = time_darcy(local, stream, n=args.darcy_n, steps=args.darcy_steps)
    long_run = None
    if rank == 0 and not args.no_long_run and "mixed" in res and "fp64" in res:
        # the mixed form's error against the FP64 form over the workload's
        # whole run (5,000 steps of the same pack): wall stress, porosity;
        # in the launch variant timed above, beside the floor of the chaotic
        # flow (FP64 against FP64 from positions moved by 1e-15 relative)
        from sphere_b200.mixed_error import compare_precisions
        long_run = compare_precisions(s, slices=50, device=local, cuda_stream=stream.cuda_stream,
                                      variant=res["mixed"]["tuning"]["variant"])
        long_run["fp64_floor"] = compare_precisions(s, slices=50, device=local,
                                                    cuda_stream=stream.cuda_stream,
                                                    precision="fp64", perturb=1e-15)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, done, secs, threads, kind, _ = cpu_reference_rate(s, 50, 25.0)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": "%d whole steps of the same %d-sphere pack (%.1f s)" % (done, n, secs)}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": H["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": H["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "f64+f32",
        "data": "synthetic (seeded GPU-relaxed pack per rank)",
        "config": bench_config(args),
        "precision": head, "forms_timed": forms,
        "roofline": H["roofline"],
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": H["gpu_launches"],
        "clocks": H["clocks"],
        "live_contacts": H["live_contacts"],
        "kernel_ms": H["kernel_ms"],
        "interact_variant": H["variant"],
        "step_gbs": H["step_gbs"],
        "device_status": H["device_status"],
        "forms": res,
    }
    if "fp64" in res and "mixed" in res:
        line["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    if adj is not None:
        line["adjoint"] = adj
    if ens is not None:
        line["ensemble"] = ens
    if bonded is not None:
        line["bonded"] = bonded
    if settling is not None:
        line["settling"] = settling
    if darcy is not None:
        line["darcy"] = darcy
    if long_run is not None:
        line["mixed_error_long_run"] = long_run
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
