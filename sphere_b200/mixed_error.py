"""The FP32-mixed form's error against the FP64 form over a whole run.

The FP64 form is bit-identical to the oracle (the FP64 restatement of the
reference's kernels, src/contactmodels.cuh, src/integration.cuh), so these
differences are the mixed form's error against the oracle.  Both forms run
the same scene for the same number of steps from the same state; every
step's box state (wall position and force, time) is copied to host memory
while the steps run (sph_step_async_states), and at the end the porosity
profile (sph_porosity, the reference's `porosity` program) and the
positions are read back.
"""
import copy
import math

import numpy

from .runner import Stepper


def _run(sim, precision, nsteps, slices, device, cuda_stream, max_slices=0, variant=None):
    st = Stepper([sim], precision=precision, length="reference", device=device)
    try:
        if cuda_stream is not None:
            st.set_stream(cuda_stream)
        if variant is not None:
            st.set_variant(variant)
        st.upload()
        nbs = st.box_state_bytes()
        states = numpy.zeros((nsteps, nbs), dtype=numpy.uint8)
        st.step_async_states(nsteps, states)
        code = st.sync(raise_on_error=False)
        boxes = [b[0] for b in st.boxes_from_states(states, nsteps)]
        if slices is None:
            # slabs thicker than 2 r_max (src/sphere.cpp:492-515), one to
            # spare so that both forms' wall positions allow the same count
            top = boxes[-1].walls.nx[0][3] if boxes else float(sim.w_x[0])
            h = top - float(sim.origo[2])
            slices = max(1, min(max_slices, int(math.ceil(h / (2.0 * float(sim.radius.max())))) - 2))
        z, por = st.porosity(slices)
        hp, _ = st.download()
    finally:
        st.close()
    return {"wall_x": numpy.array([b.walls.nx[0][3] for b in boxes]),
            "wall_force": numpy.array([b.walls.mvfd[0][2] for b in boxes]),
            "t": numpy.array([b.t_current for b in boxes]),
            "z": z, "porosity": por, "slices": slices, "x": hp.x[:, :3].copy(),
            "status": int(code)}


def perturbed(sim, rel, seed=0):
    """A copy of sim whose sphere positions are multiplied by 1 +- rel
    (a seeded random sign per coordinate)."""
    q = copy.deepcopy(sim)
    x = numpy.asarray(q.x)
    sign = numpy.random.default_rng(seed).choice([-1.0, 1.0], size=x[:, :3].shape)
    x[:, :3] *= 1.0 + rel * sign
    q.x = x
    return q


def compare_precisions(sim, nsteps=None, slices=50, device=-1, cuda_stream=None,
                       precision="mixed", variant=None, perturb=0.0, seed=0):
    """Run `sim` (one box with a stress-controlled top wall, wmode 1) for
    nsteps steps (default: time_total / dt) in the FP64 form and in
    `precision` (the FP32-mixed form by default; launch variant `variant`,
    None for the handle's default; its start positions multiplied by
    1 +- perturb, a seeded sign per coordinate, when perturb > 0) and
    return the second run's differences from the first:

    * wall stress (wall force / x-y area): the largest difference over the
      run relative to the applied stress w_sigma0 and to the FP64 series'
      largest stress, the RMS difference relative to the FP64 RMS, and the
      difference of the means over the second half of the run relative to
      the FP64 mean (the series is a train of impacts: a spike a step early
      or late makes a large largest difference, the means stay close);
    * bulk porosity below the wall, 1 - V_spheres / (A (w_x - z_floor)),
      z_floor the lowest sphere bottom at the start: the largest absolute
      difference over the run;
    * wall position: the largest difference relative to the mean radius;
    * the porosity profile at the end, in at most `slices` slabs (as many as
      slabs thicker than 2 r_max allow): the largest absolute difference;
    * sphere positions at the end: the largest difference relative to the
      mean radius.

    A sheared pack is chaotic: any difference, a rounding or a move of one
    part in 1e15 of the start positions, grows until the two runs are
    different realisations of the same flow.  precision="fp64" with
    perturb=1e-15 measures that floor: the differences two FP64 runs
    show for no other reason.
    """
    if int(sim.nw[0]) < 1 or int(sim.wmode[0]) != 1:
        raise ValueError("compare_precisions wants a stress-controlled top wall (wmode 1)")
    if nsteps is None:
        nsteps = int(round(float(sim.time_total[0]) / float(sim.time_dt[0])))
    d = _run(sim, "fp64", nsteps, None, device, cuda_stream, max_slices=slices)
    second = perturbed(sim, perturb, seed) if perturb > 0.0 else sim
    m = _run(second, precision, nsteps, d["slices"], device, cuda_stream, variant=variant)
    area = float(sim.L[0]) * float(sim.L[1])
    sigma0 = float(sim.w_sigma0[0])
    r = sim.radius
    r_mean = float(r.mean())
    v_spheres = float((4.0 / 3.0 * numpy.pi * r ** 3).sum())
    z_floor = float((sim.x[:, 2] - r).min())
    sd, sm = d["wall_force"] / area, m["wall_force"] / area
    half = nsteps // 2
    pd = 1.0 - v_spheres / (area * (d["wall_x"] - z_floor))
    pm = 1.0 - v_spheres / (area * (m["wall_x"] - z_floor))
    return {
        "steps": nsteps,
        "spheres": int(sim.np[0]),
        "second_run": {"precision": precision, "variant": variant, "perturb": perturb},
        "status": [d["status"], m["status"]],
        "times_equal": bool(numpy.array_equal(d["t"], m["t"])),
        "wall_stress_max_diff_over_sigma0": float(numpy.abs(sm - sd).max() / sigma0),
        "wall_stress_max_diff_over_max": float(numpy.abs(sm - sd).max() / numpy.abs(sd).max()),
        "wall_stress_rms_diff_over_rms": float(
            numpy.sqrt(((sm - sd) ** 2).mean()) / numpy.sqrt((sd ** 2).mean())),
        "wall_stress_mean_rel_diff_second_half": float(
            abs(sm[half:].mean() - sd[half:].mean()) / abs(sd[half:].mean())),
        "wall_stress_mean_second_half_over_sigma0_fp64": float(sd[half:].mean() / sigma0),
        "bulk_porosity_max_abs_diff": float(numpy.abs(pm - pd).max()),
        "bulk_porosity_end_fp64": float(pd[-1]),
        "wall_position_max_diff_over_rmean": float(
            numpy.abs(m["wall_x"] - d["wall_x"]).max() / r_mean),
        "porosity_profile_max_abs_diff": float(numpy.abs(m["porosity"] - d["porosity"]).max()),
        "porosity_profile_slices": int(d["slices"]),
        "positions_max_diff_over_rmean": float(
            numpy.sqrt(((m["x"] - d["x"]) ** 2).sum(1)).max() / r_mean),
    }
