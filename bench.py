#!/usr/bin/env python
"""Benchmark: cell-updates/s per RK3 time step of the planar two-phase case.

Workload: the planar two-phase (Rayleigh-Taylor type) instability on its
128x512 grid -- x periodic, no-slip walls in y, Atwood 0.5, Re 3000,
Cn 0.01, Pe 1/Cn, gravity -y -- advanced with the full diffuse-interface
substep (WENO5 + explicit diffusion + implicit biharmonic CG, density and
viscosity, momentum with velocity PCG, gravity, variable-density pressure
PCG and projection) at a constant dt of 1e-4.  Synthetic initial condition
(tanh interface at mid-height perturbed by 0.05 cos 2 pi x).  Solver
tolerances are the reference defaults except the pressure iteration cap
(2000 instead of 300: with 300 the reference's own outer Poisson loop does
not reach div < 1e-6 on this grid and aborts).

One "step" = one time step (three RK substeps).  metric = N_cells x steps /
seconds.  value: device time of the timed steps with the state resident in
HBM, the L2 flushed before every step (outside the timed intervals); the
substeps replay their launches from CUDA graphs (pvof_set_graphs, on by
default).  The per-solver times behind the roofline and the solver shares
come from a following pass of --timing-steps steps issued launch by launch
with CUDA events around every solver launch.  e2e: the same steps driven
through the C ABI with the state uploaded from pinned host buffers before
every step and downloaded after it, timed by the host's clock around the
calls (the device-event time of the same interval is reported beside it).

--batch-cases K (default 6, 0 turns it off) additionally times K replicas of
the workload advanced concurrently by pvof_run_steps_batched (the batched
form: one host thread and stream per case, so the solvers of different cases
run on different SMs) and adds a "batched" object to the line; --batch-form
(default all) picks the replicas' form: fp32 (fp32-warm) the FP32 stencil
form (plus the pressure warm start), spectral / fp32-warm-spectral add the
spectral pressure preconditioner, all adds the unregularised momentum CG too;
every form but fp64 reports its error against the FP64 path.  --forms (on by
default, --no-forms turns it off) adds a "forms" list: the workload in each form of FORMS (FP32 stencils + pressure
warm start; the spectral pressure preconditioner; with it the momentum CG
without the reference's step regularisation; all of them), each with its
throughput against the plain path's and its error.

--particles adds a "particles" object: the workload with surface tension
(We 100), a 70 degree contact angle and three resolved cylinders on the
interface (two mobile, one fixed), timed against the same case without
cylinders (run last, so a launch list of the command ends with its steps).

--batch-mixed adds a "batched_mixed" object: eight instability cases of four
sizes (two each of 64x128, 128x256, 256x512, 512x1024) in all four forms,
advanced concurrently by pvof_run_steps_batched, against the same cases
advanced one after another.

--large adds a "large" object: the instability on 1024x1024 at a density
ratio of 1e-3 (--large-steps timed steps) in the plain path, with the
spectral pressure preconditioner, and with it the unregularised momentum CG.

--axisym adds an "axisym" object: the axisymmetric bubble rising towards a
fixed sphere on the axis (256x512, density ratio 1e-3, surface tension,
contact angle 90 degrees) for --axisym-steps steps, with the reference build
(AXISYM_RZ, resolved particles) on the host for --axisym-ref-steps steps.

--learned adds a "learned" object: the learned warm start on its benchmark
case (1024x1024, three mobile cylinders on a flat interface, density ratio
1e-3): the network trained on about --learned-samples 64x64 crops of the
solver's own samples, then pressure iterations and time per step with a cold
start, the same-stage warm start and the learned one.

The line also carries a "box" object (unless --no-box): the 3D mode on the
precision form's configuration, 256^3 (--box-grid), x and z periodic, walls
in y, density ratio 1e-3: --box-warmup untimed steps and --box-steps timed
steps of the plain FP64 path (device time, L2 flushed), the per-solver times
of one more step with the pressure PCG's roofline, the FP32 stencil form
from the same start with its errors against FP64 (unless --no-box-fp32), the
spectral pressure preconditioner from the same start (unless
--no-box-spectral), and the reference's 3D build on a --box-ref-grid box on
one host core.

--impl reference runs the reference's own time step (compiled from its
sources, single rank: oracle/_ref/ref_rt2d) on the same case on the host:
--warmup untimed steps, then min(--steps, --ref-steps) timed ones.
With N > 1 (torchrun) every rank advances its own replica of the case
(replicas only; the case is not split across GPUs).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "parties-vof-ibm_b200"))

METRIC = "cell-updates/s per RK step"
UNIT = "cell-updates/s"
NXM, NYM = 128, 512
DT = 1e-4
WORKLOAD = ("planar two-phase instability 128x512 (x periodic, no-slip y), Atwood 0.5, Re 3000, Cn 0.01, "
            "dt 1e-4, full RK3 substep")
# algorithmic bytes per cell and solver iteration (x, r, direction read+write,
# plus the phase field that the coefficients are derived from)
ALG_BYTES = {0: 48.0, 1: 56.0, 2: 56.0}
# the forms --forms times: (label, stencil_fp32, pressure_warm_start,
# pressure_preconditioner, velocity_cg_unregularized)
FORMS = [
    ("fp32 stencils + pressure warm start (same stage of the previous step)", 1, 1, 0, 0),
    ("fp32 stencils + learned pressure warm start (the network on the tensor cores, trained on this run's own "
     "samples)", 1, 2, 0, 0),
    ("spectral pressure preconditioner (FP64)", 0, 0, 1, 0),
    ("spectral pressure preconditioner + unregularised momentum CG (FP64)", 0, 0, 1, 1),
    ("spectral pressure preconditioner + unregularised momentum CG + fp32 stencils + pressure warm start",
     1, 1, 1, 1),
]
# (mobile, x, y, R, u, v, omega_z, rho_s): two mobile cylinders cutting the
# interface, a fixed one below it
CYLINDERS = [(1, 0.25, 2.0, 0.08, 0, 0, 0, 2.5), (1, 0.75, 2.6, 0.08, 0, 0, 0, 2.5),
             (0, 0.5, 1.2, 0.1, 0, 0, 0, 2.5)]
# the learned form's network: trained on the solver's samples of this run
LEARNED_SAMPLE_STEPS = 12
LEARNED_EPOCHS = 15
STATE_FIELDS = ["C_L", "U", "V", "P", "CH_RHS_N", "U_EXPLICIT_OLD", "V_EXPLICIT_OLD",
                "U_VISC_EXPLICIT_OLD", "V_VISC_EXPLICIT_OLD"]


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def case():
    from pvof import cases
    return cases.rayleigh_taylor(NXM, NYM, Lx=1.0, Ly=4.0, Cn=0.01, P_CG_MAXIT=2000)


def dist_env():
    from pvof import dist as pdist
    return pdist.env()


def init_dist(ws, local):
    from pvof import dist as pdist
    return pdist.init("nccl")


def max_over_ranks(dist, x):
    from pvof import dist as pdist
    return pdist.max_over_ranks(dist, x, device="cuda")


def barrier(dist):
    if dist is not None:
        import torch
        dist.barrier()
        torch.cuda.synchronize()


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"],
                                 parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(kernel):
    """DRAM bytes per launch of a solver kernel from the committed ncu capture
    (profiles/ncu_traffic.json), or None."""
    try:
        with open(os.path.join(REPO, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
        return float(d[kernel]["dram_bytes_per_launch"])
    except (OSError, KeyError, ValueError, TypeError):
        return None


def reference_timing(steps, timeout=1800, warmup=0):
    """Run the reference build on the bench case, ``warmup`` untimed steps then
    ``steps`` timed ones; (cell-updates/s, seconds, steps)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po  # checker / CPU baseline only
    binary = po.ref_binary("rt2d")
    if not os.path.exists(binary):
        return None
    grid, params, planes = case()
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference("rt2d", wd, grid, params, planes, steps + warmup, DT, 0, timeout=timeout,
                              warmup=warmup)
    for line in cp.stdout.splitlines():
        if line.startswith("REF_TIMING"):
            kv = dict(x.split("=") for x in line.split()[1:])
            secs = float(kv["seconds"])
            cells = int(kv["cells"])
            timed = int(kv["steps"])
            return cells * timed / secs, secs, timed
    return None


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, args.ref_steps))
    r = reference_timing(steps, warmup=max(0, args.warmup))
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/ref_rt2d is missing"}))
        return 0
    value, secs, n = r
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": max(0, args.warmup), "ms_per_step": 1e3 * secs / n, "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": "%dx%d" % (NXM, NYM), "cells": NXM * NYM, "dt": DT},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "%d time steps of the same case after %d untimed ones, single-rank reference "
                                   "build (no MPI on this host), %.1f s" % (n, max(0, args.warmup), secs)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def particle_case(args, device):
    """The workload with surface tension and three resolved cylinders, timed
    like the main line (L2 flushed before every step), and the same case
    without the cylinders.  Device time per step, solver iterations, the
    cylinders' kernel launches per step."""
    from pvof import cases, runtime
    out = {}
    for label, parts, forms in (("without", None, 0), ("with", CYLINDERS, 0), ("with, all forms", CYLINDERS, 1)):
        grid, params, planes = cases.rayleigh_taylor(NXM, NYM, Lx=1.0, Ly=4.0, Cn=0.01, P_CG_MAXIT=2000,
                                                     surface_tension=True, We=100.0)
        params.contact_angle_deg = 70.0
        if forms:
            params.stencil_fp32 = params.pressure_warm_start = 1
            params.pressure_preconditioner = params.velocity_cg_unregularized = 1
        s = runtime.Solver(grid, params, device=device)
        if parts:
            s.set_particles(parts)
        s.set_planes(dict(planes, C_L=planes["F"]))
        s.initialize()
        for _ in range(args.warmup):
            s.run_steps(1, DT)
        s.set_solver_timing(True)
        l0, ms = s.launch_count(), 0.0
        for _ in range(args.steps):
            s.flush_l2()
            s.timer_start()
            s.run_steps(1, DT)
            ms += s.timer_stop()
        out[label] = {"ms_per_step": ms / args.steps, "launches_per_step": (s.launch_count() - l0) / args.steps,
                      "pressure_iterations": s.solver_timing(2)["iterations"],
                      "pressure_ms_per_step": s.solver_timing(2)["ms"] / args.steps}
        s.close()
    w = out["with"]
    return {"case": "the workload with surface tension (We 100), contact angle 70 degrees and three resolved "
                    "cylinders on the interface (two mobile R 0.08, one fixed R 0.1, solid/liquid density 2.5)",
            "value": NXM * NYM / (w["ms_per_step"] * 1e-3), "unit": UNIT, "steps": args.steps,
            "ms_per_step": w["ms_per_step"], "launches_per_step": w["launches_per_step"],
            "pressure_iterations": w["pressure_iterations"], "pressure_ms_per_step": w["pressure_ms_per_step"],
            "without_cylinders": out["without"], "with_all_forms": out["with, all forms"]}


def large_case(args, device):
    """The planar instability on 1024 x 1024 with a density ratio of 1e-3
    (Atwood 0.998, Cn 0.005, dt 2e-5): one untimed step, then --large-steps
    timed steps (device time, L2 flushed) in the plain path, with the spectral
    pressure preconditioner, and with it the unregularised momentum CG."""
    from pvof import cases, runtime
    ratio = 1e-3
    nsteps = max(1, args.large_steps)
    out = {"case": "planar instability 1024x1024, density ratio 1e-3 (Atwood 0.998), Cn 0.005, dt 2e-5",
           "steps": nsteps, "unit": UNIT}
    forms = (("plain", 0, 0), ("spectral", 1, 0), ("spectral + unregularised momentum", 1, 1))
    pick = {"plain": 0, "spectral": 1, "spectral-unreg": 2}
    wanted = [forms[pick[f]] for f in args.large_forms.split(",")]
    for label, precond, vel in wanted:
        grid, params, planes = cases.rayleigh_taylor(1024, 1024, Lx=1.0, Ly=1.0, Cn=0.005,
                                                     atwood=(1 - ratio) / (1 + ratio), P_CG_MAXIT=40000)
        params.pressure_preconditioner = precond
        params.velocity_cg_unregularized = vel
        s = runtime.Solver(grid, params, device=device)
        s.set_planes(planes)
        s.initialize()
        s.run_steps(1, 2e-5)
        ms = 0.0
        for _ in range(nsteps):
            s.flush_l2()
            s.timer_start()
            s.run_steps(1, 2e-5)
            ms += s.timer_stop()
        t, _, _ = solver_timing_pass(s, 1)
        out[label] = {"value": 1024 * 1024 / (ms / nsteps * 1e-3), "ms_per_step": ms / nsteps,
                      "pressure_iterations_per_step": t[2]["iterations"],
                      "pressure_ms_per_step": t[2]["ms"],
                      "pressure_us_per_iteration": 1e3 * t[2]["ms"] / max(1, t[2]["iterations"]),
                      "velocity_iterations_per_step": t[1]["iterations"]}
        s.close()
    if "plain" in out and "spectral + unregularised momentum" in out:
        out["spectral_vs_plain"] = out["spectral + unregularised momentum"]["value"] / out["plain"]["value"]
    return out


def poisson_case(args, device):
    """The reference's variable-density Jacobi-PCG alone
    (pvof_Pressure_solve_cg, psolve_cg.c:130-293) on a grid whose solver
    planes do not fit in L2: the planar instability at --poisson-grid with a
    density ratio of 1e-3 and a seeded random velocity, so that the
    right-hand side of Pressure_set_RHS (the divergence of that velocity over
    the stage's dt) is not small.  Each of --poisson-reps solves starts from
    zero (Pressure_set_RHS resets the correction) after an L2 flush and runs
    --poisson-maxit iterations or to the reference's tolerance, timed by CUDA
    events around the solve; achieved bandwidth counts 56 algorithmic bytes per
    cell and iteration (x, r and the direction read and written, the density
    the coefficients come from)."""
    from pvof import cases, runtime
    nxm, nym = (int(v) for v in args.poisson_grid.lower().split("x"))
    ratio = 1e-3
    grid, params, planes = cases.rayleigh_taylor(nxm, nym, Lx=1.0, Ly=nym / nxm, Cn=0.005,
                                                 atwood=(1 - ratio) / (1 + ratio), velocity_seed=7,
                                                 velocity_amp=0.01, P_CG_MAXIT=args.poisson_maxit)
    s = runtime.Solver(grid, params, device=device)
    s.set_planes(planes)
    s.initialize()
    s.set_stage(0, 1e-4)
    s.set_solver_timing(True)
    ms, iters = 0.0, 0
    for r in range(args.poisson_reps + 1):
        s.call("Pressure_set_RHS")
        s.call("Pressure_compute_preconditioner")
        s.flush_l2()
        s.timer_start()
        it = s.call("Pressure_solve_cg", None)
        t = s.timer_stop()
        if r > 0:   # the first solve warms up
            ms += t
            iters += it
    name = s.solver_kernel(2)
    s.set_solver_timing(False)
    s.close()
    cells = nxm * nym
    peak, peak_kind = measured_peak()
    gbs = ALG_BYTES[2] * cells * iters / (ms * 1e-3) / 1e9
    return {"case": "planar instability %dx%d, density ratio 1e-3, random velocity (seed 7, amplitude 0.01); "
                    "pressure Jacobi-PCG alone from zero, at most %d iterations" % (nxm, nym, args.poisson_maxit),
            "kernel": name, "cells": cells, "solves": args.poisson_reps, "iterations": iters,
            "us_per_iteration": 1e3 * ms / max(iters, 1),
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": gbs / peak, "alg_bytes_per_cell_iter": ALG_BYTES[2]}}


def box_reference(grid_str, steps, timeout=3600):
    """The reference's 3D build (oracle/_ref/ref_rt3d_st) on a smaller box of
    the same case for ``steps`` steps on one host core; (cell-updates/s,
    seconds, cells) or None."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po  # checker / CPU baseline only
    from pvof import cases
    if not os.path.exists(po.ref_binary("rt3d_st")):
        return None
    n = [int(v) for v in grid_str.lower().split("x")]
    grid, params, fields = box_setup(n, 20000)
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference("rt3d_st", wd, grid, params, fields, steps, BOX_DT, 0, timeout=timeout)
    for line in cp.stdout.splitlines():
        if line.startswith("REF_TIMING"):
            kv = dict(x.split("=") for x in line.split()[1:])
            secs = float(kv["seconds"])
            return int(kv["cells"]) * int(kv["steps"]) / secs, secs, int(kv["cells"])
    return None


BOX_DT = 1e-4


def box_setup(n, maxit):
    """The 3D box of the precision form's configuration: x, z periodic, no-slip
    walls in y, side 2 along x with cubic cells, a liquid layer under gas with
    a seeded 16-mode interface (cases.interface_box, seed 3), density ratio
    1e-3, viscosity ratio 1e-2, Re 1000, We 100, Cn 0.005."""
    from pvof import cases
    return cases.interface_box(n[0], n[1], n[2], L=2.0, seed=3, Cn=0.005, rho_ratio=1e-3, mu_ratio=1e-2,
                               Re=1000.0, We=100.0, P_CG_MAXIT=maxit)


def box_case(args, device, with_ref=True):
    """The plain FP64 path in the 3D mode on --box-grid (default 256^3, the
    only configuration whose fields do not fit in L2): --box-warmup untimed
    steps, --box-steps timed steps (device time, L2 flushed before each), one
    more step with per-solver events; the pressure Jacobi-PCG's achieved
    bandwidth counts 56 algorithmic bytes per cell and iteration; the
    reference's 3D build on a --box-ref-grid box for --box-ref-steps steps."""
    import numpy as np
    from pvof import runtime
    n = [int(v) for v in args.box_grid.lower().split("x")]
    grid, params, fields = box_setup(n, args.box_maxit)
    cells = n[0] * n[1] * n[2]
    s = runtime.Solver(grid, params, device=device)
    s.set_fields({k: fields[k] for k in ("F", "U", "V", "W", "P")})
    del fields
    s.initialize()
    m0 = s.liquid_mass()
    s.run_steps(max(0, args.box_warmup), BOX_DT)
    nsteps = max(1, args.box_steps)
    l0, ms = s.launch_count(), 0.0
    for _ in range(nsteps):
        s.flush_l2()
        s.timer_start()
        s.run_steps(1, BOX_DT)
        ms += s.timer_stop()
    launches = s.launch_count() - l0
    s.set_solver_timing(True)
    s.flush_l2()
    s.timer_start()
    st = s.run_steps(1, BOX_DT)
    step_ms = s.timer_stop()
    t = [s.solver_timing(k) for k in range(3)]
    s.set_solver_timing(False)
    m1 = s.liquid_mass()
    clamp = s.clamp_mass_total()
    ref64 = {f: s.get_g_range(f) for f in ("U", "V", "W")} if (args.box_fp32 or args.box_spectral) else None
    peak, peak_kind = measured_peak()
    names = ["biharmonic CG", "velocity PCG (u, v, w)", "pressure Jacobi-PCG"]
    out = {"case": "3D box %s, x and z periodic, no-slip walls in y, liquid layer under gas with a seeded 16-mode "
                   "interface (seed 3), density ratio 1e-3, viscosity ratio 1e-2, Re 1000, We 100, Cn 0.005, "
                   "dt %g, plain FP64" % (args.box_grid, BOX_DT),
           "value": cells * nsteps / (ms * 1e-3), "unit": UNIT, "steps": nsteps, "warmup": args.box_warmup,
           "ms_per_step": ms / nsteps, "launches_per_step": launches / nsteps, "cells": cells,
           "l2": "flushed before every timed step", "timing_step_ms": step_ms,
           "solvers": {names[k]: {"ms": t[k]["ms"], "iterations": t[k]["iterations"],
                                  "us_per_iteration": 1e3 * t[k]["ms"] / max(1, t[k]["iterations"]),
                                  "share": t[k]["ms"] / step_ms} for k in range(3)},
           "last_substep": {"ch_iters": st.ch_iters, "u_iters": st.u_iters, "v_iters": st.v_iters,
                            "w_iters": st.w_iters, "p_iters": st.p_iters, "poisson_passes": st.poisson_passes,
                            "div_max": st.div_max},
           "mass": {"initial": m0, "final": m1, "clamp_total": clamp,
                    "rel_change_net_of_clamp": (m1 - m0 - clamp) / m0}}
    for k, bpc in ((0, ALG_BYTES[0]), (2, ALG_BYTES[2])):
        if t[k]["ms"] > 0:
            gbs = bpc * t[k]["cell_iters"] / (t[k]["ms"] * 1e-3) / 1e9
            out["solvers"][names[k]]["roofline"] = {"bound": "hbm", "achieved": gbs, "peak": peak,
                                                    "peak_kind": peak_kind, "unit": "GB/s", "frac": gbs / peak,
                                                    "alg_bytes_per_cell_iter": bpc}
    s.close()
    if args.box_fp32:
        # the precision form: FP32 stencils from the same start over the same
        # steps, its throughput and its errors against the FP64 path above
        grid, params, fields = box_setup(n, args.box_maxit)
        params.stencil_fp32 = 1
        s32 = runtime.Solver(grid, params, device=device)
        s32.set_fields({k: fields[k] for k in ("F", "U", "V", "W", "P")})
        del fields
        s32.initialize()
        s32.run_steps(max(0, args.box_warmup), BOX_DT)
        ms32 = 0.0
        for _ in range(nsteps):
            s32.flush_l2()
            s32.timer_start()
            s32.run_steps(1, BOX_DT)
            ms32 += s32.timer_stop()
        s32.run_steps(1, BOX_DT)
        num = den = 0.0
        for f in ("U", "V", "W"):
            a, b = s32.get_g_range(f), ref64[f]
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b ** 2))
        m32 = s32.liquid_mass()
        out["fp32_form"] = {"value": cells * nsteps / (ms32 * 1e-3), "ms_per_step": ms32 / nsteps,
                            "velocity_rel_l2_vs_fp64": (num / den) ** 0.5,
                            "volume_rel_error_vs_fp64": abs(m32 - m1) / m1,
                            "steps_compared": max(0, args.box_warmup) + nsteps + 1}
        s32.close()
    if args.box_spectral:
        # the spectral preconditioner form from the same start over the same
        # steps (FP64 throughout), its throughput and its errors against the
        # Jacobi path above
        grid, params, fields = box_setup(n, args.box_maxit)
        params.pressure_preconditioner = 1
        ss = runtime.Solver(grid, params, device=device)
        ss.set_fields({k: fields[k] for k in ("F", "U", "V", "W", "P")})
        del fields
        ss.initialize()
        ss.run_steps(max(0, args.box_warmup), BOX_DT)
        mss = 0.0
        for _ in range(nsteps):
            ss.flush_l2()
            ss.timer_start()
            ss.run_steps(1, BOX_DT)
            mss += ss.timer_stop()
        ss.set_solver_timing(True)
        st_s = ss.run_steps(1, BOX_DT)
        ts = ss.solver_timing(2)
        ss.set_solver_timing(False)
        num = den = 0.0
        for f in ("U", "V", "W"):
            a, b = ss.get_g_range(f), ref64[f]
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b ** 2))
        ms_ = ss.liquid_mass()
        out["spectral_form"] = {"value": cells * nsteps / (mss * 1e-3), "ms_per_step": mss / nsteps,
                                "vs_plain": (cells * nsteps / (mss * 1e-3)) / out["value"],
                                "pressure_iterations_per_step": ts["iterations"],
                                "pressure_us_per_iteration": 1e3 * ts["ms"] / max(1, ts["iterations"]),
                                "last_substep_p_iters": st_s.p_iters,
                                "velocity_rel_l2_vs_jacobi": (num / den) ** 0.5,
                                "volume_rel_error_vs_jacobi": abs(ms_ - m1) / m1}
        ss.close()
    if args.box_ref_steps > 0 and with_ref:
        r = box_reference(args.box_ref_grid, args.box_ref_steps)
        if r is not None:
            out["cpu_reference"] = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": "%d time step(s) of the same case on a %s box (%d cells) by the "
                                              "single-rank 3D reference build, %.1f s" % (args.box_ref_steps,
                                                                                       args.box_ref_grid, r[2], r[1])}
            out["vs_cpu_reference"] = out["value"] / r[0]
    return out


# the axisymmetric benchmark case: a bubble (R 0.5 at z = 1) rising towards a
# fixed sphere (R 0.25 at z = 2.5) on the axis, 256 x 512 cells over
# r in [0, 2], z in [0, 4]
AXI_SPHERE = [(0, 0.0, 2.5, 0.25, 0, 0, 0, 2.5)]
AXI_DT = 1e-4


def axisym_setup():
    from pvof import cases
    grid, params, planes = cases.rising_bubble(NXM=256, NYM=512, rmax=2.0, zmax=4.0, radius=0.5, zc=1.0, Cn=0.01,
                                               rho_ratio=1e-3, mu_ratio=1e-2, Re=100.0, surface_tension=True,
                                               We=200.0, P_CG_MAXIT=40000)
    params.contact_angle_deg = 90.0
    return grid, params, planes


def axisym_reference(steps, timeout=3600):
    """The reference build with AXISYM_RZ and resolved particles
    (oracle/_ref/ref_ibm_axi_st) on the axisymmetric case for ``steps``
    steps on the host; (cell-updates/s, seconds) or None."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po  # checker / CPU baseline only
    if not os.path.exists(po.ref_binary("ibm_axi_st")):
        return None
    grid, params, planes = axisym_setup()
    fixed = [p[1:7] for p in AXI_SPHERE if not p[0]]
    mobile = [p[1:7] for p in AXI_SPHERE if p[0]]
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, AXI_DT, 0, case="ibm_axi_st",
                                  mode="steps", nsteps=steps, timeout=timeout)
    for line in cp.stdout.splitlines():
        if line.startswith("REF_TIMING"):
            kv = dict(x.split("=") for x in line.split()[1:])
            secs = float(kv["seconds"])
            return int(kv["cells"]) * int(kv["steps"]) / secs, secs
    return None


def axisym_case(args, device):
    """The axisymmetric bubble-and-sphere case (density ratio 1e-3, viscosity
    ratio 1e-2, Re 100, We 200, Cn 0.01, contact angle 90 degrees):
    --axisym-warmup untimed steps, then --axisym-steps timed steps replayed
    from CUDA graphs (device time, L2 flushed), one more step launch by launch
    for the solver counts, and the reference build on the host for
    --axisym-ref-steps steps."""
    from pvof import runtime
    grid, params, planes = axisym_setup()
    cells = grid.NXM * grid.NYM
    s = runtime.Solver(grid, params, device=device)
    s.set_particles(AXI_SPHERE)
    s.set_planes(dict(planes, C_L=planes["F"]))
    s.initialize()
    # untimed steps first: a substep replays from a CUDA graph (the sphere's
    # bookkeeping included) from the third time its launches recur
    s.run_steps(max(1, args.axisym_warmup), AXI_DT)
    nsteps = max(1, args.axisym_steps)
    l0, r0, ms = s.launch_count(), s.graph_replays(), 0.0
    for _ in range(nsteps):
        s.flush_l2()
        s.timer_start()
        s.run_steps(1, AXI_DT)
        ms += s.timer_stop()
    replays = s.graph_replays() - r0
    launches = s.launch_count() - l0
    timing, _, _ = solver_timing_pass(s, 1)   # one more step, launch by launch, for the solver counts
    t = timing[2]
    out = {"case": "axisymmetric bubble (R 0.5, z 1) below a fixed sphere on the axis (R 0.25, z 2.5), 256x512, "
                   "r in [0,2], z in [0,4], density ratio 1e-3, viscosity ratio 1e-2, Re 100, We 200, Cn 0.01, "
                   "contact angle 90 degrees, dt 1e-4",
           "value": cells * nsteps / (ms * 1e-3), "unit": UNIT, "steps": nsteps, "ms_per_step": ms / nsteps,
           "launches_per_step": launches / nsteps, "graph_replayed_substeps": "%d of %d" % (replays, 3 * nsteps),
           "pressure_iterations_per_step": t["iterations"], "pressure_ms_per_step": t["ms"],
           "pressure_kernel": s.solver_kernel(2)}
    s.close()
    if args.axisym_ref_steps > 0:
        r = axisym_reference(args.axisym_ref_steps)
        if r is not None:
            out["cpu_reference"] = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": "%d time steps of the same case (after the start-up) by the "
                                              "single-rank reference build with AXISYM_RZ and resolved "
                                              "particles, %.1f s" % (args.axisym_ref_steps, r[1])}
            out["vs_cpu_reference"] = out["value"] / r[0]
    return out


def learned_case(args, device):
    """The learned warm start on its benchmark case: three mobile cylinders
    (R 0.1, solid density 2.5, contact angle 110 degrees) on a flat
    interface, 1024 x 1024, density ratio 1e-3, Jacobi-PCG pressure solve.
    The network is trained on random 64 x 64 crops of the solver's own
    samples (the same-stage warm start's run), then the case is advanced with
    a cold start, the same-stage warm start and the learned one: pressure
    iterations and device time per step of --learned-steps steps after two
    (which fill the kept corrections)."""
    import numpy as np
    from pvof import cases, cnn, runtime
    dt = 2e-5
    grid, params, planes, parts = cases.sinking_cylinders(P_CG_MAXIT=40000)
    planes_cl = dict(planes, C_L=planes["F"])
    t0 = time.time()
    nplanes = 3 * (args.learned_sample_steps - 2)
    per_plane = max(1, -(-args.learned_samples // max(nplanes, 1)))
    samples = cnn.generate_crop_samples(grid, params, planes, parts, args.learned_sample_steps, dt, 64, per_plane,
                                        device=device)
    t_samples = time.time() - t0
    t0 = time.time()
    net, hist = cnn.train(samples, 64, 64, epochs=args.learned_epochs, batch=32, lr=1e-3, device=device)
    loss, base = net.evaluate(samples[: min(len(samples), 2000)])
    t_train = time.time() - t0
    P = net.params()
    del samples, net
    out = {"case": "planar 1024x1024, x periodic, three mobile cylinders (R 0.1, rho_s 2.5, contact angle 110 deg) "
                   "on a flat interface at y 0.6, density ratio 1e-3, We 100, Re 100, Cn 0.005, dt 2e-5, "
                   "Jacobi-PCG pressure solve to the reference's absolute tolerance 1e-7",
           "network": {"crops": nplanes * per_plane, "crop": "64x64", "epochs": args.learned_epochs,
                       "loss": loss, "loss_predicting_no_change": base, "sampling_s": t_samples,
                       "training_s": t_train},
           "steps": args.learned_steps}
    fields = {}
    for label, warm in (("cold", 0), ("same_stage", 1), ("learned", 2)):
        from pvof import abi
        p = abi.Params.from_buffer_copy(params)
        p.pressure_warm_start = warm
        s = runtime.Solver(grid, p, device=device)
        s.set_particles(parts)
        if warm == 2:
            s.set_pressure_network(P)
        s.set_planes(planes_cl)
        s.initialize()
        iters = 0
        for n in range(2 + args.learned_steps):
            timed = n >= 2
            if timed and n == 2:
                ms = 0.0
            if timed:
                s.flush_l2()
                s.timer_start()
            for rk in range(3):
                if n > 0 and rk == 0:
                    s.call("Velocity_cell_center")
                s.set_stage(rk, dt)
                st = s.substep()
                if timed:
                    iters += st.p_iters_total
            if timed:
                ms += s.timer_stop()
        out[label] = {"pressure_iterations": iters, "ms_per_step": ms / args.learned_steps}
        fields[label] = {f: s.get(f) for f in ("U", "V", "P")}
        s.close()
    for label in ("same_stage", "learned"):
        out[label]["velocity_rel_l2_vs_cold"] = max(
            float(np.linalg.norm(fields[label][f] - fields["cold"][f]) / np.linalg.norm(fields["cold"][f]))
            for f in ("U", "V"))
    out["learned_vs_cold_iterations"] = out["learned"]["pressure_iterations"] / max(1, out["cold"]["pressure_iterations"])
    out["learned_vs_same_stage_iterations"] = (out["learned"]["pressure_iterations"] /
                                              max(1, out["same_stage"]["pressure_iterations"]))
    return out


# uneven batch: the planar instability at four sizes, two cases each
MIXED_SIZES = [(64, 128), (64, 128), (128, 256), (128, 256), (256, 512), (256, 512), (512, 1024), (512, 1024)]


def mixed_batch(args, device):
    """Cases of uneven size (MIXED_SIZES, domain 1 x 2, Cn 2 / NXM) in all
    four forms, advanced concurrently by pvof_run_steps_batched, against the
    same cases advanced one after another; device time, L2 flushed first."""
    from pvof import cases, runtime
    nsteps = max(1, min(args.steps, args.batch_steps))

    def make():
        out = []
        for nx, ny in MIXED_SIZES:
            grid, params, planes = cases.rayleigh_taylor(nx, ny, Lx=1.0, Ly=2.0, Cn=2.0 / nx, P_CG_MAXIT=4000)
            params.stencil_fp32 = params.pressure_warm_start = 1
            params.pressure_preconditioner = params.velocity_cg_unregularized = 1
            s = runtime.Solver(grid, params, device=device)
            s.set_planes(planes)
            s.initialize()
            out.append(s)
        return out

    cells = sum(nx * ny for nx, ny in MIXED_SIZES)
    reps = make()
    runtime.run_steps_batched(reps, 2, DT)
    for r in reps:
        r.flush_l2()
    for r in reps:
        r.timer_start()
    runtime.run_steps_batched(reps, nsteps, DT)
    span = max(r.timer_stop() for r in reps)
    seq_ms = 0.0
    for r in reps:   # the same cases one after another
        r.flush_l2()
        r.timer_start()
        r.run_steps(nsteps, DT)
        seq_ms += r.timer_stop()
    for r in reps:
        r.close()
    return {"cases": ["%dx%d" % sz for sz in MIXED_SIZES], "cells": cells, "steps": nsteps,
            "form": "fp32-stencils + pressure warm start + spectral pressure preconditioner + unregularised momentum CG",
            "value": cells * nsteps / (span * 1e-3), "unit": UNIT, "ms_per_step": span / nsteps,
            "sequential_value": cells * nsteps / (seq_ms * 1e-3),
            "vs_sequential": seq_ms / span}


DROP_DT = 1e-4


def droplet_reference(case, steps, timeout=1800):
    """The reference build with resolved particles and surface tension
    (oracle/_ref/ref_ibm2d_st) on one droplet case for ``steps`` steps on the
    host; (cell-updates/s, seconds) or None."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po  # checker / CPU baseline only
    if not os.path.exists(po.ref_binary("ibm2d_st")):
        return None
    grid, params, planes, parts = case
    fixed = [p[1:7] for p in parts if not p[0]]
    mobile = [p[1:7] for p in parts if p[0]]
    with tempfile.TemporaryDirectory() as wd:
        cp = po.run_reference_ibm(wd, grid, params, planes, fixed, mobile, DROP_DT, 0, case="ibm2d_st",
                                  mode="steps", nsteps=steps, timeout=timeout)
    for line in cp.stdout.splitlines():
        if line.startswith("REF_TIMING"):
            kv = dict(x.split("=") for x in line.split()[1:])
            secs = float(kv["seconds"])
            return int(kv["cells"]) * int(kv["steps"]) / secs, secs
    return None


def droplet_batch(args, dist, device, ws, rank):
    """The batching form's workload: --droplets seeded sessile droplets on
    static cylinders (pvof.cases.droplet_batch: grids log-uniform from 64x128
    to 512x1024 on the widths 2^a, 3 2^a, 5 2^a, droplet radius U(0.3,0.6),
    cylinder radius U(0.2,0.4), contact angle U(30,150) degrees, density
    ratio 1e-3, Cn 0.01) in all four forms (FP32 stencils, warm start,
    spectral preconditioner, unregularised momentum CG).  The cases are split over the
    ranks by cell count (pvof.dist.run_sharded_batch, no collective on the
    data path); each rank advances its shard concurrently with
    pvof_run_steps_batched, every substep replayed from CUDA graphs, timed by
    the host clock (max over ranks).  Rank 0 also runs the two smallest cases
    in the plain FP64 path for the forms' error and times the reference on the
    smallest."""
    from pvof import cases, runtime
    from pvof import dist as pdist
    kw = dict(P_CG_MAXIT=20000, stencil_fp32=1, pressure_warm_start=1, pressure_preconditioner=1,
              velocity_cg_unregularized=1)
    allc = cases.droplet_batch(args.droplets, seed=args.droplet_seed, **kw)
    costs = [float(g.NXM * g.NYM) for g, _, _, _ in allc]
    nsteps = max(1, min(args.steps, args.droplet_steps))

    def start(case):
        g, p, pl, parts = case
        s = runtime.Solver(g, p, device=device)
        s.set_particles(parts)
        s.set_planes(dict(pl, C_L=pl["F"]))
        s.initialize()
        return s

    def run_batch(idx, cases_=None):
        cases_ = allc if cases_ is None else cases_
        solvers = [start(cases_[q]) for q in idx]
        # stencil tiles: each case tuned alone on the GPU (launch times taken
        # while other cases run would include their waits), a few steps each
        for s in solvers:
            s.set_autotune(True)
            for _ in range(8):
                if not s.autotune_active():
                    break
                s.run_steps(1, DROP_DT)
        if solvers:
            runtime.run_steps_batched(solvers, max(1, args.droplet_warmup), DROP_DT)
        m0 = [s.liquid_mass() for s in solvers]
        c0 = [s.clamp_mass_total() for s in solvers]
        r0 = [s.graph_replays() for s in solvers]
        barrier(dist)
        t0 = time.perf_counter()
        if solvers:
            runtime.run_steps_batched(solvers, nsteps, DROP_DT)
        secs = time.perf_counter() - t0
        res = {}
        for q, s, m, c, r in zip(idx, solvers, m0, c0, r0):
            rep = s.autotune_report()
            res[q] = {"grid": "%dx%d" % (allc[q][0].NXM, allc[q][0].NYM),
                      "volume_change": (s.liquid_mass() - m) / m, "clamp_change": (s.clamp_mass_total() - c) / m,
                      "graph_replays": s.graph_replays() - r, "substeps": 3 * nsteps,
                      "tuned": sum(1 for e in rep if e["decided"]), "tunable": len(rep),
                      "tiles": {e["kernel"]: [e["tile"], round(e["best_us"], 2), round(e["default_us"], 2)]
                                for e in rep}}
            s.close()
        return res, secs

    merged, shard, secs = pdist.run_sharded_batch(dist, costs, run_batch, device="cuda")
    cells = int(sum(costs))
    plain = None
    if args.droplet_plain:   # the same cases in the plain FP64 path (no form), timed the same way
        plain_cases = cases.droplet_batch(args.droplets, seed=args.droplet_seed, P_CG_MAXIT=20000)
        _, _, psecs = pdist.run_sharded_batch(dist, costs, lambda idx: run_batch(idx, plain_cases), device="cuda")
        plain = {"value": cells * nsteps / psecs, "seconds": psecs,
                 "form": "plain FP64 (the reference's solvers), same tuning, warm-up and graph replay"}
    out = {"cases": len(allc), "cells": cells, "steps": nsteps, "warmup_steps": max(1, args.droplet_warmup),
           "dt": DROP_DT, "value": cells * nsteps / secs, "unit": UNIT, "seconds": secs,
           "clock": "host wall clock around pvof_run_steps_batched, max over ranks",
           "form": "all four forms: fp32 stencils, same-stage pressure warm start, spectral pressure "
                   "preconditioner, unregularised momentum CG (solves and reductions in FP64)",
           "sharding": "%d rank(s), cases split by cell count" % ws,
           "graph_replayed_substeps": sum(v["graph_replays"] for v in merged.values()),
           "substeps": sum(v["substeps"] for v in merged.values()),
           "max_abs_volume_change_net_of_clamp": max(abs(v["volume_change"] - v["clamp_change"])
                                                     for v in merged.values()),
           "grids": {"min": min(merged.values(), key=lambda v: int(v["grid"].split("x")[0]))["grid"],
                     "max": max(merged.values(), key=lambda v: int(v["grid"].split("x")[0]))["grid"]},
           "autotune": {"kernels_decided": sum(v["tuned"] for v in merged.values()),
                        "kernels_met": sum(v["tunable"] for v in merged.values()),
                        "note": "stencil tile per kernel and case, picked by the autotuner (pvof_set_autotune) with "
                                "the case alone on the GPU before the warm-up; kernel: [tile, mean us there, mean us "
                                "at the default 32x8]",
                        "smallest_case": merged[min(merged, key=lambda q: (costs[q], q))]["tiles"],
                        "largest_case": merged[max(merged, key=lambda q: (costs[q], q))]["tiles"]}}
    if plain is not None:
        out["plain"] = plain
        out["vs_plain"] = out["value"] / plain["value"]
    if rank == 0:
        small = sorted(range(len(allc)), key=lambda q: (costs[q], q))[:2]
        errs = []
        for q in small:
            st = {}
            for fp32 in (0, 1):
                forms = dict(stencil_fp32=fp32, pressure_warm_start=fp32, pressure_preconditioner=fp32,
                             velocity_cg_unregularized=fp32)
                g, p, pl, parts = cases.droplet_batch(args.droplets, seed=args.droplet_seed, **dict(kw, **forms))[q]
                s = start((g, p, pl, parts))
                s.run_steps(max(1, args.droplet_warmup) + nsteps, DROP_DT)
                st[fp32] = ({f: s.get(f) for f in ("U", "V")}, s.liquid_mass())
                s.close()
            import numpy as np
            vel = max(float(np.linalg.norm(st[1][0][f] - st[0][0][f]) / max(np.linalg.norm(st[0][0][f]), 1e-300))
                      for f in ("U", "V"))
            errs.append({"grid": "%dx%d" % (allc[q][0].NXM, allc[q][0].NYM), "velocity_rel_l2": vel,
                         "volume_rel": abs(st[1][1] - st[0][1]) / st[0][1]})
        out["error_vs_fp64"] = errs
        if args.droplet_ref_steps > 0:
            q = small[0]
            r = droplet_reference(cases.droplet_batch(args.droplets, seed=args.droplet_seed)[q],
                                  args.droplet_ref_steps)
            if r is not None:
                out["cpu_reference"] = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference",
                                        "sample": "%d time step(s) of the smallest case (%dx%d) by the single-rank "
                                                  "reference build with resolved particles and surface tension, "
                                                  "%.1f s" % (args.droplet_ref_steps, allc[q][0].NXM, allc[q][0].NYM,
                                                              r[1])}
    return out


def pinned_like(n):
    import torch
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()


def solver_timing_pass(g, nsteps):
    """nsteps more steps with CUDA events around every solver launch: per
    solver {ms, iterations, ...}, its kernel names, the steps' device time."""
    g.set_solver_timing(True)
    ms = 0.0
    for _ in range(nsteps):
        g.flush_l2()
        g.timer_start()
        g.run_steps(1, DT)
        ms += g.timer_stop()
    timing = {k: g.solver_timing(k) for k in (0, 1, 2)}
    names = {k: g.solver_kernel(k) for k in (0, 1, 2)}
    g.set_solver_timing(False)
    return timing, names, ms


def time_forms(args, snap, m64, grid, params, planes, device, cells, value, timing, tsteps):
    """The workload in each form of FORMS, timed like the main line, with its
    error against the plain path's state after the same steps (snap, m64);
    solver iterations and pressure time from a following per-solver timing
    pass of tsteps steps, like the plain path's (timing)."""
    from pvof import abi, cnn, runtime
    import numpy as np
    forms = []
    net_params, net_info = None, None
    for label, fp32, warm, precond, vel in FORMS:
        fparams = abi.Params.from_buffer_copy(params)
        fparams.stencil_fp32 = fp32
        fparams.pressure_warm_start = warm
        fparams.pressure_preconditioner = precond
        fparams.velocity_cg_unregularized = vel
        if warm == 2 and net_params is None:
            # samples from the solver on this workload, then training on the device
            t0 = time.time()
            samples = cnn.generate_samples(grid, params, planes, LEARNED_SAMPLE_STEPS, DT, device=device)
            net, hist = cnn.train(samples, grid.NYM, grid.NXM, epochs=LEARNED_EPOCHS, batch=6, lr=2e-3,
                                  device=device)
            loss, base = net.evaluate(samples)
            net_params = net.params()
            net_info = {"samples": len(samples), "epochs": LEARNED_EPOCHS, "loss": loss, "loss_predicting_no_change": base,
                        "training_s": time.time() - t0}
            del samples, net
        fg = runtime.Solver(grid, fparams, device=device)
        if warm == 2:
            fg.set_pressure_network(net_params)
        fg.set_planes(planes)
        fg.initialize()
        for _ in range(args.warmup):
            fg.run_steps(1, DT)
        f_ms = 0.0
        for _ in range(args.steps):
            fg.flush_l2()
            fg.timer_start()
            fg.run_steps(1, DT)
            f_ms += fg.timer_stop()
        err = {"velocity_rel_l2": max(float(np.linalg.norm(fg.get(f) - snap[f]) / np.linalg.norm(snap[f]))
                                      for f in ("U", "V")),
               "pressure_rel_l2": float(np.linalg.norm(fg.get("P") - snap["P"]) / np.linalg.norm(snap["P"])),
               "volume_rel": abs(fg.liquid_mass() - m64) / abs(m64)}
        fvalue = cells * args.steps / (f_ms * 1e-3)
        ft, _, _ = solver_timing_pass(fg, tsteps)
        forms.append({"form": label, "value": fvalue, "unit": UNIT, "ms_per_step": f_ms / args.steps,
                      "vs_plain": fvalue / value,
                      "solver_timing_steps": tsteps,
                      "pressure_iterations": ft[2]["iterations"],
                      "pressure_iterations_plain": timing[2]["iterations"],
                      "pressure_ms_per_step": ft[2]["ms"] / tsteps,
                      "velocity_iterations": ft[1]["iterations"],
                      "velocity_iterations_plain": timing[1]["iterations"],
                      "error_vs_fp64": err})
        if warm == 2:
            forms[-1]["network"] = net_info
        fg.close()
    return forms


def time_batched(args, grid, params, planes, device, cells, total_ms):
    """K replicas of the workload advanced concurrently in the chosen form."""
    from pvof import runtime
    from pvof import abi
    bparams = abi.Params.from_buffer_copy(params)
    bparams.stencil_fp32 = 1 if args.batch_form.startswith("fp32") or args.batch_form == "all" else 0
    bparams.pressure_warm_start = 1 if args.batch_form in ("fp32-warm", "fp32-warm-spectral", "all") else 0
    bparams.pressure_preconditioner = 1 if args.batch_form in ("spectral", "fp32-warm-spectral", "all") else 0
    bparams.velocity_cg_unregularized = 1 if args.batch_form == "all" else 0
    reps = []
    for q in range(args.batch_cases):
        r = runtime.Solver(grid, bparams, device=device)
        r.set_planes(planes)
        r.initialize()
        reps.append(r)
    runtime.run_steps_batched(reps, 1, DT)
    bsteps = max(1, min(args.steps, args.batch_steps))
    for r in reps:
        r.flush_l2()
    for r in reps:
        r.timer_start()
    runtime.run_steps_batched(reps, bsteps, DT)
    span = max(r.timer_stop() for r in reps)
    bvalue = args.batch_cases * cells * bsteps / (span * 1e-3)
    batched = {"cases": args.batch_cases, "steps": bsteps, "value": bvalue, "unit": UNIT,
               "ms_per_step": span / bsteps, "vs_single": bvalue / (cells * args.steps / (total_ms * 1e-3)),
               "note": "replicas of the workload advanced concurrently by pvof_run_steps_batched "
                       "(one host thread and stream per case); device time of the slowest case",
               "form": {"fp64": "fp64", "fp32": "fp32-stencils",
                        "fp32-warm": "fp32-stencils + pressure warm start",
                        "spectral": "spectral pressure preconditioner",
                        "fp32-warm-spectral": "fp32-stencils + pressure warm start + spectral pressure "
                                              "preconditioner",
                        "all": "fp32-stencils + pressure warm start + spectral pressure preconditioner + "
                               "unregularised momentum CG"}[args.batch_form]}
    if args.batch_form != "fp64":
        import numpy as np
        # the error of the form: one replica against the FP64 path after the same steps
        ref = runtime.Solver(grid, params, device=device)
        ref.set_planes(planes)
        ref.initialize()
        ref.run_steps(1 + bsteps, DT)
        vel = max(float(np.linalg.norm(reps[0].get(f) - ref.get(f)) / np.linalg.norm(ref.get(f)))
                  for f in ("U", "V"))
        m64 = ref.liquid_mass()
        batched["error_vs_fp64"] = {"velocity_rel_l2": vel,
                                    "volume_rel": abs(reps[0].liquid_mass() - m64) / abs(m64)}
        ref.close()
    for r in reps:
        r.close()

    return batched


def run_ours(args):
    ws, rank, local = dist_env()
    dist = init_dist(ws, local)
    from pvof import abi, cases, runtime
    grid, params, planes = case()
    cells = NXM * NYM
    g = runtime.Solver(grid, params, device=local)
    g.set_planes(planes)
    g.initialize()
    log("rank %d: warmup %d steps" % (rank, args.warmup))
    for _ in range(args.warmup):
        g.run_steps(1, DT)
    g.synchronize()
    # the state at the start of the timed steps: the end-to-end pass below
    # replays the same steps from it, through host buffers
    start_blocks = {f: pinned_like(g.block_count(f)) for f in STATE_FIELDS}
    for f in STATE_FIELDS:
        g.download(f, out=start_blocks[f])

    # ---- device-resident timing (substeps replayed from CUDA graphs) --------
    clocks = Clocks(local)
    barrier(dist)
    l0 = g.launch_count()
    clamp0, mass0 = g.clamp_mass_total(), g.liquid_mass()
    clocks.start()
    wall0 = time.time()
    total_ms = 0.0
    for _ in range(args.steps):
        g.flush_l2()
        g.timer_start()
        g.run_steps(1, DT)
        total_ms += g.timer_stop()
    wall = time.time() - wall0
    clk = clocks.stop()
    barrier(dist)
    launches = g.launch_count() - l0
    graph_steps = g.graph_replays()
    t_max = max_over_ranks(dist, total_ms)
    value = ws * cells * args.steps / (t_max * 1e-3)
    snap = {f: g.get(f) for f in ("U", "V", "P", "C_L")}   # the forms' reference state
    m64 = g.liquid_mass()
    # liquid volume over the timed steps: the change the C_L clamp made (the
    # only non-conservative operation of the substep) and the total change
    mass_report = {"clamp_mass_timed_steps": g.clamp_mass_total() - clamp0, "liquid_mass_change": m64 - mass0,
                   "liquid_mass": mass0}

    # ---- end to end through the C ABI with host buffers: the timed steps
    # again, from the state they started from (same iterations, same work),
    # the state uploaded before and downloaded after every step ----------------
    blocks = start_blocks
    h2d = d2h = 0
    NX, NY, NZ = cases.dims(grid)
    plane_flow = (NX + 6) * (NY + 6) * 8
    plane_ng = NX * NY * 8
    for f in STATE_FIELDS:
        ng = abi.FIELD[f] in abi.NG_FIELDS
        h2d += plane_ng if ng else plane_flow
        d2h += (plane_ng if ng else plane_flow) * NZ
    e2e_steps = max(1, min(args.steps, args.e2e_steps or args.steps))
    barrier(dist)
    e2e_ms = 0.0
    g.synchronize()
    host0 = time.perf_counter()
    for _ in range(e2e_steps):
        g.timer_start()
        for f in STATE_FIELDS:
            g.upload(f, blocks[f])
        g.run_steps(1, DT)
        for f in STATE_FIELDS:
            g.download(f, out=blocks[f])
        e2e_ms += g.timer_stop()
    # the downloads are synchronous: the host holds every step's state when
    # its call returns, so the host clock here is what a caller observes
    e2e_host_ms = (time.perf_counter() - host0) * 1e3
    barrier(dist)
    e2e_max = max_over_ranks(dist, e2e_host_ms)
    e2e_device_max = max_over_ranks(dist, e2e_ms)
    e2e_value = ws * cells * e2e_steps / (e2e_max * 1e-3)

    # ---- per-solver timing: the next steps launch by launch, CUDA events
    # around every solver launch (for the roofline and the solver shares) ----
    tsteps = max(1, min(args.steps, args.timing_steps))
    timing, names, ts_ms = solver_timing_pass(g, tsteps)

    # ---- the chosen forms on the same workload (a failure here keeps the line) ----
    forms = None
    if args.forms:
        try:
            forms = time_forms(args, snap, m64, grid, params, planes, local, cells, value, timing, tsteps)
        except Exception as e:   # noqa: BLE001 -- reported in the line, the plain numbers stand
            forms = {"error": "%s: %s" % (type(e).__name__, e)}

    # ---- roofline of the dominant kernel ----------------------------------
    dom = max(timing, key=lambda k: timing[k]["ms"])
    t = timing[dom]
    peak, peak_kind = measured_peak()
    achieved = ALG_BYTES[dom] * t["cell_iters"] / (t["ms"] * 1e-3) / 1e9 if t["ms"] > 0 else 0.0
    traffic = profile_traffic(names[dom])
    shares = {names[k]: round(timing[k]["ms"] / ts_ms, 4) for k in timing}

    # ---- batched form: K replicas advanced concurrently (a failure keeps the line) ----
    batched = None
    if args.batch_cases > 1:
        try:
            batched = time_batched(args, grid, params, planes, local, cells, total_ms)
        except Exception as e:   # noqa: BLE001
            batched = {"error": "%s: %s" % (type(e).__name__, e)}

    particles = particle_case(args, local) if args.particles else None
    mixed = None
    if args.batch_mixed:
        try:
            mixed = mixed_batch(args, local)
        except Exception as e:   # noqa: BLE001
            mixed = {"error": "%s: %s" % (type(e).__name__, e)}
    learned = None
    if args.learned:
        try:
            learned = learned_case(args, local)
        except Exception as e:   # noqa: BLE001
            learned = {"error": "%s: %s" % (type(e).__name__, e)}
    axisym = None
    if args.axisym:
        try:
            axisym = axisym_case(args, local)
        except Exception as e:   # noqa: BLE001
            axisym = {"error": "%s: %s" % (type(e).__name__, e)}
    droplets = None
    if args.droplets > 0:
        try:
            droplets = droplet_batch(args, dist, local, ws, rank)
        except Exception as e:   # noqa: BLE001
            droplets = {"error": "%s: %s" % (type(e).__name__, e)}
    poisson = None
    if args.poisson:
        try:
            poisson = poisson_case(args, local)
        except Exception as e:   # noqa: BLE001
            poisson = {"error": "%s: %s" % (type(e).__name__, e)}
    box = None
    if args.box:
        try:
            box = box_case(args, local, with_ref=(rank == 0 and ws == 1))
        except Exception as e:   # noqa: BLE001
            box = {"error": "%s: %s" % (type(e).__name__, e)}
    large = None
    if args.large:
        try:
            large = large_case(args, local)
        except Exception as e:   # noqa: BLE001
            large = {"error": "%s: %s" % (type(e).__name__, e)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        r = reference_timing(args.cpu_steps)
        if r is not None:
            v, secs, n = r
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "%d time steps of the same 128x512 case by the single-rank reference build, %.1f s"
                             % (n, secs)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": "%dx%d" % (NXM, NYM), "cells": cells, "dt": DT,
                       "parallelism": "replicas" if ws > 1 else "single",
                       "l2": "flushed before every timed step (memset of 2x L2, outside the timed intervals)",
                       "solver_iterations": {names[k]: timing[k]["iterations"] for k in timing},
                       "solver_time_share": shares,
                       "solver_timing_steps": tsteps,
                       "graphs": "substeps replayed from CUDA graphs in the timed steps: %d of %d"
                                 % (graph_steps, 3 * (args.warmup + args.steps))},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "clock": "host wall clock around the C ABI calls",
                    "ms_per_step": e2e_max / e2e_steps, "device_ms_per_step": e2e_device_max / e2e_steps},
            "gpu_launches": launches,
            "mass": mass_report,
            "roofline": {"kernel": names[dom], "bound": "hbm", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_cell_iter": ALG_BYTES[dom],
                         "avg_launch_ms": t["ms"] / max(t["launches"], 1)},
            "clocks": clk,
            "wall_s": wall,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if batched is not None:
            line["batched"] = batched
        if forms is not None:
            line["forms"] = forms
        if particles is not None:
            line["particles"] = particles
        if large is not None:
            line["large"] = large
        if axisym is not None:
            line["axisym"] = axisym
        if box is not None:
            line["box"] = box
        if poisson is not None:
            line["poisson"] = poisson
        if learned is not None:
            line["learned"] = learned
        if mixed is not None:
            line["batched_mixed"] = mixed
        if droplets is not None:
            line["batched_droplets"] = droplets
        print(json.dumps(line))
    g.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the end-to-end pass (0: --steps, the same steps)")
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--ref-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-cases", type=int, default=6,
                    help="also time this many replicas advanced concurrently (batched form; 0: off)")
    ap.add_argument("--batch-steps", type=int, default=10)
    ap.add_argument("--timing-steps", type=int, default=20,
                    help="steps of the per-solver timing pass after the timed steps")
    ap.add_argument("--droplets", type=int, default=64,
                    help="also time this many seeded droplet-on-cylinder cases (the batching form's workload: 64; "
                         "0: off), split over the ranks and advanced concurrently")
    ap.add_argument("--droplet-steps", type=int, default=3)
    ap.add_argument("--droplet-warmup", type=int, default=6,
                    help="untimed concurrent steps after the cases' tile tuning: a substep replays from a CUDA graph "
                         "from the third time its launches recur (stage x surface-tension buffer parity x warm "
                         "start: about six steps)")
    ap.add_argument("--droplet-seed", type=int, default=0)
    ap.add_argument("--no-droplet-plain", dest="droplet_plain", action="store_false",
                    help="skip timing the droplet cases in the plain FP64 path")
    ap.add_argument("--droplet-ref-steps", type=int, default=1,
                    help="steps of the reference build on the smallest droplet case (0: off)")
    ap.add_argument("--batch-mixed", action="store_true",
                    help="also time eight cases of four sizes (64x128 .. 512x1024) in all forms, batched")
    ap.add_argument("--large", action="store_true",
                    help="also time 1024x1024 at density ratio 1e-3 (plain, spectral, spectral + momentum form)")
    ap.add_argument("--axisym-warmup", type=int, default=6)
    ap.add_argument("--large-steps", type=int, default=3)
    ap.add_argument("--large-forms", default="plain,spectral,spectral-unreg",
                    help="comma-separated forms of --large: plain, spectral, spectral-unreg")
    ap.add_argument("--poisson", action="store_true",
                    help="also time the reference's pressure Jacobi-PCG alone on --poisson-grid (default 2048x2048, "
                         "solver planes larger than L2) against the HBM roofline")
    ap.add_argument("--poisson-grid", default="2048x2048")
    ap.add_argument("--poisson-maxit", type=int, default=3000)
    ap.add_argument("--poisson-reps", type=int, default=3)
    ap.add_argument("--no-box", dest="box", action="store_false",
                    help="leave out the 3D mode on --box-grid (the precision form's 256^3 box; timed by default)")
    ap.add_argument("--box-grid", default="256x256x256")
    ap.add_argument("--box-steps", type=int, default=2)
    ap.add_argument("--box-warmup", type=int, default=1)
    ap.add_argument("--box-maxit", type=int, default=20000)
    ap.add_argument("--no-box-fp32", dest="box_fp32", action="store_false",
                    help="leave out the FP32 stencil form of the 3D box (from the same start, with its errors "
                         "against FP64)")
    ap.add_argument("--no-box-spectral", dest="box_spectral", action="store_false",
                    help="leave out the 3D box with the spectral pressure preconditioner")
    ap.add_argument("--box-ref-grid", default="64x64x64")
    ap.add_argument("--box-ref-steps", type=int, default=1)
    ap.add_argument("--axisym", action="store_true",
                    help="also time the axisymmetric bubble-and-sphere case (256x512) and the reference on it")
    ap.add_argument("--axisym-steps", type=int, default=10)
    ap.add_argument("--axisym-ref-steps", type=int, default=2)
    ap.add_argument("--learned", action="store_true",
                    help="also train the warm-start network on the 1024x1024 three-cylinder case and time it")
    ap.add_argument("--learned-steps", type=int, default=4)
    ap.add_argument("--learned-sample-steps", type=int, default=8)
    ap.add_argument("--learned-samples", type=int, default=20000)
    ap.add_argument("--learned-epochs", type=int, default=3)
    ap.add_argument("--particles", action="store_true",
                    help="also time the workload with surface tension and three resolved cylinders")
    ap.add_argument("--forms", action="store_true", default=True,
                    help="also time each form of FORMS on the workload (error against FP64); on by default")
    ap.add_argument("--no-forms", dest="forms", action="store_false")
    ap.add_argument("--batch-form", default="all", choices=["fp64", "fp32", "fp32-warm", "spectral", "fp32-warm-spectral", "all"],
                    help="fp32: the batched replicas use the FP32 stencil form (error against FP64 reported)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        log("note: fewer than 3 warm-up steps")
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
