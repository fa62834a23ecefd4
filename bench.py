#!/usr/bin/env python
"""RK cell-updates/s of the residual / time-step path on B200.

Workload: the isentropic-vortex problem (periodic [0,10]^2, vortex of
strength 5 at (5,5), free stream (1,1,1,1), 4096 quadrants of 16x16 =
1024^2 cells, SSP-RK3, CFL 0.5). One step = one full RK3 time step (three
fused stage kernels, the next step's CFL minimum folded into the last one).

  value : device-resident throughput of the FP32-flux / FP64-state form,
          every step timed with CUDA events on the solver's stream, L2
          flushed between steps (per-step events exclude the flush)
  e2e   : the same metric through the reference's C ABI
          (hpc_amr_evolve_solver) on pinned host arrays, one call per
          10-step segment (the reference example's regrid interval), H2D
          and D2H of the whole state inside the timed region
  forms : the plain FP64 form (bit-exact with the reference) beside it
  learned_amr : the metric's own comparison on an adaptive workload --
          learned indicator + FP32-flux form against plain indicator +
          plain FP64 form, at (measured) equal L1(rho), regrid time
          included; the model is trained on the GPU in the same run

`--impl reference` times the reference's own CPU path (its C driver over
the restated Fortran kernels, oracle/_ref, compiled -O3) on the same 1024^2
mesh on all host cores instead: one MPI rank per core (threads over a
multi-rank MPI stand-in, the reference's ghost exchange every stage).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "amr-demo_b200")]
os.environ.setdefault("AMRGPU_QUIET", "1")

METRIC = "RK cell-updates/s on 1 B200: learned+FP32 form vs plain FP64, at equal L1(rho)"
UNIT = "cell-updates/s"
WORKLOAD = "isentropic vortex, periodic [0,10]^2, 4096 quads x 16x16 = 1024^2 cells, SSP-RK3, CFL 0.5"


def workload_name(mesh, n):
    if n == 16 and mesh.ncell == 4096:
        return WORKLOAD
    side = int(round(mesh.ncells ** 0.5))
    return (f"isentropic vortex, periodic [0,10]^2, {mesh.ncell} quads x {n}x{n} = {side}^2 cells, "
            "SSP-RK3, CFL 0.5")
# Algorithmic HBM bytes per cell-update (one RK step of one cell, summed over
# its stages). FP64 exact SSP-RK3: stage 1 reads X, writes Y and K (96 B);
# stage 2 reads Y, X, K, writes X, K (160 B); stage 3 reads X, K, writes Y
# (96 B) = 352 B. FP32-flux Shu-Osher RK3 keeps no K: 64 + 96 + 96 = 256 B.
B_ALG = {0: 352.0, 1: 256.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU baseline
def _quiet(fn):
    """Runs fn() with the process's stdout (fd 1) sent to /dev/null: the
    reference's driver prints a report every call."""
    sys.stdout.flush()
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)
    try:
        return fn()
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(steps=10, one_rank_steps=2, level=6):
    """The reference's own CPU path on this host, on the benchmark's own
    workload (the 1024^2 vortex mesh, built in NumPy by oracle/workload.py:
    no product library is loaded): its C driver (physics_go over the
    restated Fortran kernels) compiled -O3 for this CPU, run as P MPI ranks
    = P threads (one per host core) over the multi-rank MPI stand-in, each
    rank holding a Morton range of quads plus its ghost quads and
    exchanging them every stage as physics_mpi_real_to_ghost does. value =
    cells x steps / the slowest rank's time in physics_go. A one-rank run of
    the same mesh is reported beside it."""
    from oracle import oracle as O, workload as WL
    from amrgpu import shard as S  # NumPy partitioning only; the library is not loaded
    n = 16
    mesh = WL.uniform_periodic_mesh(level, n)
    s0 = WL.vortex_state(mesh)
    procs = max(1, min(host_cores(), 128, mesh.ncell))
    mt_path, flags = O.timing_build("libref_physics_mt")
    one_path, _ = O.timing_build("libref_physics")
    offs = S.partition(mesh.ncell, procs)
    shards = [S.make_shard(mesh, offs, r) for r in range(procs)]
    cfg = WL.vortex_config(n, steps=steps)
    states = [sh.local_state(s0) for sh in shards]
    out = _quiet(lambda: O.reference_mt_go(shards, states, n, cfg, path=mt_path))
    value = mesh.ncells * steps / out["wall"]
    cfg1 = WL.vortex_config(n, steps=one_rank_steps)
    q = s0.copy()
    t0 = time.perf_counter()
    _quiet(lambda: O.reference_go(mesh, q, n, cfg1, path=one_path))
    one = mesh.ncells * one_rank_steps / (time.perf_counter() - t0)
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"the reference's physics_go ({flags}) on the {int(round(mesh.ncells ** 0.5))}^2 vortex mesh "
                      f"({mesh.ncell} quads of 16x16), {steps} RK3 steps, {procs} MPI ranks as threads with the "
                      f"reference's ghost exchange every stage; slowest rank {out['wall']:.2f} s",
            "one_rank": {"value": one, "unit": UNIT, "cores": 1, "steps": one_rank_steps,
                         "sample": f"one rank, the same mesh, {one_rank_steps} RK3 steps"},
            "same_config": True}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i in range(4) if r[i].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ GPU arm
def autotune(s):
    """The library's stage-launch autotuner (amrgpu_session_autotune), timed
    afresh on this GPU: it compares the compiled launch shapes that give
    bits identical to the default and keeps the fastest."""
    t = s.autotune(retime=True)
    qpb, thr, mb, sweep = s.launch_variant_info(t["variant"])
    return {"quads_per_block": qpb, "threads": thr, "min_blocks": mb, "kernel": "row sweep" if sweep else "block",
            "variant": t["variant"]}


def time_form(ag, mesh, cfg, s0, form, steps, warmup, tune_on=True):
    import torch
    s = ag.Session(mesh, cfg, form=form)
    s.upload(s0)
    tune = autotune(s) if tune_on else None
    s.upload(s0)
    st = torch.cuda.ExternalStream(s.stream())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    s.step(warmup)
    s.sync()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    l0 = s.launch_count()
    for k in range(steps):
        with torch.cuda.stream(st):
            flush.zero_()
        evs[k][0].record(st)
        s.step(1)
        evs[k][1].record(st)
    rep = s.sync()
    launches = s.launch_count() - l0
    ms = [a.elapsed_time(b) for a, b in evs]
    return s, {"ms_steps": ms, "report": rep, "tune": tune, "launches": launches}


def e2e_form(ag, mesh, cfg, s0, form, steps, segment, pinned=False):
    """hpc_amr_evolve_solver on a host array, `segment` steps a call, the
    whole state copied in and out by every call. pinned=False: ordinary
    pageable memory, as the reference's driver allocates it
    (P4EST_ALLOC, amr_external.c:268); True: page-locked memory."""
    import numpy as np
    import torch
    if pinned:
        host = torch.empty(mesh.dof, dtype=torch.float64, pin_memory=True).numpy()
    else:
        host = np.empty(mesh.dof, dtype=np.float64)
    host[:] = s0
    c = ag.Config.current()
    c["form"] = form
    c["time_steps"] = 10 ** 9
    c["regrid_interval"] = segment
    c["final_time"] = 0.0
    c.apply()
    r = ag.evolve_solver(mesh, host, 0)  # warm-up segment (session build, tuning, graphs)
    torch.cuda.synchronize()
    ist = r["istep"]
    calls = max(1, steps // segment)
    t0 = time.perf_counter()
    for _ in range(calls):
        r = ag.evolve_solver(mesh, host, ist)
        ist = r["istep"]
    wall = time.perf_counter() - t0
    return {"value": mesh.ncells * calls * segment / wall, "unit": UNIT,
            "h2d_bytes_per_step": mesh.dof * 8, "d2h_bytes_per_step": mesh.dof * 8,
            "host_memory": "pinned" if pinned else "pageable (numpy)",
            "step": f"one hpc_amr_evolve_solver call = {segment} RK3 steps",
            "error": r["error"]}


def traffic_per_launch(form):
    p = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    v = d.get("fp32_flux" if form == 1 else "fp64_exact")
    return v.get("dram_bytes_per_launch") if v else None


L1_BOUND = 1e-3  # learned run's L1(rho) relative to the plain FP64 run


def learned_amr(args):
    """The metric's comparison on an adaptive workload (unseen seeds of the
    vortex family under AMR: levels 3 to --learned-max-level, default 7 =
    1024^2 at the finest, 8x8 patches, relative density-jump tolerance 0.02,
    t = 3). Five arms per seed, rates with the regrid time included:

      plain_fp64       plain indicator, plain FP64 form, regrid every 5 steps
                       (the baseline)
      plain_fp64_at_I  plain indicator, plain FP64 form, every I steps (the
                       baseline at the learned run's interval)
      plain_fp32       plain indicator, FP32-flux form, every 5 steps (the
                       form's share)
      plain_fp32_at_I  plain indicator, FP32-flux form, every I steps
                       (form + interval)
      learned_fp32     learned indicator, FP32-flux form, every I steps (I =
                       --learned-interval; the model is trained in this run
                       on covering labels: a quad is labelled refine when the
                       plain indicator asks for refinement at any 5-step point
                       of the interval, coarsen only when it asks for
                       coarsening at all of them; its judge counts the quads
                       it leaves coarser than the plain indicator would)

    The learned run is held to the north-star bound: its final density on
    the finest level's uniform grid must be within 1e-3 (relative L1) of the
    plain FP64 run's. A seed that misses it falls back -- its delivered
    result is the plain FP64 run's, and the learned arm is charged both
    runs' time. The same check against the same-interval plain FP64 run is
    reported beside it."""
    import numpy as np
    from amrgpu import learned as L
    n, lo, hi, tol = 8, 3, args.learned_max_level, 0.02
    I = args.learned_interval
    t0 = time.perf_counter()
    m = L.Mlp(seed=0)
    rows = L.collect(m, range(args.learned_seeds), n, lo, hi, tol, regrid_interval=I, regrids=25, cover_every=5)
    t1 = time.perf_counter()
    hist, _ = L.train(m, epochs=20, batch=8192, lr=1e-3, seed=0)
    t2 = time.perf_counter()
    out = {"workload": f"isentropic vortex family under AMR, periodic [0,10]^2, levels 3-{hi}, 8x8 patches, "
                       "density-jump tol 0.02, SSP-RK3 CFL 0.5, t = 3, unseen seeds 5000-5002",
           "training": {"rows": rows, "epochs": 20, "batch": 8192, "lr": 1e-3, "collect_s": t1 - t0,
                        "train_s": t2 - t1, "final_loss": hist[-1][0], "final_accuracy": hist[-1][1],
                        "seeds": args.learned_seeds, "labels": f"covering: plain classes every 5 steps over {I}"},
           "l1_bound": L1_BOUND}
    arms = (("plain_fp64", None, 0, 5), ("plain_fp64_at_I", None, 0, I), ("plain_fp32", None, 1, 5),
            ("plain_fp32_at_I", None, 1, I), ("learned_fp32", m, 1, I))
    # one untimed run of every arm first (seed 4999): kernels load on their
    # first launch and the library's autotuner times a launch shape for each
    # mesh-size bucket it meets first; neither one-time cost should land in
    # whichever arm happens to run first
    for key, mlp, form, ri in arms:
        f, cfg, soln, par = L.vortex_amr(4999, n, lo, hi, tol, form=form)
        s, _ = L.run(f, soln, n, cfg, final_time=3.0, regrid_interval=ri, min_level=lo, max_level=hi, tol=tol,
                     mlp=mlp, form=form, seed=4999, judge_coarser=mlp is not None)
        s.close()
    runs = {k: [] for k, _, _, _ in arms}
    for seed in (5000, 5001, 5002):
        ends = {}
        for key, mlp, form, ri in arms:
            f, cfg, soln, par = L.vortex_amr(seed, n, lo, hi, tol, form=form)
            s, r = L.run(f, soln, n, cfg, final_time=3.0, regrid_interval=ri, min_level=lo, max_level=hi, tol=tol,
                         mlp=mlp, form=form, seed=seed, judge_coarser=mlp is not None)
            q = s.download()
            r["l1_rho_vs_exact"] = L.l1_rho_vs_exact(s.mesh, q, n, r["time"], par)
            r["secs"] = r["solve_s"] + r["regrid_s"]
            ends[key] = L.to_uniform(f, q, n, hi)
            runs[key].append(r)
            s.close()
        base = runs["plain_fp64"][-1]

        def dist(a, b):
            return float(np.abs(ends[a] - ends[b]).sum() / np.abs(ends[b]).sum())

        for key, _, _, _ in arms[1:]:
            runs[key][-1]["l1_rho_vs_plain_run"] = dist(key, "plain_fp64")
        for key in ("plain_fp32_at_I", "learned_fp32"):
            runs[key][-1]["l1_rho_vs_plain_run_at_I"] = dist(key, "plain_fp64_at_I")
        lr = runs["learned_fp32"][-1]
        lr["within_bound"] = lr["l1_rho_vs_plain_run"] <= L1_BOUND
        lr["within_bound_at_I"] = lr["l1_rho_vs_plain_run_at_I"] <= L1_BOUND
        # what the checked learned run delivers and costs
        lr["delivered_cell_updates"] = lr["cell_updates"] if lr["within_bound"] else base["cell_updates"]
        lr["charged_s"] = lr["secs"] if lr["within_bound"] else lr["secs"] + base["secs"]
    for key, rs in runs.items():
        cu = sum(r["cell_updates"] for r in rs)
        secs = sum(r["secs"] for r in rs)
        out[key] = {"value": cu / secs, "unit": UNIT, "regrid_interval": dict((k, ri) for k, _, _, ri in arms)[key],
                    "mean_cells": float(np.mean([r["mean_cells"] for r in rs])),
                    "l1_rho_vs_exact": float(np.mean([r["l1_rho_vs_exact"] for r in rs])),
                    "regrids": int(sum(r["regrids"] for r in rs)),
                    "solve_s": sum(r["solve_s"] for r in rs), "regrid_s": sum(r["regrid_s"] for r in rs)}
        if key != "plain_fp64":
            out[key]["l1_rho_vs_plain_run"] = [float(r["l1_rho_vs_plain_run"]) for r in rs]
        if key in ("plain_fp32_at_I", "learned_fp32"):
            out[key]["l1_rho_vs_plain_run_at_I"] = [float(r["l1_rho_vs_plain_run_at_I"]) for r in rs]
    lr = runs["learned_fp32"]
    checked = sum(r["delivered_cell_updates"] for r in lr) / sum(r["charged_s"] for r in lr)
    out["learned_fp32"].update({"judge_disagreement": float(np.mean([r["disagree_rate"] for r in lr])),
                                "judge_coarser_than_plain": float(np.mean([r["coarser_rate"] for r in lr])),
                                "judge_fallbacks": [r["fallback_at"] for r in lr],
                                "within_bound": [bool(r["within_bound"]) for r in lr],
                                "within_bound_at_I": [bool(r["within_bound_at_I"]) for r in lr],
                                "checked_value": checked})
    base = out["plain_fp64"]["value"]
    base_i = out["plain_fp64_at_I"]["value"]
    out["speedup_over_plain_fp64"] = {k: out[k]["value"] / base for k in ("plain_fp64_at_I", "plain_fp32",
                                                                         "plain_fp32_at_I", "learned_fp32")}
    out["speedup_over_plain_fp64"]["learned_fp32_checked"] = checked / base
    out["speedup_over_plain_fp64_at_I"] = {k: out[k]["value"] / base_i for k in ("plain_fp32_at_I", "learned_fp32")}
    out["indicator_share"] = out["learned_fp32"]["value"] / out["plain_fp32_at_I"]["value"]
    out["target_met"] = bool(all(r["within_bound"] for r in lr) and checked / base >= 2.0)
    out["target_met_at_I"] = bool(all(r["within_bound_at_I"] for r in lr) and
                                  out["learned_fp32"]["value"] / base_i >= 2.0)
    # the same comparison read two other ways: wall time to reach t = 3
    # (every arm runs the same simulated time; an indicator that needs fewer
    # cells lowers cell-updates/s but not the time), and the error against
    # the exact vortex (no worse than the plain FP64 run's)
    secs = {k: out[k]["solve_s"] + out[k]["regrid_s"] for k in out if isinstance(out[k], dict) and "solve_s" in out[k]}
    out["time_to_solution_speedup"] = {k: secs["plain_fp64"] / v for k, v in secs.items() if k != "plain_fp64"}
    out["l1_vs_exact_no_worse_than_plain_fp64"] = {
        k: bool(out[k]["l1_rho_vs_exact"] <= out["plain_fp64"]["l1_rho_vs_exact"])
        for k in ("plain_fp64_at_I", "plain_fp32", "plain_fp32_at_I", "learned_fp32")}
    m.close()
    return out


def vortex_period(args):
    """Config 2 to its end: the 1024^2 vortex (16x16 patches, level 6) run to
    t = 10, one period, in both forms on the device (CUDA graphs of 60 steps,
    the last step clipped at t = 10). Reports steps, wall time and rate, the
    relative L1(rho) of each form against the exact translated vortex and
    between the forms."""
    import numpy as np
    import torch
    import amrgpu as ag
    from amrgpu import learned as L, workloads as W
    out = {"workload": "isentropic vortex, periodic [0,10]^2, 4096 quads x 16x16 = 1024^2 cells, SSP-RK3, "
                       "CFL 0.5, run to t = 10 (one period)"}
    ends = {}
    for form, key in ((1, "fp32_flux"), (0, "plain_fp64")):
        f, mesh, cfg, s0 = W.vortex_1024(level=args.level, n=args.patch, final_time=10.0, steps=10 ** 9)
        s = ag.Session(mesh, cfg, form=form)
        s.upload(s0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        steps = 0
        while True:
            s.step(600, graph_steps=60)
            rep = s.sync()
            if rep["time"] >= 10.0 or rep["error"] or rep["steps"] == steps:
                break
            steps = rep["steps"]
        wall = time.perf_counter() - t0
        q = s.download()
        s.close()
        ends[key] = q
        out[key] = {"steps": rep["steps"], "time": rep["time"], "wall_s": wall,
                    "value": mesh.ncells * rep["steps"] / wall, "unit": UNIT, "error": rep["error"],
                    "l1_rho_vs_exact": L.l1_rho_vs_exact(mesh, q, args.patch, rep["time"], (5.0, 5.0, 5.0))}
    a = ends["fp32_flux"].reshape(-1, 4)[:, 0]
    b = ends["plain_fp64"].reshape(-1, 4)[:, 0]
    out["l1_rho_rel_fp32_vs_fp64"] = float(np.abs(a - b).sum() / np.abs(b).sum())
    return out


def amr_workload(args):
    """One adaptive workload through the library's AMR loop (regrid every 5
    steps: GPU tagging by the density jump, host forest refine / coarsen /
    2:1 balance, in-place GPU remap). --warmup steps untimed, then --steps
    steps timed: cell-updates/s with the regrid time included (the
    metric's definition for adaptive runs) and of the solve alone. The
    whole run is made twice from a fresh forest and session and the second
    is reported: the first loads the kernels and lets the autotuner time a
    launch shape for every mesh size the run meets (what a production run
    has from its tuning cache)."""
    first = _amr_workload_once(args)
    out = _amr_workload_once(args)
    out["note"] = "second of two identical runs (the first loads kernels and tunes launch shapes)"
    out["first_run_value"] = first["value"]
    return out


def _amr_workload_once(args):
    import amrgpu as ag
    from amrgpu import amr, workloads as W
    t0 = time.perf_counter()
    rule = None
    if args.workload == "four_quadrant":
        f, mesh, cfg, soln = W.four_quadrant(seed=0, min_level=4, max_level=9, n=16, form=args.amr_form)
        desc = ("four-quadrant Riemann problem, unit square, levels 4-9, 16x16 patches, density-jump tol 0.05, "
                "SSP-RK3 CFL 0.5, regrid every 5 steps")
        lo, hi = 4, 9
        if args.mixed:
            # 8x8 patches on the two coarsest levels (the smooth far field),
            # 16x16 on the refined levels
            rule = lambda lv: 8 if lv <= lo + 1 else 16  # noqa: E731
            sizes = f.patch_sizes(rule)
            mesh = f.mesh_mixed(sizes)
            soln = f.initialize(sizes)
            desc = desc.replace("16x16 patches", "mixed patches (8x8 at levels 4-5, 16x16 at 6-9, one work list)")
    else:
        f, mesh, cfg, soln = W.shock_bubble(seed=0, min_level=5, max_level=args.max_level, n=16, form=args.amr_form)
        desc = (f"Mach-2 shock-bubble interaction, [0,2]x[0,1] (2x1 trees), levels 5-{args.max_level}, 16x16 "
                "patches, density-jump tol 0.1, SSP-RK3 CFL 0.5, regrid every 5 steps")
        lo, hi = 5, args.max_level
    t_setup = time.perf_counter() - t0
    cells0 = mesh.ncells
    cfg["final_time"] = 0.0
    s = ag.Session(mesh, cfg, form=args.amr_form)
    if rule is not None:
        s.set_patch_rule(rule)  # regrids build the mixed mesh on the device
    # buffers for meshes up to 3x the initial one, reserved before the
    # clock starts: regrids within it allocate nothing
    s.reserve(3 * mesh.ncells, 3 * mesh.ncell)
    s.upload(soln)
    for _ in range(max(1, args.warmup // 5)):
        s.step(5)
        s.sync()
        amr.regrid(f, s, 16, lo, hi, size_of_level=rule)
    import numpy as np
    solve = reg = 0.0
    cu = steps = 0
    cells = []
    cycles = max(1, args.steps // 5)
    for _ in range(cycles):
        # the regrid of amr.regrid: tags, refine / coarsen (on the device
        # too, overlapped with the host forest's), balance, descriptors and
        # remap in one call
        a = time.perf_counter()
        s.step(5)
        rep = s.sync()
        b = time.perf_counter()
        cu += rep["steps"] * s.mesh.ncells
        steps += rep["steps"]
        cells.append(s.mesh.ncells)
        s.adapt_regrid(f, lo, hi)
        h = time.perf_counter()
        solve += b - a
        reg += h - b
    err = rep["error"]
    s.close()
    return {"metric": METRIC, "workload": args.workload, "config": {"workload": desc},
            "form": "FP32 flux, FP64 state" if args.amr_form == 1 else "plain FP64 (bit-exact)",
            "value": cu / (solve + reg), "unit": UNIT, "solve_only": cu / solve, "steps": steps,
            "regrids": steps // 5, "cells_start": cells0, "cells_min": min(cells), "cells_max": max(cells),
            "solve_s": solve, "regrid_s": reg, "setup_s": t_setup, "error": err,
            "regrid_ms": 1e3 * reg / cycles,
            "solve_ms_per_5_steps": 1e3 * solve / cycles}


def time_sharded(ag, S, mesh, cfg, s0, form, steps, warmup, tune_on, world, rank):
    """One rank of the sharded run: Morton-range shard of the global mesh,
    per-stage ghost exchange and per-step CFL MIN over NCCL (amrgpu.shard);
    every step timed with CUDA events on the rank's solver stream (exchange
    included), L2 flushed between steps."""
    import torch
    import torch.distributed as dist
    sh = S.make_shard(mesh, S.partition(mesh.ncell, world), rank)
    cfg["form"] = form
    r = S.GpuRank(sh, cfg)
    local = sh.local_state(s0)
    tune = None
    if tune_on:
        r.upload(local)
        tune = autotune(r.session)
    drv = S.Distributed(r)
    drv.start(local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    drv.step(warmup)
    torch.cuda.synchronize()
    dist.barrier()
    # each step one CUDA graph launch (its exchanges and the CFL reduction
    # captured with the kernels) when every rank could capture; else eager
    graphed = drv.capture()
    ok = torch.tensor([1 if graphed else 0], dtype=torch.int32, device="cuda")
    dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    graphed = bool(ok.item())
    stepper = drv.step_graphs if graphed else drv.step
    stepper(3)  # the graphs' first launches
    torch.cuda.synchronize()
    dist.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    l0 = r.session.launch_count()
    for k in range(steps):
        with torch.cuda.stream(r.stream):
            flush.zero_()
            evs[k][0].record(r.stream)
        stepper(1)
        evs[k][1].record(r.stream)
    rep = drv.report()
    launches = r.session.launch_count() - l0
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    return r, drv, {"ms_steps": ms, "report": rep, "tune": tune, "launches": launches,
                    "ghosts": int(len(sh.ghosts)), "sends": int(len(sh.send_quads)), "local_quads": sh.nlocal,
                    "step_graphs": graphed}


def e2e_sharded(drv, local, steps, segment):
    """Per rank: upload of the rank's state from pinned host memory, a
    segment of steps, download of the state, wall-clock per segment."""
    import torch
    import torch.distributed as dist
    host = torch.empty(len(local), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = local
    calls = max(1, steps // segment)
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(calls):
        drv.start(host)
        drv.step(segment)
        drv.download(host)
    wall = time.perf_counter() - t0
    t = torch.tensor([wall], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item()), calls


def run_sharded(args, world, rank, local):
    """--gpus N > 1: weak scaling, one 1024^2 tree per rank on a periodic
    N x 1 brick, ranks exchange ghost quads before every stage."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import amrgpu as ag
    from amrgpu import shard as S
    from amrgpu import workloads as W
    f, mesh, cfg, s0 = W.vortex_1024(level=args.level, final_time=0.0, steps=10 ** 9, trees_x=world)
    hbm, peak_kind = peaks()
    run_forms = (0, 1) if args.form < 0 else (args.form,)
    res = {}
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for form in run_forms:
            res[form] = time_sharded(ag, S, mesh, cfg, s0, form, args.steps, args.warmup, not args.no_tune,
                                     world, rank)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = clk.summary()
    out = {}
    for form, (r, drv, d) in res.items():
        t = torch.tensor([sum(d["ms_steps"])], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
        cells = mesh.ncells  # all ranks
        avg_ms = tot_ms / args.steps
        per_rank_cells = d["local_quads"] * mesh.n * mesh.n
        out[form] = {"value": cells * args.steps / (tot_ms * 1e-3), "ms_per_step": avg_ms,
                     "achieved_gbs": per_rank_cells * B_ALG[form] / (avg_ms * 1e-3) / 1e9, **d}
    e2e = None
    if not args.no_e2e and 1 in res:
        r, drv, d = res[1]
        local_state = r.shard.local_state(s0)
        wall, calls = e2e_sharded(drv, local_state, args.steps, args.segment)
        e2e = {"value": mesh.ncells * calls * args.segment / wall, "unit": UNIT,
               "h2d_bytes_per_step": len(local_state) * 8, "d2h_bytes_per_step": r.shard.mesh.dof * 8,
               "step": f"per rank: upload + {args.segment} RK3 steps (sharded driver) + download, "
                       "slowest rank's wall clock"}
    for form, (r, drv, d) in res.items():
        drv.release_graphs()  # graphs holding NCCL calls go before the process group
        r.close()
    if rank == 0:
        head = out[1] if 1 in out else out[run_forms[0]]
        hf = 1 if 1 in out else run_forms[0]
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 state" if hf == 1 else "f64",
            "data": "synthetic (seeded analytic vortex; no dataset exists)",
            "config": {"workload": f"isentropic vortex, periodic [0,{10 * world}]x[0,10] ({world}x1 trees), "
                                   f"{mesh.ncell} quads x 16x16 = {mesh.ncells} cells, one 1024^2 tree per rank, "
                                   "SSP-RK3, CFL 0.5",
                       "cells": mesh.ncells, "quads": mesh.ncell, "patch": "16x16",
                       "ghost_quads_per_rank": head["ghosts"], "send_quads_per_rank": head["sends"],
                       "l2": "flushed between steps (256 MB write; per-step CUDA events exclude it)",
                       "launch": head["tune"],
                       "parallelism": f"dp{world}: Morton-range shards, NCCL ghost exchange before every "
                                      "stage, MIN all-reduce of the CFL step every step",
                       "step_graphs": bool(head.get("step_graphs"))},
            "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                         "frac": head["achieved_gbs"] / hbm, "traffic": traffic_per_launch(hf),
                         "peak_kind": peak_kind, "bytes_per_cell_update": B_ALG[hf],
                         "note": "per rank; step time includes the ghost exchange"},
            "forms": {("plain_fp64" if k == 0 else "fp32_flux"): {"value": v["value"],
                                                                   "ms_per_step": v["ms_per_step"]}
                      for k, v in out.items()},
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": int(sum(v["launches"] for v in out.values())),
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    dist.barrier()
    dist.destroy_process_group()


def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1 or args.shard:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        return run_sharded(args, world, rank, local)
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_baseline()

    import amrgpu as ag
    from amrgpu import workloads as W
    f, mesh, cfg, s0 = W.vortex_1024(level=args.level, n=args.patch, final_time=0.0, steps=10 ** 9)
    hbm, peak_kind = peaks()
    run_forms = (0, 1) if args.form < 0 else (args.form,)

    forms = {}
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for form in run_forms:
            s, r = time_form(ag, mesh, cfg, s0, form, args.steps, args.warmup, not args.no_tune)
            forms[form] = (s, r)
    torch.cuda.synchronize()
    clocks = clk.summary()

    out = {}
    for form, (s, r) in forms.items():
        tot_ms = sum(r["ms_steps"])
        cells = mesh.ncells
        value = cells * args.steps / (tot_ms * 1e-3)
        avg_ms = tot_ms / args.steps
        achieved = cells * B_ALG[form] / (avg_ms * 1e-3) / 1e9
        out[form] = {"value": value, "ms_per_step": avg_ms, "achieved_gbs": achieved, "report": r["report"],
                     "tune": r["tune"], "launches": r["launches"]}

    if len(run_forms) == 1:
        if rank == 0:
            r = out[run_forms[0]]
            print(json.dumps({"metric": METRIC, "value": r["value"], "unit": UNIT, "form": run_forms[0],
                              "level": args.level, "ms_per_step": r["ms_per_step"],
                              "achieved_gbs": r["achieved_gbs"], "launches": r["launches"],
                              "clocks": clocks}), flush=True)
        return
    # accuracy of the FP32 form against the FP64 form after the same steps
    q64 = forms[0][0].download().reshape(-1, 4)
    q32 = forms[1][0].download().reshape(-1, 4)
    l1 = float(np.abs(q32[:, 0] - q64[:, 0]).sum() / np.abs(q64[:, 0]).sum())

    e2e = e2e_pinned = None
    if not args.no_e2e:
        e2e = e2e_form(ag, mesh, cfg, s0, 1, args.steps, args.segment)
        e2e_pinned = e2e_form(ag, mesh, cfg, s0, 1, args.steps, args.segment, pinned=True)
    amr = None
    if not args.no_learned:
        amr = learned_amr(args)
    config3 = None
    if not args.no_amr:
        # config 3: the four-quadrant AMR loop (levels 4-9, regrid every 5
        # steps, regrid time included) with 16x16 patches and with mixed
        # 8x8 / 16x16 patches in one work list
        import argparse as _ap
        config3 = {}
        for key, mixed in (("uniform_16", False), ("mixed_8_16", True)):
            a3 = _ap.Namespace(workload="four_quadrant", mixed=mixed, amr_form=1, steps=60, warmup=10,
                               max_level=args.max_level)
            r3 = amr_workload(a3)
            config3[key] = {k: r3[k] for k in ("value", "solve_only", "steps", "regrids", "cells_min", "cells_max",
                                               "error", "regrid_ms")}
            # the same steps (same finest cell, same dt) for both: wall time
            # per step, regrid included, is the like-for-like figure
            config3[key]["wall_ms_per_step"] = 1e3 * (r3["solve_s"] + r3["regrid_s"]) / max(r3["steps"], 1)
            config3[key]["workload"] = r3["config"]["workload"]
        config3["mixed_over_uniform"] = config3["mixed_8_16"]["value"] / config3["uniform_16"]["value"]
        config3["uniform_over_mixed_wall_time"] = (config3["uniform_16"]["wall_ms_per_step"] /
                                                   config3["mixed_8_16"]["wall_ms_per_step"])
    head = out[1]
    # the committed ncu traffic figure is for the default workload (16x16, level 6)
    traffic = traffic_per_launch(1) if (args.patch == 16 and args.level == 6) else None
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 flux / f64 state",
        "data": "synthetic (seeded analytic vortex; no dataset exists)",
        "config": {"workload": workload_name(mesh, args.patch), "cells": mesh.ncells, "quads": mesh.ncell,
                   "patch": f"{args.patch}x{args.patch}",
                   "form": "FP32 flux, FP64 state, Shu-Osher SSP-RK3", "l2": "flushed between steps "
                   "(256 MB write; per-step CUDA events exclude it)", "launch": head["tune"],
                   "parallelism": "1 GPU"},
        "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": head["achieved_gbs"] / hbm, "traffic": traffic,
                     "peak_kind": peak_kind, "bytes_per_cell_update": B_ALG[1]},
        "forms": {
            "plain_fp64": {"value": out[0]["value"], "ms_per_step": out[0]["ms_per_step"],
                           "achieved_gbs": out[0]["achieved_gbs"], "frac": out[0]["achieved_gbs"] / hbm,
                           "bytes_per_cell_update": B_ALG[0], "launch": out[0]["tune"],
                           "bound": "fp64 pipe (IEEE div/sqrt sequences)"},
            "fp32_flux": {"value": out[1]["value"], "ms_per_step": out[1]["ms_per_step"]},
            "speedup_fp32_over_fp64": out[1]["value"] / out[0]["value"],
            "l1_rho_rel_fp32_vs_fp64": l1,
        },
        "e2e": e2e,
        "e2e_pinned": e2e_pinned,
        "learned_amr": amr,
        "amr_config3": config3,
        "clocks": clocks,
        "gpu_launches": int(out[0]["launches"] + out[1]["launches"]),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_reference(args):
    """The reference arm: the reference's own CPU path (cpu_baseline) on the
    benchmark's mesh, --warmup untimed steps then --steps timed steps on all
    host cores; rank 0 of a torchrun launch alone runs it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O, workload as WL  # noqa: F401
    cpu_baseline(steps=max(1, args.warmup), one_rank_steps=1)  # warm-up: page in, first touch
    cb = cpu_baseline(steps=args.steps, one_rank_steps=2)
    value = cb["value"]
    ms = 1e3 * (1024 * 1024) / value
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded analytic vortex)",
            "config": {"workload": WORKLOAD, "parallelism": f"{cb['cores']} MPI ranks (threads) on host cores"},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--segment", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--level", type=int, default=6, help="forest level (6: the 1024^2 workload)")
    ap.add_argument("--patch", type=int, default=16, choices=[8, 16],
                    help="subgrid patch size of the vortex workload (16: the 1024^2 workload at level 6)")
    ap.add_argument("--form", type=int, default=-1, help="time one form only (0 FP64, 1 FP32 flux)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shape")
    ap.add_argument("--shard", action="store_true",
                    help="use the sharded multi-rank driver also at one rank (under torchrun)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-indicator AMR comparison")
    ap.add_argument("--learned-only", action="store_true", help="run only the learned-indicator AMR comparison")
    ap.add_argument("--learned-seeds", type=int, default=64, help="seeded runs that make the training set")
    ap.add_argument("--learned-interval", type=int, default=20,
                    help="regrid interval of the learned run (its model predicts the plain class that many steps ahead)")
    ap.add_argument("--learned-max-level", type=int, default=7,
                    help="finest level of the learned-indicator workload (8x8 patches; 7 = 1024^2 at the finest)")
    ap.add_argument("--workload", choices=["vortex", "vortex_period", "four_quadrant", "shock_bubble"],
                    default="vortex",
                    help="vortex: the headline line; vortex_period: both forms to t = 10 with their errors; "
                         "the others time one adaptive workload")
    ap.add_argument("--amr-form", type=int, default=1, help="form of the adaptive workloads (0 FP64, 1 FP32 flux)")
    ap.add_argument("--no-amr", action="store_true", help="skip the adaptive config-3 lines (uniform and mixed)")
    ap.add_argument("--mixed", action="store_true",
                    help="four_quadrant with mixed patch sizes (8x8 on the coarsest two levels, 16x16 above)")
    ap.add_argument("--max-level", type=int, default=11, help="finest level of the shock-bubble workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "vortex_period":
        sys.path[:0] = [ROOT, os.path.join(ROOT, "amr-demo_b200")]
        print(json.dumps({"metric": METRIC, "vortex_period": vortex_period(args)}), flush=True)
    elif args.workload != "vortex":
        sys.path[:0] = [ROOT, os.path.join(ROOT, "amr-demo_b200")]
        print(json.dumps(amr_workload(args)), flush=True)
    elif args.learned_only:
        sys.path[:0] = [ROOT, os.path.join(ROOT, "amr-demo_b200")]
        print(json.dumps({"metric": METRIC, "learned_amr": learned_amr(args)}), flush=True)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
