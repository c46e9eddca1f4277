#!/usr/bin/env python
"""Benchmark of the finite-volume right-hand side and time step on B200: cell-updates per second per RK stage.

Workload (the configuration the metric is quoted on): 3-D Taylor-Green vortex, compressible Navier-Stokes, periodic
[0, 2 pi]^3, 256^3 cells, WENO5-Z + low-Mach HLLC + SSP-RK3, mu = 6.25e-4 (Re = 1600), Pr = 0.71, gamma = 1.4, CFL 0.5,
Ma = 0.1 initial state. A "step" is one SSP-RK3 time step (three residual stages, each the viscous sweep and the fused
reconstruction / Riemann / balance / update kernel); the metric counts cells x 3 per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line on rank 0. `value` is timed on the device with CUDA events on the run's stream (state resident in HBM);
`e2e` goes through the public API per step with the state copied from pinned host memory and the result read back;
`roofline` relates the stage kernel's algorithmic bytes to its measured duration; `cpu_baseline` times the reference
solver (compiled from its sources, oracle/_ref) on this machine's host cores on a bounded sample of the same workload.
Under torchrun (N > 1) the workload is slab-decomposed: one 256^3 part per rank of a 256 x 256 x 256 N mesh, the
interface planes and wave speeds exchanged over NCCL (weak scaling).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per RK stage, mixed+learned vs plain FP64 on B200 at stated L1 err"
UNIT = "cell-updates/s"
STAGES = 3
BYTES_PER_CELL_STAGE = (2 + 3 + 3) / 3 * 5 * 8   # SSP-RK3, 3-D: stage 1 reads U writes R; stages 2-3 read two states, write one


def tgv_workload(n):
    """The configuration string of the Taylor-Green workload (the same in both arms of the benchmark)."""
    return f"Taylor-Green vortex 3-D {n}^3, WENO5-Z + low-Mach HLLC + SSP-RK3, viscous Re 1600 Pr 0.71, CFL 0.5"


def workload(n):
    L = 2 * math.pi
    return dict(nx=n, ny=n, nz=n, Lx=L, Ly=L, Lz=L, gamma=1.4, use_viscous=True, mu=6.25e-4, pr=0.71,
                bc_xmin="periodic", bc_xmax="periodic", bc_ymin="periodic", bc_ymax="periodic", bc_zmin="periodic", bc_zmax="periodic",
                riemann_solver="HLLC (Low-Mach Thornber)", reconstruction="weno5", time_scheme="SSP Runge-Kutta 3", cfl=0.5)


def tgv_state(n, gamma=1.4):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, rho = 1, p = 1/(gamma Ma^2) + (cos 2x + cos 2y)(cos 2z + 2)/16,
    Ma = 0.1, at the cell centres, as conservative cells [rho, rho u, rho v, rho E, rho w] (cell (k*n + j)*n + i)."""
    h = 2 * math.pi / n
    c = (np.arange(n) + 0.5) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    u = (np.sin(x) * np.cos(y) * np.cos(z)).ravel()
    v = (-np.cos(x) * np.sin(y) * np.cos(z)).ravel()
    p = (1.0 / (gamma * 0.01) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0).ravel()
    U = np.zeros((n ** 3, 5))
    U[:, 0] = 1.0
    U[:, 1] = u
    U[:, 2] = v
    U[:, 3] = p / (gamma - 1.0) + 0.5 * (u * u + v * v)
    return U


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs: the sampler is running (its
    first line has arrived) before the region starts, samples every 50 ms, and only the lines that arrive inside the
    region are kept."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = 0

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10 and self.proc.poll() is None:
            time.sleep(0.005)
        self.first = len(self.lines)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            end = len(self.lines)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.reader.join(timeout=5)
            self.out = "".join(self.lines[self.first:end])

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) != len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_profile(name):
    """The committed ncu summary of a stage kernel (profiles/<name>: per-launch DRAM bytes at its cell count, pipe and
    issue fractions, what limits it), or {}."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def ncu_traffic(n, name):
    """Per-launch DRAM bytes of a stage kernel from its committed ncu summary, scaled to n^3 cells, or None."""
    d = ncu_profile(name)
    try:
        return d["dram_bytes_per_launch"] * (n ** 3) / d["cells"]
    except KeyError:
        return None


def cpu_reference_rate(n, warm, timed):
    """The reference solver (oracle/_ref, compiled from its sources) on the host cores: RK3 steps of the same workload."""
    from oracle.oracle import Reference

    ref = Reference({k: v for k, v in workload(n).items()}, initial_profile="taylor_green_3d")
    ref.steps(warm, 1e30)
    t0 = time.perf_counter()
    done = len(ref.steps(timed, 1e30)[0])
    wall = time.perf_counter() - t0
    return n ** 3 * STAGES * done / wall, wall, done


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    return world, rank, local


def _reduce_device():
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device=_reduce_device())
    dist.all_reduce(t)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def load_sensor(local):
    """The trained sensor (fenice_b200/sensor_weights.npz, written by python -m fenice_b200.train_sensor) and its threshold."""
    from fenice_b200.sensor import Sensor

    s = Sensor.load(os.path.join(ROOT, "fenice_b200", "sensor_weights.npz"), device=local)
    return s, float(s.meta["threshold"])


def timed_run(params, U0, precision, args, world, local, sensor=None):
    """W untimed steps, then K steps timed with CUDA events on the run's stream (and around every stage / viscous
    launch), the SM clock sampled meanwhile; returns the run, the device milliseconds (max over ranks), the kernel
    timings and the clock summary."""
    import torch

    from fenice_b200 import Run

    run = Run(params, U=U0, precision=precision, device=local)
    if sensor is not None:
        run.set_sensor(sensor[0], sensor[1])
    ext = torch.cuda.ExternalStream(run.stream(), device=torch.device("cuda", local))
    if args.warmup:
        run.run(1e30, max_steps=args.warmup)
    run.synchronize()
    run.set_timing(True)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        start.record(ext)
        steps = run.run(1e30, max_steps=args.steps)
        end.record(ext)
        run.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    tm = run.timing()
    run.set_timing(False)
    assert steps == args.steps, f"{steps} of {args.steps} steps ran"
    return run, allmax(start.elapsed_time(end), world), tm, clk.summary()


def roofline_of(tm, ms, cells, kernel, traffic, profile=None):
    """The HBM roofline of the stage kernel (algorithmic bytes per launch over its live CUDA-event duration against the
    measured copy bandwidth) and, from its committed ncu summary, what actually limits it: the FP64 or FP32 pipe and
    issue fractions (the stencil is compute- or latency-bound, far below the HBM roof)."""
    peak, peak_kind = measured_peak()
    stage_avg_ms = tm["stage_ms"] / max(tm["stage_launches"], 1)
    alg_bytes = cells * BYTES_PER_CELL_STAGE
    achieved = alg_bytes / (stage_avg_ms * 1e-3) / 1e9
    prof = profile or {}
    limits = {k: prof[k] for k in ("fp64_pipe_frac", "fp64_flop_frac", "fma_pipe_frac", "issue_frac") if k in prof}
    if limits:
        limits["source"] = "ncu --set full of one launch at 192^3 (profiles/)"
    return {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_kind})", "kernel": kernel,
            "limiter": prof.get("limiter"), "pipe_fractions": limits or None,
            "algorithmic_bytes_per_launch": alg_bytes, "stage_launch_ms": round(stage_avg_ms, 4),
            "viscous_launch_ms": round(tm["viscous_ms"] / max(tm["viscous_launches"], 1), 4),
            "stage_share_of_step": round(tm["stage_ms"] / ms, 4), "viscous_share_of_step": round(tm["viscous_ms"] / ms, 4)}


def history_run(params, U0, precision, local, steps, every, sensor=None):
    """`steps` steps of one form with the monitor (kinetic energy, enstrophy: fvg_monitor in its fast order) at step 0
    and every `every` steps; the steps are timed with CUDA events on the run's stream chunk by chunk (the monitor calls
    between the chunks are outside the timed region). Returns (state, ms, history, linear share or None)."""
    import torch

    from fenice_b200 import Run

    warm = Run(params, U=U0, precision=precision, device=local)
    if sensor is not None:
        warm.set_sensor(*sensor)
    warm.run(1e30, max_steps=3)
    warm.close()
    run = Run(params, U=U0, precision=precision, device=local)
    if sensor is not None:
        run.set_sensor(*sensor)
    ext = torch.cuda.ExternalStream(run.stream(), device=torch.device("cuda", local))
    hist, ms, done = [], 0.0, 0

    def sample():
        m = run.monitor("fast")
        hist.append({"step": done, "t": run.t, "kinetic_energy": m["kinetic_energy"], "enstrophy": m["enstrophy"]})

    sample()
    while done < steps:
        k = min(every, steps - done)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(ext)
        got = run.run(1e30, max_steps=k)
        end.record(ext)
        run.synchronize()
        ms += start.elapsed_time(end)
        assert got == k, f"{got} of {k} steps ran"
        done += k
        sample()
    share = None
    if sensor is not None:
        lin, ev = run.sensor_counts()
        share = lin / max(ev, 1)
    U = run.state()
    run.close()
    return U, ms, hist, share


def history_block(n, local, steps, every, world):
    """The Taylor-Green vortex run `steps` steps in the three forms: the kinetic-energy and enstrophy histories of each,
    the throughput of each over the run, and the distance of the mixed forms from the plain FP64 form at the last step."""
    params, U0 = workload(n), tgv_state(n)
    out = {"steps": steps, "monitor_every": every,
           "monitor": "volume averages of 1/2 |m|^2 / rho and 1/2 |curl u|^2 (central differences over 2h, periodic), fvg_monitor's fast order"}
    states = {}
    for name, prec, sens in (("plain_fp64", 0, None), ("mixed", 1, None), ("mixed_learned", 1, load_sensor(local))):
        U, ms, hist, share = history_run(params, U0, prec, local, steps, every, sens)
        ms = allmax(ms, world)
        states[name] = U
        out[name] = {"value": world * n ** 3 * STAGES * steps / (ms * 1e-3), "ms_per_step": ms / steps, "history": hist}
        if share is not None:
            out[name]["linear_share_of_tile_axes"] = share
    for name in ("mixed", "mixed_learned"):
        out[name]["vs_fp64_at_last_step"] = l1_errors(states[name], states["plain_fp64"])
        out[name]["kinetic_energy_rel_diff_at_last_step"] = (out[name]["history"][-1]["kinetic_energy"] /
                                                             out["plain_fp64"]["history"][-1]["kinetic_energy"] - 1.0)
        out[name]["enstrophy_rel_diff_at_last_step"] = (out[name]["history"][-1]["enstrophy"] / out["plain_fp64"]["history"][-1]["enstrophy"] - 1.0)
    out["l1_rho_bar"] = 1e-4
    out["l1_rho_within_bar"] = all(out[k]["vs_fp64_at_last_step"]["rho"]["l1_rel"] <= 1e-4 for k in ("mixed", "mixed_learned"))
    return out


def l1_errors(U, Uref):
    out = {}
    for q, name in enumerate(["rho", "rho_u", "rho_v", "rho_E", "rho_w"]):
        scale = float(np.abs(Uref[:, q]).sum())
        d = np.abs(U[:, q] - Uref[:, q])
        out[name] = {"l1_rel": float(d.sum()) / scale if scale else 0.0,
                     "linf_rel": float(d.max()) / float(np.abs(Uref[:, q]).max()) if scale else 0.0}
    return out


BATCH_T_END = 0.15
BYTES_PER_CELL_STAGE_2D = (2 + 3 + 3) / 3 * 4 * 8   # SSP-RK3 on a 2-D mesh (4 state planes)


BATCH_WORKLOAD = ("512 seeded shock tubes, nx log-uniform in [128, 8192] x 1, rho ~ U[0.1, 1], p ~ U[0.05, 1], u ~ U[-1, 1], "
                  "WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive, to t = 0.15")


def cpu_batch_rate(budget_s):
    """The reference solver (oracle/_ref) on the host cores over the shock tubes in order, one Simulation each, until
    budget_s seconds of work: cell-stages per second."""
    from fenice_b200 import initial
    from oracle.oracle import Reference

    params, states, _ = initial.shock_tubes(512, seed=0)
    work, wall, done = 0, 0.0, 0
    for p, U in zip(params, states):
        ref = Reference(p, initial_state=(1, 0, 0, 1, 0))
        ref.set_state(U)
        t0 = time.perf_counter()
        n = len(ref.steps(1000000, BATCH_T_END)[0])
        wall += time.perf_counter() - t0
        work += n * 3 * p["nx"]
        done += 1
        if wall > budget_s:
            break
    return work / wall, wall, f"the first {done} of the 512 tubes, each run to t = 0.15 ({work} cell-stages in {wall:.1f} s)"


def batch_timed(params, states, precision, schedule, local, timing=False):
    """One whole batch run to t = 0.15 on a fresh batch, timed with CUDA events on the batch's stream."""
    import torch

    from fenice_b200 import Batch

    b = Batch(params, states, precision=precision, device=local)
    b.set_schedule(*schedule)
    if timing:
        b.set_timing(True)
    ext = torch.cuda.ExternalStream(b.stream(), device=torch.device("cuda", local))
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(ext)
    work = b.run(BATCH_T_END)
    end.record(ext)
    torch.cuda.synchronize()
    return b, start.elapsed_time(end), work


def batch_arm(args, world, rank, local):
    """The batched uneven workload: 512 seeded shock tubes (nx log-uniform in [128, 8192], WENO5-Z + HLLC + SSP-RK3,
    CFL 0.4) to t = 0.15, all problems of a GPU in one persistent launch per stage under CUDA graphs. With N GPUs the
    problems are split by cost (no exchange); the time is the slowest GPU's."""
    import torch

    from fenice_b200 import Batch, initial
    from fenice_b200.runtime import split_batch

    params, states, _ = initial.shock_tubes(512, seed=0)
    mine = split_batch(params, world)[rank]
    params = [params[i] for i in mine]
    states = [states[i] for i in mine]
    out = {}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        warm = Batch(params, states, precision=prec, device=local)
        shape, cps, stage_ms = warm.autotune()
        warm.run(1e30, max_steps=max(args.warmup, 3))
        warm.close()
        barrier(world)
        with Clocks(local) as clk:
            b, ms, work = batch_timed(params, states, prec, (shape, cps), local)
        U = b.state()
        b.close()
        ms = allmax(ms, world)
        work_all = allsum(work, world)
        bt, _, _ = batch_timed(params, states, prec, (shape, cps), local, timing=True)
        tm = bt.timing()
        bt.close()
        sched = {"tile": [[64, 1], [128, 1], [256, 1], [16, 15]][shape], "ctas_per_sm": cps, "autotune_stage_ms": stage_ms}
        mixed_schedule = (shape, cps)
        stage_avg = tm["stage_ms"] / max(tm["stage_launches"], 1)
        # algorithmic bytes of one stage launch, averaged over the run: the cells of the running problems per launch
        alg = BYTES_PER_CELL_STAGE_2D * work / max(tm["stage_launches"], 1)
        peak, peak_kind = measured_peak()
        achieved = alg / (stage_avg * 1e-3) / 1e9
        out[name] = {"value": work_all / (ms * 1e-3), "ms": ms, "cell_stages": work_all, "schedule": sched, "clocks": clk.summary(),
                     "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                                  "traffic": None, "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_kind})",
                                  "kernel": f"batch_{'mixed' if prec else 'stage'}_kernel<WENO5, HLLC> (persistent, all problems)",
                                  "stage_launch_ms": round(stage_avg, 4), "stage_launches": tm["stage_launches"],
                                  "stage_share_of_run": round(tm["stage_ms"] / ms, 4),
                                  "note": "the three state pools (about 32 MB each) stay in L2: the bound is the FP64 / FP32 pipe, not HBM"}}
        out[name + "_state"] = U
    U64, Um = out.pop("fp64_state"), out.pop("mixed_state")
    offs = np.concatenate([[0], np.cumsum([p["nx"] for p in params])])
    l1 = [np.abs(Um[a:b_, 0] - U64[a:b_, 0]).sum() / np.abs(U64[a:b_, 0]).sum() for a, b_ in zip(offs[:-1], offs[1:])]
    out["accuracy"] = {"vs": "the FP64 batch (the reference's arithmetic)", "l1_rho_worst": float(max(l1)), "l1_rho_median": float(np.median(l1)),
                       "l1_rho_bar": 1e-4, "within_bar": bool(max(l1) <= 1e-4)}
    out["speedup_of_mixed"] = out["mixed"]["value"] / out["fp64"]["value"]
    # end to end through the public API (mixed form): upload from pinned host memory, the whole run, download
    if args.e2e_steps > 0:
        host = torch.empty((int(offs[-1]), 5), dtype=torch.float64, pin_memory=True).numpy()
        host[:] = np.concatenate(states)
        b = Batch(params, None, precision=1, device=local)
        b.set_schedule(*mixed_schedule)
        barrier(world)
        t0 = time.perf_counter()
        b.set_state(host)
        work = b.run(BATCH_T_END)
        b.state(out=host)
        wall = allmax(time.perf_counter() - t0, world)
        b.close()
        out["e2e"] = {"value": allsum(work, world) / wall, "unit": UNIT,
                      "h2d_bytes_per_step": int(offs[-1]) * 40, "d2h_bytes_per_step": int(offs[-1]) * 40,
                      "timing": "host wall clock around upload + whole run + download (one step = the whole batch to t = 0.15)"}
    out["problems"] = len(params)
    out["cells"] = int(offs[-1])
    return out


QUAD_WORKLOAD = ("seeded four-quadrant Riemann problem (held-out seed {seed}), {n}^2 cells of [0,1]^2, rho, p ~ U[0.1, 2], u, v ~ U[-1, 1], "
                 "WENO5-Z + HLLC + SSP-RK3, CFL 0.4, transmissive, to t = 0.25")


def quad_arm(args, world, rank, local):
    """The four-quadrant workload: one whole run to t = 0.25 per form (plain FP64, mixed, mixed + learned sensor), each
    timed with CUDA events on its stream; L1 of the mixed forms against the plain FP64 run."""
    import torch

    from fenice_b200 import Run, initial

    n, seed = args.size, args.seed
    params, U0 = initial.quadrant_params(n), initial.riemann_quadrants(n, seed)
    sensor = load_sensor(local)
    out, states = {}, {}
    for name, prec, sens in (("plain_fp64", 0, None), ("mixed", 1, None), ("mixed_learned", 1, sensor)):
        warm = Run(params, U=U0, precision=prec, device=local)
        if sens:
            warm.set_sensor(*sens)
        warm.run(1e30, max_steps=max(args.warmup, 3))
        warm.close()
        run = Run(params, U=U0, precision=prec, device=local)
        if sens:
            run.set_sensor(*sens)
        ext = torch.cuda.ExternalStream(run.stream(), device=torch.device("cuda", local))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            start.record(ext)
            steps = run.run(0.25)
            end.record(ext)
            run.synchronize()
        ms = allmax(start.elapsed_time(end), world)
        states[name] = run.state()
        out[name] = {"value": world * n * n * 3 * steps / (ms * 1e-3), "ms": ms, "steps": steps, "clocks": clk.summary()}
        if sens:
            lin, ev = run.sensor_counts()
            out[name]["linear_share_of_tile_axes"] = lin / max(ev, 1)
        run.close()
    for name in ("mixed", "mixed_learned"):
        out[name]["l1_rho_vs_fp64"] = float(np.abs(states[name][:, 0] - states["plain_fp64"][:, 0]).sum() / np.abs(states["plain_fp64"][:, 0]).sum())
    out["l1_rho_learned_vs_mixed"] = float(np.abs(states["mixed_learned"][:, 0] - states["mixed"][:, 0]).sum() / np.abs(states["mixed"][:, 0]).sum())
    return out


CELLS_WORKLOAD = "the cell engine of an adaptive mesh with every leaf of level 0 (leaves in Morton order), fixed dt (the first step's CFL dt): "


def cells_arm(args, world, rank, local):
    """The cell engine (fvg_cells_*) on the benchmark configuration as a level-0 leaf list: steps of fixed length (the first
    step's CFL dt), timed with CUDA events on its stream; the same steps through the public API with the leaf state
    copied from pinned host memory and back (e2e); the reference's own engine (CellFluxEngine + CellAdvance, oracle/_ref)
    on the host cores for one step (cpu_baseline)."""
    import torch

    from fenice_b200.cells import CellEngine, base_leaves

    n = args.size
    params = workload(n)
    lv, ci, cj, ck = base_leaves(params)
    U = tgv_state(n)[(ck.astype(np.int64) * n + cj) * n + ci]
    t0 = time.perf_counter()
    eng = CellEngine(params, lv, ci, cj, ck, U=U, device=local)
    build_s = time.perf_counter() - t0
    _, s0 = eng.residual()
    dx = 2 * math.pi / n
    dt = params["cfl"] * 2.0 / (3.0 / dx) / (s0 + 1e-10)
    ext = torch.cuda.ExternalStream(eng.stream(), device=torch.device("cuda", local))
    eng.advance(dt, max(args.warmup, 3))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        a.record(ext)
        eng.advance(dt, args.steps)
        b.record(ext)
        torch.cuda.synchronize()
    ms = allmax(a.elapsed_time(b), world) / args.steps
    cells = n ** 3
    per_stage = 3 + (2 if params.get("use_viscous") else 0)   # primitive, faces, gather (+ viscous cells, viscous faces)
    out = {"value": world * cells * STAGES / (ms * 1e-3), "ms_per_step": ms, "steps": args.steps, "dt": dt, "faces": eng.nface,
           "gpu_launches": per_stage * STAGES * args.steps,
           "build_s": build_s, "clocks": clk.summary(),
           "roofline": {"bound": "hbm", "achieved": round(cells * STAGES * BYTES_PER_CELL_STAGE / (ms * 1e-3) / 1e9, 2), "peak": measured_peak()[0],
                        "unit": "GB/s", "kernel": "the cell engine's step (primitive, face, viscous cell and face, gather kernels)"}}
    out["roofline"]["frac"] = round(out["roofline"]["achieved"] / out["roofline"]["peak"], 4)
    # e2e: the leaf state from pinned host memory, one step, the state back
    hin = torch.from_numpy(U).pin_memory().numpy()
    hout = torch.empty(U.shape, dtype=torch.float64).pin_memory().numpy()
    eng.set_state(hin)
    eng.step(dt)
    eng.state(out=hout)
    k = max(1, args.e2e_steps)
    t0 = time.perf_counter()
    for _ in range(k):
        eng.set_state(hin)
        eng.step(dt)
        eng.state(out=hout)
    wall = (time.perf_counter() - t0) / k
    out["e2e"] = {"value": world * cells * STAGES / wall, "unit": UNIT, "h2d_bytes_per_step": int(U.nbytes), "d2h_bytes_per_step": int(U.nbytes),
                  "steps": k, "timing": "host wall clock around upload + fvg_cells_step + download of the leaf state"}
    eng.close()
    if rank == 0 and world == 1 and args.cpu_baseline:
        try:
            from oracle.oracle import Reference, ReferenceCells

            os.environ.setdefault("OMP_NUM_THREADS", str(len(os.sched_getaffinity(0))))
            ref = Reference(params, initial_state=(1, 0, 0, 1, 0))
            rc = ReferenceCells(ref, 0)
            rc.set_state(tgv_state(n)[(rc.ck.astype(np.int64) * n + rc.cj) * n + rc.ci])
            rc.steps(dt, 1)
            t0 = time.perf_counter()
            rc.steps(dt, 1)
            wall = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": cells * STAGES / wall, "unit": UNIT, "cores": len(os.sched_getaffinity(0)), "kind": "reference",
                                   "sample": f"1 CellAdvance step of the {n}^3 level-0 mesh after 1 untimed ({wall:.1f} s)"}
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "kind": "reference", "sample": f"unavailable: {e}"}
    return out


CYL_WORKLOAD = ("Mach 2 flow over a cylinder (diameter 1, sharp ghost-cell immersed boundary, slip wall) in an 8 x 12 box, {nx} x {ny}, "
                "inflow rho 1.4, p 1, Mach 2, transmissive elsewhere, from the free stream, {steps} steps; plain: MUSCL (MC) + HLLC + "
                "MUSCL-Hancock; mixed: WENO5-Z + HLLC + SSP-RK3 (FP32 stencil, FP64 state)")


def cyl_arm(args, world, rank, local):
    """The Mach 2 cylinder: plain FP64, mixed and mixed + sensor runs of `steps` steps from the free stream at nx x ny, each
    timed with CUDA events; bow-shock stand-off, Cd and a digest of the final state of each; the reference (CPU) timed on a
    bounded sample of the same mesh."""
    import torch

    from fenice_b200 import Run
    from fenice_b200 import diagnostics as D

    nx, ny, steps = args.cyl_nx, args.cyl_nx * 3 // 2, args.cyl_steps
    sensor = load_sensor(local)
    out = {}
    t_final = None
    for name, form, prec, sens in (("plain_fp64", "plain", 0, None), ("mixed", "mixed", 1, None), ("mixed_learned", "mixed", 1, sensor)):
        params = D.cylinder_params(nx, ny, form)
        run = Run(params, U=D.free_stream(params), precision=prec, device=local)
        if sens:
            run.set_sensor(*sens)
        run.run(1e30, max_steps=3)   # warm-up (graph capture, first refresh)
        run.close()
        run = Run(params, U=D.free_stream(params), precision=prec, device=local)
        if sens:
            run.set_sensor(*sens)
        ext = torch.cuda.ExternalStream(run.stream(), device=torch.device("cuda", local))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            start.record(ext)
            done = run.run(1e30, max_steps=steps)
            end.record(ext)
            run.synchronize()
        ms = allmax(start.elapsed_time(end), world)
        stages = 1 if form == "plain" else 3
        loads = run.ibm_loads()
        U = run.state()
        import hashlib
        out[name] = {"value": world * nx * ny * stages * done / (ms * 1e-3), "ms": ms, "steps": done, "t": run.t, "stages_per_step": stages,
                     "standoff_over_diameter": D.bow_shock_standoff(U, params), "Cd": loads["Cd"], "Cl": loads["Cl"], "clocks": clk.summary(),
                     "state_sha256": hashlib.sha256(np.ascontiguousarray(U).tobytes()).hexdigest()}
        if sens:
            lin, ev = run.sensor_counts()
            out[name]["linear_share_of_tile_axes"] = lin / max(ev, 1)
        if name == "plain_fp64":
            t_final = run.t
        run.close()
    if args.cpu_baseline and rank == 0:
        from oracle.oracle import Reference

        q = D.cylinder_params(nx, ny, "plain")
        ref = Reference(q, initial_state=(D.RHO_IN, q["u_in"], 0.0, D.P_IN))
        ref.steps(2, 1e30)
        t0 = time.perf_counter()
        n = len(ref.steps(40, 1e30)[0])
        wall = time.perf_counter() - t0
        out["reference_cpu"] = {"steps": n, "wall_s": wall, "value": nx * ny * n / wall, "threads": len(os.sched_getaffinity(0))}
    return out


SLAB_WORKLOAD = ("Taylor-Green vortex 3-D, WENO5-Z + low-Mach HLLC + SSP-RK3, viscous Re 1600 Pr 0.71, CFL 0.5, slab-decomposed along z "
                 "(fenice_b200.slabs): {layout}")


def slab_arm(args, world, rank, local):
    """The slab decomposition: at N = 1, the --size^3 mesh as --parts parts in this process on one GPU (the interface
    planes and speeds copied between the parts' buffers), against the whole run of the same mesh, bit for bit; under
    torchrun, one --size^3 part per rank of a mesh of N --size planes along z (halo exchange and speed all-reduce over
    NCCL). Plain FP64 and mixed forms; each timed with CUDA events on the parts' streams over --steps steps after
    --warmup."""
    import hashlib

    import torch

    from fenice_b200 import Run, slabs

    n = args.size
    out = {}
    for name, prec in (("plain_fp64", 0), ("mixed", 1)):
        if world == 1:
            params = workload(n)
            U0 = tgv_state(n)
            nparts = args.parts
            parts = [slabs.Part(params, nparts, i, U=u, precision=prec, device=local) for i, u in enumerate(slabs.split_state(params, U0, nparts))]
            ex = slabs.LocalExchange(parts)
        else:
            params = dict(workload(n), nz=n * world, Lz=2 * math.pi * world)
            grid = tgv_state(n)   # every rank's part starts from the periodic Taylor-Green box (the mesh is N boxes along z)
            parts = [slabs.Part(params, world, rank, U=grid, precision=prec, device=local)]
            ex = slabs.DistExchange.for_part(parts[0])
        slabs.advance(parts, ex, 1e30, args.warmup)
        streams = [torch.cuda.ExternalStream(p.stream(), device=torch.device("cuda", local)) for p in parts]
        torch.cuda.synchronize()
        barrier(world)
        start = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in parts]
        with Clocks(local) as clk:
            start.record(streams[0])
            for st in streams[1:]:
                st.wait_event(start)
            steps, _ = slabs.advance(parts, ex, 1e30, args.steps)
            for e, st in zip(ends, streams):
                e.record(st)
            torch.cuda.synchronize()
        ms = allmax(max(start.elapsed_time(e) for e in ends), world)
        cells = n ** 3 * world
        out[name] = {"value": cells * STAGES * steps / (ms * 1e-3), "ms": ms, "steps": steps, "clocks": clk.summary()}
        if world == 1:
            Ud = slabs.join_states(params, [p.state() for p in parts])
            for p in parts:
                p.close()
            whole = Run(params, U=U0, precision=prec, device=local)
            whole.run(1e30, max_steps=args.warmup)
            ext = torch.cuda.ExternalStream(whole.stream(), device=torch.device("cuda", local))
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record(ext)
            whole.run(1e30, max_steps=args.steps)
            s1.record(ext)
            torch.cuda.synchronize()
            wms = s0.elapsed_time(s1)
            Uw = whole.state()
            whole.close()
            out[name]["whole_run_ms"] = wms
            out[name]["decomposition_overhead"] = ms / wms - 1.0
            out[name]["bits_equal_whole_run"] = bool(np.array_equal(Ud.view(np.uint64), Uw.view(np.uint64)))
            out[name]["state_sha256"] = hashlib.sha256(np.ascontiguousarray(Ud).tobytes()).hexdigest()
        else:
            for p in parts:
                p.close()
    return out


def dist_gpu_arm(args, world, rank, local):
    """N > 1: the workload slab-decomposed along z, one n^3 part per GPU of an n x n x (n N) periodic mesh (weak
    scaling; every part starts from the Taylor-Green box, so the mesh is N boxes along z), the interface planes and the
    speeds exchanged over NCCL on each part's stream (fenice_b200.slabs.DistExchange). The three forms, each W steps
    untimed then K steps timed with CUDA events on the part's stream, the time the slowest rank's."""
    import torch

    from fenice_b200 import slabs

    n = args.size
    params = dict(workload(n), nz=n * world, Lz=2 * math.pi * world)
    U0 = tgv_state(n)
    sensor = load_sensor(local)
    out = {}
    for name, prec, sens in (("plain_fp64", 0, None), ("mixed", 1, None), ("mixed_learned", 1, sensor)):
        part = slabs.Part(params, world, rank, U=U0, precision=prec, device=local)
        if sens:
            part.set_sensor(*sens)
        ex = slabs.DistExchange.for_part(part)
        slabs.advance([part], ex, 1e30, args.warmup)
        st = torch.cuda.ExternalStream(part.stream(), device=torch.device("cuda", local))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier(world)
        with Clocks(local) as clk:
            start.record(st)
            steps, _ = slabs.advance([part], ex, 1e30, args.steps, check_every=args.steps)
            end.record(st)
            torch.cuda.synchronize()
        barrier(world)
        ms = allmax(start.elapsed_time(end), world)
        out[name] = {"value": world * n ** 3 * STAGES * steps / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps, "clocks": clk.summary()}
        if sens:
            lin, ev = part.sensor_counts()
            out[name]["linear_share_of_tile_axes"] = lin / max(ev, 1)
        if sens and args.e2e_steps > 0:
            # end to end through the public API: every step each rank's part state comes from pinned host memory and goes
            # back there (Part.set_state / advance / Part.state: the copies not overlapped with the step)
            host = torch.empty((n ** 3, 5), dtype=torch.float64, pin_memory=True).numpy()
            host[:] = part.state()
            barrier(world)
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                part.set_state(host)
                slabs.advance([part], ex, 1e30, 1)
                part.state(out=host)
            wall = allmax(time.perf_counter() - t0, world)
            out["e2e"] = {"value": world * n ** 3 * STAGES * args.e2e_steps / wall, "unit": UNIT, "h2d_bytes_per_step": world * n ** 3 * 40,
                          "d2h_bytes_per_step": world * n ** 3 * 40, "steps": args.e2e_steps,
                          "timing": "host wall clock: every rank's part state in from pinned host memory, one step, out again"}
        part.close()
    m = out["mixed_learned"]
    # per RK3 step: 3 stage + 3 viscous + 6 pack / unpack + 3 local maxima + dt + axpy + 2 stage speeds + end, the
    # sensor's refresh (network + 2 gate passes) on every step (the kernels return at once off the refresh steps)
    launches = args.steps * (3 + 3 + 6 + 3 + 1 + 1 + 2 + 1 + 3)
    return {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": m["steps"], "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 stencil / f64 state (mixed form) with bf16 sensor; plain form f64",
            "data": "synthetic (Taylor-Green initial state computed in numpy)",
            "config": {"workload": tgv_workload(n), "cells": n ** 3 * world, "stages_per_step": STAGES,
                       "mesh": f"{n} x {n} x {n * world}, one {n}^3 part per GPU",
                       "parallelism": f"slab decomposition along z, {world} parts, NCCL halo exchange and speed all-reduce",
                       "l2": f"inputs larger than L2 ({n ** 3 * 40 / 1e6:.0f} MB per state field and GPU), no flush"},
            "form_of_value": "the mixed-precision form gated by the learned sensor, decomposed (tile rows next to an interface stay WENO5-Z)",
            "forms": out, "e2e": out.pop("e2e", None), "gpu_launches": launches, "clocks": m["clocks"]}


def gpu_arm(args, world, rank, local):
    import torch

    if world > 1:
        return dist_gpu_arm(args, world, rank, local)
    n = args.size
    cells = n ** 3
    params = workload(n)
    U0 = tgv_state(n)
    # the plain FP64 form (the reference's arithmetic, bit for bit) and the mixed form (FP32 stencil, FP64 state)
    plain, ms_p, tm_p, clk_p = timed_run(params, U0, 0, args, world, local)
    U_plain = plain.state()
    plain.close()
    mixed, ms_m, tm_m, clk_m = timed_run(params, U0, 1, args, world, local)
    errs_m = l1_errors(mixed.state(), U_plain)
    mixed.close()
    # the mixed form gated by the learned sensor (the metric's form)
    sensor = load_sensor(local)
    learned, ms_l, tm_l, clk_l = timed_run(params, U0, 1, args, world, local, sensor=sensor)
    errs = l1_errors(learned.state(), U_plain)
    lin, ev = learned.sensor_counts()
    del U_plain
    value = world * cells * STAGES * args.steps / (ms_l * 1e-3)
    value_m = world * cells * STAGES * args.steps / (ms_m * 1e-3)
    value_p = world * cells * STAGES * args.steps / (ms_p * 1e-3)
    mixed = learned

    # end to end through the public API (the value's form): every step takes the state from pinned host memory and
    # writes the new state back there (fvg_step_host: the copies cross the host link in slabs, overlapped with the first
    # and the last stage); one untimed call first (the copy stream and its events are made on the first call)
    e2e = None
    if args.e2e_steps > 0:
        host = torch.empty((cells, 5), dtype=torch.float64, pin_memory=True).numpy()
        host[:] = mixed.state()
        mixed.step_host(host, 1e30)
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            mixed.step_host(host, 1e30)
        wall = allmax(time.perf_counter() - t0, world)
        e2e = {"value": world * cells * STAGES * args.e2e_steps / wall, "unit": UNIT, "h2d_bytes_per_step": cells * 5 * 8,
               "d2h_bytes_per_step": cells * 5 * 8, "steps": args.e2e_steps,
               "timing": "host wall clock around fvg_step_host: pinned host state in, one step, pinned host state out"}
    mixed.close()

    rl_l = roofline_of(tm_l, ms_l, cells, "mixed_stage_kernel_tma<LowMach, gated> (FP32 reconstruction, linear or WENO5-Z per tile-axis, + "
                       "Riemann + balance, FP64 RK update; the cross form on tiles linear along every axis)",
                       ncu_traffic(n, "mixed_stage_kernel_tma_gated_3d.json"), ncu_profile("mixed_stage_kernel_tma_gated_3d.json"))
    rl_m = roofline_of(tm_m, ms_m, cells, "mixed_stage_kernel_tma<LowMach> (the per-axis sweep: FP32 WENO5-Z + Riemann + balance, FP64 RK update)",
                       ncu_traffic(n, "mixed_stage_kernel_weno5_3d.json"), ncu_profile("mixed_stage_kernel_weno5_3d.json"))
    rl_p = roofline_of(tm_p, ms_p, cells, "stage_kernel<3, WENO5, LowMach> (FP64, the reference's arithmetic)",
                       ncu_traffic(n, "stage_kernel_weno5_3d.json"), ncu_profile("stage_kernel_weno5_3d.json"))
    # per RK3 step: 3 viscous + 3 stage + dt + axpy + 2 stage maxima + end; one begin per run; the gated run adds the
    # sensor's refresh (network, 3 dilation passes, tile reduction) to every step (the kernels return at once off the
    # refresh steps)
    launches = 3 * (args.steps * 11 + 1) + args.steps * 5
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_l / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 stencil / f64 state (mixed form) with bf16 sensor; plain form f64",
            "data": "synthetic (Taylor-Green initial state computed in numpy)",
            "config": {"workload": tgv_workload(n), "cells": cells, "stages_per_step": STAGES,
                       "parallelism": f"replicas{world}" if world > 1 else "single GPU",
                       "l2": f"inputs larger than L2 ({cells * 40 / 1e6:.0f} MB per state field), no flush"},
            "accuracy": {"vs": f"plain FP64 form after {args.warmup + args.steps} steps from the same state (the value's form)", "fields": errs,
                         "l1_rho_bar": 1e-4, "l1_rho_within_bar": errs["rho"]["l1_rel"] <= 1e-4},
            "plain_fp64": {"value": value_p, "ms_per_step": ms_p / args.steps, "roofline": rl_p, "clocks": clk_p,
                           "speedup_of_value": value / value_p},
            "mixed": {"value": value_m, "ms_per_step": ms_m / args.steps, "roofline": rl_m, "clocks": clk_m, "speedup_vs_plain": value_m / value_p,
                      "accuracy_l1_rho": errs_m["rho"]["l1_rel"]},
            "sensor": {"threshold": sensor[1], "tile_axes_linear": lin, "tile_axes": ev, "linear_share": lin / max(ev, 1),
                       "refresh_every_steps": 10, "speedup_vs_mixed": value / value_m},
            "form_of_value": "the mixed-precision form gated by the learned sensor; mixed: without the sensor; plain_fp64: the reference's arithmetic",
            "roofline": rl_l, "e2e": e2e, "gpu_launches": launches, "clocks": clk_l}
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fenice_b200", choices=["fenice_b200", "reference"])
    ap.add_argument("--size", type=int, default=256, help="cells per axis (256: the benchmark workload)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the reference on the host cores (rank 0, N = 1)")
    ap.add_argument("--parts", type=int, default=2, help="slab workload at N = 1: parts of the mesh in one process")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "tgv200", "batch", "quadrants", "cylinder", "slab", "cells"],
                    help="tgv: the 3-D Taylor-Green vortex (default); batch: 512 shock tubes in one persistent launch per stage; "
                         "quadrants: a seeded four-quadrant Riemann problem (--size cells per axis, default 2048 for it)")
    ap.add_argument("--seed", type=int, default=2048, help="seed of the quadrants workload")
    ap.add_argument("--cyl-nx", type=int, default=1600, help="cylinder workload: cells along x (y: 3/2 of it)")
    ap.add_argument("--cyl-steps", type=int, default=20000, help="cylinder workload: steps of each GPU form")
    ap.add_argument("--batch", type=int, default=1, help="with --workload tgv at N = 1: add the batched workload's figures")
    ap.add_argument("--history-steps", type=int, default=200,
                    help="with --workload tgv: add the kinetic-energy and enstrophy histories of a run of this many steps in each form (0: none)")
    ap.add_argument("--monitor-every", type=int, default=10, help="steps between two monitor samples of the histories")
    args = ap.parse_args()
    world, rank, local = (1, 0, 0) if args.impl == "reference" and int(os.environ.get("WORLD_SIZE", "1")) == 1 else dist_setup()
    threads = len(os.sched_getaffinity(0))
    if args.impl == "reference":
        if rank != 0:
            return
        os.environ.setdefault("OMP_NUM_THREADS", str(threads))
        if args.workload == "batch":
            rate, wall, sample = cpu_batch_rate(20.0)
            line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * wall,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "impl": "reference",
                    "data": "synthetic (seeded shock tubes)", "config": {"workload": BATCH_WORKLOAD},
                    "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
                    "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
            return
        warm, timed = min(args.warmup, 1), max(1, min(args.steps, 3))
        rate, wall, done = cpu_reference_rate(args.size, warm, timed)
        sample = f"{done} SSP-RK3 step(s) of the {args.size}^3 mesh after {warm} untimed, {threads} OpenMP threads"
        line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": done, "warmup": warm,
                "ms_per_step": 1e3 * wall / done, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (the reference's taylor_green_3d profile)", "impl": "reference",
                "config": {"workload": tgv_workload(args.size), "cells": args.size ** 3, "stages_per_step": STAGES},
                "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
                "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if args.workload == "cylinder":
        cy = cyl_arm(args, world, rank, local)
        m = cy["mixed_learned"]
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": m["steps"], "warmup": 3,
                "ms_per_step": m["ms"] / m["steps"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 stencil / f64 state with bf16 sensor (value); plain form f64", "data": "synthetic (uniform inflow)",
                "config": {"workload": CYL_WORKLOAD.format(nx=args.cyl_nx, ny=args.cyl_nx * 3 // 2, steps=args.cyl_steps) + "; value: mixed + learned sensor",
                           "cells": args.cyl_nx * (args.cyl_nx * 3 // 2)},
                "clocks": m["clocks"], "forms": cy, "e2e": None, "gpu_launches": None}
        if "reference_cpu" in cy:
            r = cy["reference_cpu"]
            line["cpu_baseline"] = {"value": r["value"], "unit": "cell-updates/s", "cores": r["threads"], "kind": "reference",
                                    "sample": f"{r['steps']} MUSCL-Hancock steps of the same mesh from the free stream after 2 untimed"}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "slab":
        sl = slab_arm(args, world, rank, local)
        m = sl["mixed"]
        layout = (f"{args.size}^3 as {args.parts} parts in one process on one GPU" if world == 1
                  else f"{args.size} x {args.size} x {args.size * world}, one {args.size}^3 part per GPU, NCCL halo exchange")
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": m["steps"], "warmup": args.warmup,
                "ms_per_step": m["ms"] / m["steps"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 stencil / f64 state (value); plain form f64", "data": "synthetic (Taylor-Green state)",
                "config": {"workload": SLAB_WORKLOAD.format(layout=layout) + "; value: mixed form", "cells": args.size ** 3 * world,
                           "parallelism": f"slab decomposition z, {max(world, args.parts if world == 1 else world)} parts"},
                "clocks": m["clocks"], "forms": sl, "e2e": None, "gpu_launches": None}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "quadrants":
        if args.size == 256:
            args.size = 2048
        q = quad_arm(args, world, rank, local)
        m = q["mixed_learned"]
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": m["steps"], "warmup": args.warmup,
                "ms_per_step": m["ms"] / m["steps"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 stencil / f64 state with bf16 sensor (value); plain form f64", "data": "synthetic (seeded quadrant states)",
                "config": {"workload": QUAD_WORKLOAD.format(seed=args.seed, n=args.size) + "; value: mixed + learned sensor",
                           "cells": args.size ** 2, "l2": "inputs larger than L2 from 2048^2 on (134 MB per state), no flush"},
                "clocks": m["clocks"], "forms": q, "e2e": None, "gpu_launches": None}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "batch":
        b = batch_arm(args, world, rank, local)
        m = b["mixed"]
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": args.warmup,
                "ms_per_step": m["ms"], "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32 stencil / f64 state (mixed form); plain form f64", "data": "synthetic (seeded shock tubes)",
                "config": {"workload": BATCH_WORKLOAD + "; value: the mixed-precision batch; fp64: the reference's arithmetic",
                           "problems": b["problems"], "cells": b["cells"], "parallelism": f"problems split by cost over {world} GPUs" if world > 1 else "single GPU",
                           "l2": "the state pools fit in L2 (no flush; one step is the whole run)"},
                "roofline": m["roofline"], "clocks": m["clocks"], "e2e": b.get("e2e"), "accuracy": b["accuracy"], "fp64": b["fp64"],
                "speedup_of_mixed": b["speedup_of_mixed"], "gpu_launches": None}
        if rank == 0 and world == 1 and args.cpu_baseline:
            os.environ.setdefault("OMP_NUM_THREADS", str(threads))
            rate, wall, sample = cpu_batch_rate(12.0)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "cells":
        c = cells_arm(args, world, rank, local)
        line = {"metric": METRIC, "value": c["value"], "unit": UNIT, "n_gpus": world, "steps": c["steps"], "warmup": args.warmup,
                "ms_per_step": c["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (Taylor-Green initial state computed in numpy)",
                "config": {"workload": CELLS_WORKLOAD + tgv_workload(args.size), "cells": args.size ** 3, "faces": c["faces"],
                           "stages_per_step": STAGES, "l2": f"inputs larger than L2 ({args.size ** 3 * 40 / 1e6:.0f} MB per state field), no flush"},
                "roofline": c["roofline"], "clocks": c["clocks"], "e2e": c["e2e"], "build_s": c["build_s"], "gpu_launches": c["gpu_launches"]}
        if "cpu_baseline" in c:
            line["cpu_baseline"] = c["cpu_baseline"]
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload == "tgv200":
        hb = history_block(args.size, local, args.history_steps or 200, args.monitor_every, world)
        m = hb["mixed_learned"]
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": hb["steps"], "warmup": 3,
                "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 stencil / f64 state with bf16 sensor (value); plain form f64", "data": "synthetic (Taylor-Green initial state computed in numpy)",
                "config": {"workload": tgv_workload(args.size) + f", {hb['steps']} steps", "cells": args.size ** 3, "stages_per_step": STAGES,
                           "l2": f"inputs larger than L2 ({args.size ** 3 * 40 / 1e6:.0f} MB per state field), no flush"},
                "form_of_value": "mixed-precision form gated by the learned sensor", "history": hb, "e2e": None, "gpu_launches": None}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    line = gpu_arm(args, world, rank, local)
    if args.history_steps > 0 and world == 1:
        line["history"] = history_block(args.size, local, args.history_steps, args.monitor_every, world)
    if world == 1 and args.batch:
        line["batch"] = batch_arm(args, world, rank, local)
        line["batch"]["workload"] = BATCH_WORKLOAD
    if rank == 0 and world == 1 and args.cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(threads))
        try:
            rate, wall, done = cpu_reference_rate(args.size, 1, 1)
            line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": f"{done} SSP-RK3 step of the {args.size}^3 mesh after 1 untimed ({wall:.1f} s)"}
        except Exception as e:  # the reference binary is absent: say so
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
