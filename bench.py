#!/usr/bin/env python
"""FP64 cell-updates/s of the GenASiS Fluid_P_I finite-volume step on B200.

Workload (default): 3-D sine-wave advection on the 256^3 periodic unit cube,
FP64, gamma = 1.4, rho = 1 + 0.5 sin(2 pi (x+y+z)), v = (1,1,1), p = 1,
PLM (generalized minmod, theta 1.4) + HLLC, RK2, CFL 0.8.  One step = one
integrator cycle: CFL time step + RK2 step (two fused stages, features,
ghost refresh), device-resident, replayed from a CUDA graph.  Synthetic
seeded inputs with the benchmark's shape; the 845 MB state exceeds L2.

The headline runs the fast build (libgfx_fluid_fast.so, FP64 with fused
multiply-adds); the exact build (libgfx_fluid.so, the reference's rounding)
is measured beside it, and both are checked against the oracle per step on
the 256^3 state in the same run.  After the timed region the line also
carries the full-crossing L1 error and the other benchmark configurations
(Sod 128^3, 512 bricks, the Kelvin-Helmholtz adjoint, Rayleigh-Taylor
384 x 384 x 768, the 256^3 wave as a 2 x 2 x 2 chart); --no-extras skips them.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the benchmark fixes one GPU per domain;
the path has no data exchange between replicas), one rank per GPU.
--impl reference times the reference's CPU step (the C restatement in
oracle/, the reference itself being Fortran + MPI that cannot be compiled
here) on the host cores, with all host threads.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-updates/s"
UNIT = "cell-updates/s"
# Algorithmic bytes per cell of each fused stage (6 FP64 conserved fields):
# stage 1 reads U^n and writes Y; stage 2 reads Y and U^n and writes U^n+1.
STAGE_BYTES = {"stage1": 96.0, "stage2": 144.0}
STEP_BYTES = 240.0
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="cells per axis of the sine wave")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="sine",
                    choices=["sine", "bricks", "adjoint", "adjoint_step", "rt", "sod", "chart"],
                    help="sine: the 256^3 headline; bricks: 512 uneven bricks, batched "
                         "launch against a loop of per-brick launches; adjoint: 128^3 "
                         "Kelvin-Helmholtz, adjoint against forward and finite differences")
    ap.add_argument("--directions", type=int, default=64,
                    help="adjoint workload: finite-difference directions")
    ap.add_argument("--adjoint-steps", type=int, default=10,
                    help="rt workload: steps of the adjoint run at the end")
    ap.add_argument("--no-full-crossing", action="store_true",
                    help="sine workload: skip the run to t = 1 (one crossing) for the L1 error")
    ap.add_argument("--no-extras", action="store_true",
                    help="sine workload: only the headline (no fast build, no per-step "
                         "parity at full size, no C1 / C3 / C4 / C5 sub-objects)")
    ap.add_argument("--variant", default="fast", choices=["exact", "fast"],
                    help="library build of the headline (sine workload; the other build is "
                         "measured beside it) or of the workload")
    ap.add_argument("--tile-rows", type=int, default=0,
                    help="sine workload: tile rows (8 or 16) instead of the autotuner's choice")
    ap.add_argument("--z-chunk", type=int, default=0,
                    help="sine workload: pencil length instead of the autotuner's choice")
    ap.add_argument("--bricks", type=int, default=512)
    ap.add_argument("--riemann", default="HLLC", choices=["HLLC", "HLL"],
                    help="sine workload: the Riemann solver (the benchmark's is HLLC)")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region,
    every 20 ms, with each sample's time, so that the samples that fall in
    the timed window can be told apart from those around it."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None
        time.sleep(0.3)

    def stop(self, window=None):
        """The summary of the samples; window = (t0, t1), host wall-clock
        seconds around the timed region, adds the samples inside it."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:  # noqa: BLE001
            self.proc.kill()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        return self.summarize(lines, window)

    @classmethod
    def summarize(cls, lines, window=None):
        """Median and maximum SM clock and the throttle reasons seen (any
        sample), and, for the samples whose time falls in window, their count
        and lowest SM clock."""
        import datetime

        rows = []
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [x for x in (num(r[2]) for r in rows) if x is not None]
        mx = [x for x in (num(r[3]) for r in rows) if x is not None]
        reasons = sorted({cls.REASONS[i] for r in rows for i in range(4) if r[6 + i] == "Active"})
        out = {"sm_mhz": statistics.median(sm) if sm else None,
               "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
               "samples": len(rows), "interval_ms": 20}
        if window is not None:
            t0, t1 = window
            inside = []
            for r in rows:
                try:
                    t = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                if t0 <= t <= t1 and num(r[2]) is not None:
                    inside.append(num(r[2]))
            out["timed_samples"] = len(inside)
            out["timed_sm_mhz_min"] = min(inside) if inside else None
        return out


def dist_init():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """The largest x over the ranks (the slowest replica's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    """The sum of x over the ranks (counts of the whole job)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return type(x)(t.item())


def replica_rate(cells, steps, ms_per_rank, world):
    """Whole-job cell-updates/s of independent replicas: every rank's cells
    over the slowest rank's time."""
    return world * cells * steps / (max_over_ranks(ms_per_rank, world) / 1000.0)


def cpu_step_rate(n, steps, warmup=1):
    """The CPU oracle on an n^3 sine-wave brick: cell-updates/s over `steps`
    RK2 steps (after `warmup` untimed ones), all host threads."""
    from genasis_b200 import problems
    from oracle.oracle import Oracle

    cfg, prim = problems.sine_wave(n)
    o = Oracle(cfg)
    o.set_primitive(prim)
    i = 0
    for _ in range(warmup):
        o.step(o.timestep(i))
        i += 1
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(o.timestep(i))
        i += 1
    el = time.perf_counter() - t0
    return n ** 3 * steps / el, el, Oracle.n_threads()


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # a bounded sample of the workload per step: the largest cube whose step
    # keeps the whole run within a few minutes (calibrated on one step)
    rate, _, cores = cpu_step_rate(64, 1, warmup=0)
    budget_s = 150.0
    n = args.n
    while n > 32 and (n ** 3) * (args.steps + args.warmup) / rate > budget_s:
        n //= 2
    value, el, cores = cpu_step_rate(n, args.steps, warmup=args.warmup)
    sample = ("%d RK2 steps (after %d warm-up) of a %d^3 brick of the sine-wave workload "
              "(HLLC, periodic), per-cell cost independent of brick size" %
              (args.steps, args.warmup, n))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "sine_wave_%d" % args.n, "sample_cells": n ** 3,
                   "riemann": "HLLC", "boundary": "periodic", "cfl": 0.8},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp64_peak(reps=10, iters=4096):
    """The device's FP64 rate (FLOP/s, a fused multiply-add counting two):
    genasis_b200/libgfx_probe.so times chains of fused multiply-adds on every
    SM, best of `reps` launches of `iters` steps per chain (4096 steps take
    about 0.55 ms on a B200)."""
    import ctypes

    try:
        probe = ctypes.CDLL(os.path.join(ROOT, "genasis_b200", "libgfx_probe.so"))
        f, ms = ctypes.c_double(), ctypes.c_double()
        if probe.gfx_probe_fp64_chains(int(reps), int(iters), ctypes.byref(f),
                                       ctypes.byref(ms)) == 0:
            return f.value
    except OSError:
        pass
    return None


def fp64_counts(variant, riemann, kernel):
    """FP64 operations per cell of a stage kernel launch, counted by ncu
    (profiles/stage_fp64.json: dadd + dmul + 2 dfma thread instructions,
    predicated on, per cell of the captured launch)."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage_fp64.json")) as f:
            return json.load(f)[variant][riemann][kernel]
    except Exception:  # noqa: BLE001
        return None


def _stage_profile(kernel):
    path = os.path.join(ROOT, "profiles", "stage_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)[kernel]
    except Exception:  # noqa: BLE001
        return {}


def traffic_per_launch(kernel, cells):
    """DRAM bytes per launch of the stage kernel from the committed ncu summary
    (bytes per cell measured on a smaller case, scaled by the cells)."""
    per_cell = _stage_profile(kernel).get("dram_bytes_per_cell")
    return per_cell * cells if per_cell is not None else None


def pipe_use(kernel):
    """FP64 pipe and issue activity of the stage kernel from the committed
    ncu capture: what bounds it instead of HBM."""
    p = _stage_profile(kernel)
    return {"fp64_pipe_active": p.get("fp64_pipe_active"), "issue_active": p.get("issue_active"),
            "source": "profiles/stage_traffic.json (ncu, 160^3)"}


def _timed_evolve(box, steps, warmup, local, world):
    """Warm-up cycles (they also capture the cycle graph), then `steps` cycles
    of gfx_fluid_evolve timed with CUDA events on the launching stream between
    barriers, with the clocks sampled meanwhile.  The sampler starts first;
    then the FP64 probe of the roofline runs (about 0.2 s of full load), so
    that the device is at its running clock, not ramping up from idle, when
    the warm-up cycles and the timed region follow without a gap.  The events
    are the ones gfx_fluid_evolve_timed records just before its first and
    after its last launch (a host delay before the call's first launch, or
    before it returns, would otherwise count as device time); events around
    the call are kept beside them as "ms_call"."""
    import torch

    stream = torch.cuda.current_stream()
    sampler = ClockSampler(local)
    sampler.start()
    fp64 = fp64_peak(reps=20, iters=20 * 4096)
    t_sim, cyc = box.evolve(1e30, 0.0, 0, max_cycles=max(warmup, 3))
    torch.cuda.synchronize()
    launches0 = box.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    ev0.record(stream)
    t_sim, cyc2, ms = box.evolve_timed(1e30, t_sim, cyc, max_cycles=steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    barrier(world)
    clocks = sampler.stop(window=(w0, w1))
    return {"ms": ms, "ms_call": ev0.elapsed_time(ev1), "steps": cyc2 - cyc, "t_sim": t_sim,
            "cycle": cyc2, "launches": box.kernel_launches() - launches0, "clocks": clocks,
            "fp64": fp64}


def _sine_box(args, cfg, prim, variant):
    """The 256^3 sine-wave brick of a library build, with the autotuner's tile
    and pencil (or the command line's), initialised from prim."""
    from genasis_b200 import autotune
    from genasis_b200.fluid import FluidBox

    if args.tile_rows or args.z_chunk:
        box = FluidBox(cfg, variant=variant)
        box.set_tuning(args.z_chunk, 0, args.tile_rows)
    else:
        box = autotune.tuned_box(cfg, adjoint=False, variant=variant)
    box.compute_from_primitive(prim)
    return box


def _sine_l1(box, cfg, t):
    from genasis_b200 import problems

    prim_t, _ = box.compute_from_conserved(primitive=True)
    l1 = problems.l1_error(prim_t[0].cpu().numpy(), problems.sine_density(cfg, t), cfg)
    del prim_t
    return l1


def _oracle_sine(n, steps, warmup=1, riemann="HLLC"):
    """The CPU oracle on the n^3 sine wave: `warmup` untimed steps, then
    `steps` timed ones, all host threads; returns the rate, the seconds, the
    threads, and the last timed step as (state before it, cycle, dt, state
    after it) for the per-step parity of the GPU builds."""
    from genasis_b200 import problems
    from oracle.oracle import Oracle

    cfg, prim = problems.sine_wave(n, riemann_solver=riemann, courant=0.8, n_ramp_cycles=1)
    o = Oracle(cfg)
    o.set_primitive(prim)
    i = 0
    for _ in range(warmup):
        o.step(o.timestep(i))
        i += 1
    el = 0.0
    before = None
    for k in range(steps):
        dt = o.timestep(i)
        if k == steps - 1:
            before = (o.conserved(), i, dt)
        t0 = time.perf_counter()
        o.step(dt)
        el += time.perf_counter() - t0
        i += 1
    return n ** 3 * steps / el, el, Oracle.n_threads(), before + (o.conserved(),)


def _field_errors(a, b, idx):
    """max |a - b| per field over idx, relative to the field's max |b|."""
    import numpy as np

    return [float(np.abs(a[f][idx] - b[f][idx]).max()) /
            max(float(np.abs(b[f][idx]).max()), 1e-300) for f in range(a.shape[0])]


def _quantity_errors(a, b, idx):
    """As _field_errors, with each momentum component relative to the largest
    momentum component's max (the momentum vector's scale)."""
    import numpy as np

    scale = [max(float(np.abs(b[f][idx]).max()), 1e-300) for f in range(b.shape[0])]
    scale[1:4] = [max(scale[1:4])] * 3
    return [float(np.abs(a[f][idx] - b[f][idx]).max()) / scale[f] for f in range(a.shape[0])]


def _step_parity(box, cfg, before):
    """One GPU step from the oracle's state before its last timed step (the
    same dt, features detected from that state) against the oracle's result:
    errors per field (relative to the field's max) and per quantity
    (momentum components relative to the momentum vector's max), and the
    CFL time step of the state against the oracle's."""
    import numpy as np
    import torch

    U_prev, cycle, dt, U_next = before
    box.set_conserved(torch.as_tensor(U_prev, device="cuda"))
    box.detect_features()
    dt_g = box.compute_time_step(cycle)
    box.step(dt)
    g = box.U.cpu().numpy()
    p = cfg.proper
    fe = _field_errors(g, U_next, p)
    qe = _quantity_errors(g, U_next, p)
    bitwise = [bool(np.array_equal(g[f][p], U_next[f][p])) for f in range(6)]
    del g
    return {"max_rel_err_per_field": fe, "max_rel_err_per_quantity": qe,
            "max_rel_err": max(fe), "within_1e-12": max(fe) <= 1e-12,
            "bitwise_equal_fields": bitwise, "dt_rel_diff": abs(dt_g - dt) / dt,
            "dt_equal": dt_g == dt}


def _stage_timing(box, cfg, cyc, steps, fp64_rate=None):
    """Per-kernel device times of an evolve cycle's kernels (CUDA events per
    launch, gfx_fluid_step_timed) and the roofline of the dominant stage,
    with its FP64 rate against the measured FP64 peak beside the HBM one."""
    cells = cfg.n_proper
    dt = box.compute_time_step(cyc)
    per = {"features": [], "stage1": [], "stage2": [], "ghosts": []}
    for _ in range(min(steps, 10)):
        f, s1, s2, gh = box.step_timed(dt)
        per["features"].append(f)
        per["stage1"].append(s1)
        per["stage2"].append(s2)
        per["ghosts"].append(gh)
    avg = {k: sum(v) / len(v) for k, v in per.items()}
    dom = max(("stage1", "stage2"), key=lambda k: avg[k])
    peak, peak_kind = peaks()
    achieved = STAGE_BYTES[dom] * cells / (avg[dom] / 1000.0) / 1e9
    roof = {
        "bound": "hbm", "kernel": "stage_kernel (%s)" % dom, "achieved": achieved,
        "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": traffic_per_launch(dom, cells), "peak_source": peak_kind,
        "algorithmic_bytes_per_cell": STAGE_BYTES[dom], "avg_launch_ms": avg[dom],
        "kernel_ms": avg}
    riemann = cfg.riemann_solver if isinstance(cfg.riemann_solver, str) else "HLLC"
    counts = fp64_counts(box.variant, riemann, dom)
    if counts is not None:
        # the DRAM bytes of this build's launch, per cell, scaled to the cells
        roof["traffic"] = counts["dram_bytes_per_cell"] * cells
        roof["traffic_source"] = "profiles/stage_fp64.json (ncu at 160^3, per cell x cells)"
        per_cell = counts["fp64_ops_per_cell"]
        rate = per_cell * cells / (avg[dom] / 1000.0)
        roof["fp64"] = {"ops_per_cell": per_cell, "achieved_tflops": rate / 1e12,
                        "peak_tflops": fp64_rate / 1e12 if fp64_rate else None,
                        "frac": rate / fp64_rate if fp64_rate else None,
                        "peak_source": "measured by genasis_b200/libgfx_probe.so (chains of "
                                       "fused multiply-adds, best of 20 launches of about "
                                       "11 ms run right before the warm-up cycles)",
                        "counts_source": "profiles/stage_fp64.json (ncu thread instructions "
                                         "dadd + dmul + 2 dfma, %s)" % counts.get("case", "")}
    return dt, avg, dom, roof


def run_ours(args):
    import torch

    world, rank, local = dist_init()
    from genasis_b200 import problems

    cfg, prim = problems.sine_wave(args.n, riemann_solver=args.riemann, courant=0.8,
                                   n_ramp_cycles=1)
    cells = cfg.n_proper
    box = _sine_box(args, cfg, prim, args.variant)
    t = _timed_evolve(box, args.steps, args.warmup, local, world)
    ms, steps_done, t_sim, cyc2 = t["ms"], t["steps"], t["t_sim"], t["cycle"]
    ms_max = max_over_ranks(ms, world)
    ms_call_max = max_over_ranks(t["ms_call"], world)
    value = replica_rate(cells, steps_done, ms, world)
    # L1 density error against the exact translated profile at the end of the
    # timed region (before the extra steps below move the state on)
    l1 = _sine_l1(box, cfg, t_sim)

    rate64 = t["fp64"] or fp64_peak()
    dt, avg, dom, roofline = _stage_timing(box, cfg, cyc2, args.steps, rate64)
    roofline["step_hbm_frac"] = STEP_BYTES * value / world / 1e9 / roofline["peak"]
    roofline["ncu_pipes"] = pipe_use(dom)

    # end to end: H2D of the state from pinned host memory, the step, D2H
    e2e = None
    if not args.no_e2e:
        host = box.U.detach().cpu().pin_memory()
        nbytes = host.numel() * host.element_size()
        # gfx_fluid_step_host copies in the fields D, S1, S2, S3, G (DS is
        # rewritten by the step and never read) and copies back all six
        h2d = nbytes * 5 // 6
        n_e = max(3, min(args.steps, 20))
        box.step_host(host, dt)
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(n_e):
            box.step_host(host, dt)
        el = time.perf_counter() - t0
        el = max_over_ranks(el, world)
        e2e = {"value": world * cells * n_e / el, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": nbytes, "steps": n_e,
               "how": "gfx_fluid_step_host on a pinned host state, pipelined over z slabs"}
        del host

    single = rank == 0 and world == 1
    extras = single and not args.no_extras
    crossing = None
    if extras and not args.no_full_crossing:
        # on to t = 1 (one box crossing), the last step cut to land on it
        box.compute_from_primitive(prim)
        t_end, c_end = box.evolve(1.0, 0.0, 0)
        torch.cuda.synchronize()
        crossing = {"time": t_end, "cycles": c_end, "l1_density_error": _sine_l1(box, cfg, t_end),
                    "norm": "sum |rho - rho_exact| / sum |rho_exact| over proper cells"}

    cpu = parity = None
    if single and not args.no_cpu_baseline:
        rate, el, cores, before = _oracle_sine(args.n, 2, warmup=1, riemann=args.riemann)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "2 RK2 steps (after 1 warm-up) of the %d^3 sine-wave workload on the "
                         "CPU oracle (the C restatement, -O3 -ffp-contract=off; not GenASiS's "
                         "Fortran), %.1f s" % (args.n, el)}
        parity = {"workload": "sine_wave_%d" % args.n,
                  "how": "one GPU step from the oracle's state before its last timed step, "
                         "same dt, against the oracle's result, proper cells",
                  args.variant: _step_parity(box, cfg, before)}
    box.close()
    del box
    torch.cuda.empty_cache()

    fast = None
    if extras:
        other = "fast" if args.variant == "exact" else "exact"
        fb = _sine_box(args, cfg, prim, other)
        tf = _timed_evolve(fb, args.steps, args.warmup, local, world)
        vf = cells * tf["steps"] / (tf["ms"] / 1000.0)
        l1_f = _sine_l1(fb, cfg, tf["t_sim"])  # before the timed steps below move it on
        _, avg_f, dom_f, roof_f = _stage_timing(fb, cfg, tf["cycle"], args.steps, rate64)
        fast = {"variant": other, "library": "genasis_b200/" + (
                    "libgfx_fluid_fast.so" if other == "fast" else "libgfx_fluid.so"),
                "value": vf, "unit": UNIT, "ms_per_step": tf["ms"] / tf["steps"],
                "steps": tf["steps"], "roofline": roof_f,
                "step_hbm_frac": STEP_BYTES * vf / 1e9 / roof_f["peak"],
                "clocks": tf["clocks"], "gpu_launches": tf["launches"],
                "l1_density_error": l1_f}
        if parity is not None:
            parity[other] = _step_parity(fb, cfg, before)
        fb.close()
        del fb
        torch.cuda.empty_cache()
    del prim

    configs = None
    if extras:
        configs = {}
        v = args.variant
        # C1's free run is the bitwise check: it runs on the exact build
        for key, fn in (("c1_sod", lambda: sod_result(128, 100, "exact")),
                        ("c3_bricks", lambda: bricks_result(50, 3, 512, v)),
                        ("c4_adjoint", lambda: adjoint_result(128, 64, 3, True, v)),
                        ("c5_rt", lambda: rt_result(200, 3, 10, v)),
                        # the chart against the single brick: bit for bit on the exact
                        # build (the same arithmetic on every cell); the fast build's
                        # chart kernels may fuse differently from its single-brick ones
                        ("chart_2x2x2", lambda: chart_result(args.n, (2, 2, 2), args.steps,
                                                             args.warmup, "exact")),
                        ("chart_2x2x2_fast", lambda: chart_result(args.n, (2, 2, 2),
                                                                  args.steps, args.warmup,
                                                                  "fast"))):
            t0 = time.perf_counter()
            try:
                configs[key] = fn()
            except Exception as e:  # noqa: BLE001 -- reported, the headline stands
                configs[key] = {"error": "%s: %s" % (type(e).__name__, e)}
            configs[key]["wall_s"] = time.perf_counter() - t0
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps_done, "warmup": max(args.warmup, 3),
            "ms_per_step": ms_max / steps_done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "sine_wave_%d" % args.n, "cells": cells,
                       "riemann": args.riemann,
                       "reconstruction": "PLM theta 1.4", "boundary": "periodic",
                       "cfl": 0.8, "rk": 2, "parallelism": "replicas" if world > 1 else "single",
                       "library": args.variant,
                       "l2": "inputs larger than L2 (state %.0f MB)" % (
                           6 * (args.n + 4) ** 3 * 8 / 1e6),
                       "l1_density_error": l1, "sim_time": t_sim,
                       "full_crossing": crossing,
                       "tuning": _tuning_of(args, cfg),
                       "timing": "CUDA events on the launching stream, recorded by "
                                 "gfx_fluid_evolve_timed just before its first and after its "
                                 "last launch; ms_per_step_call: events around the call"},
            "ms_per_step_call": ms_call_max / steps_done,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": t["launches"],
            "clocks": t["clocks"],
            "parity": parity,
            "other_build": fast,
            "configs": configs,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def _tuning_of(args, cfg):
    from genasis_b200 import autotune

    if args.tile_rows or args.z_chunk:
        return {"z_chunk": args.z_chunk, "tile": "32x%d" % (args.tile_rows or 16)}
    e = autotune.load_cache().get(autotune.brick_key(cfg, args.variant), {})
    return {"z_chunk": e.get("z_chunk"), "tile": "32x%s" % e.get("tile_rows")}


def bricks_result(steps=50, warmup=3, n_bricks=512, variant="exact", world=1, rank=0):
    """512 independent bricks, edges U{16..96} per axis (seeded), seeded
    two-state Riemann problems, outflow, PLM + HLL, RK2, CFL 0.8: K cycles of
    the batched path (one persistent launch per stage, one graph per cycle)
    against K cycles of each brick's own single-brick path, brick after brick,
    each timed with CUDA events.  With world > 1 ranks (one per GPU) the
    bricks are split over the ranks (genasis_b200.batch.shard_bricks), each
    rank advances its own with no data exchange, and the times are the
    slowest rank's."""
    import torch

    from genasis_b200 import problems
    from genasis_b200.batch import FluidBatch, shard_bricks

    if world == 1:
        torch.cuda.set_device(0)
    all_cfgs = [c for c, _ in problems.random_bricks(count=n_bricks, seed=20261203,
                                                      riemann_solver="HLL", only=set())]
    mine = shard_bricks(all_cfgs, world, rank)
    bricks = problems.random_bricks(count=n_bricks, seed=20261203, riemann_solver="HLL",
                                    only=set(mine))
    cfgs = [bricks[i][0] for i in mine]
    prims = [bricks[i][1] for i in mine]
    del bricks
    cells = sum(c.n_proper for c in all_cfgs)
    cells_mine = sum(c.n_proper for c in cfgs)
    batch = FluidBatch(cfgs, variant=variant)
    K = steps
    # the pencil length of the batch's work items: autotuned (cached per GPU
    # and brick set), outside the timed region
    from genasis_b200 import autotune

    t_tune = time.perf_counter()
    z_chunk, tune_ms, from_cache = autotune.tune_batch(batch, prims)
    t_tune = time.perf_counter() - t_tune
    # warm-up (graph capture) on a copy of the initial states, then reset
    batch.set_primitives(prims)
    batch.evolve(n_cycles=max(warmup, 3))
    torch.cuda.synchronize()
    batch.set_primitives(prims)
    batch.set_clocks(0.0, 0)
    torch.cuda.synchronize()
    barrier(world)
    l0 = batch.kernel_launches()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    batch.evolve(n_cycles=K)
    e[1].record()
    torch.cuda.synchronize()
    t_batch = e[0].elapsed_time(e[1]) / 1000.0
    launches_batch = batch.kernel_launches() - l0
    U_batch = [b.U.clone() for b in batch.boxes]
    # the same bricks through the single-brick path, one after another
    for b, p in zip(batch.boxes, prims):
        b.compute_from_primitive(p)
        b.evolve(1e300, 0.0, 0, max_cycles=2)
    for b, p in zip(batch.boxes, prims):
        b.compute_from_primitive(p)
    torch.cuda.synchronize()
    barrier(world)
    l1 = sum(b.kernel_launches() for b in batch.boxes)
    e[2].record()
    for b in batch.boxes:
        b.evolve(1e300, 0.0, 0, max_cycles=K)
    e[3].record()
    torch.cuda.synchronize()
    t_plain = e[2].elapsed_time(e[3]) / 1000.0
    launches_plain = sum(b.kernel_launches() for b in batch.boxes) - l1
    same = all(torch.equal(a, b.U) for a, b in zip(U_batch, batch.boxes))
    # the job's figures: the slowest rank's times, every rank's launches, and
    # the batch equal to the loop on every rank (the same steps on all ranks)
    t_batch = max_over_ranks(t_batch, world)
    t_plain = max_over_ranks(t_plain, world)
    launches_batch = sum_over_ranks(launches_batch, world)
    launches_plain = sum_over_ranks(launches_plain, world)
    same = max_over_ranks(0.0 if same else 1.0, world) == 0.0
    line = {
        "metric": "FP64 cell-updates/s (batched bricks)", "value": cells * K / t_batch,
        "unit": UNIT, "n_gpus": world, "steps": K, "warmup": max(warmup, 3),
        "ms_per_step": 1000.0 * t_batch / K, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "bricks_%d" % n_bricks, "cells": cells, "riemann": "HLL",
                   "boundary": "outflow", "cfl": 0.8, "edges": "U{16..96}", "seed": 20261203,
                   "library": variant,
                   "parallelism": ("bricks split over %d ranks by proper cells, no data "
                                   "exchange" % world) if world > 1 else "single",
                   "cells_this_rank": cells_mine, "bricks_this_rank": len(mine),
                   "plain_loop": "each brick's own gfx_fluid_evolve (a graph per cycle), "
                                 "brick after brick"},
        "plain_loop": {"value": cells * K / t_plain, "ms_per_step": 1000.0 * t_plain / K,
                       "gpu_launches": launches_plain},
        "speedup_vs_plain_loop": t_plain / t_batch,
        "autotune": {"tile": "32x%d" % z_chunk[0], "z_chunk": z_chunk[1],
                     "ms_per_cycle_by_candidate": tune_ms, "from_cache": from_cache,
                     "tuning_s": t_tune},
        "bitwise_equal_to_plain": same,
        "gpu_launches": launches_batch,
    }
    batch.close()
    return line


def stage_roofline(box, cells, dt, n):
    """CUDA-event times of the phases of n steps (gfx_fluid_step_timed) and
    the roofline of the dominant stage kernel."""
    per = {"features": [], "stage1": [], "stage2": [], "ghosts": []}
    for _ in range(n):
        f, s1, s2, gh = box.step_timed(dt)
        per["features"].append(f)
        per["stage1"].append(s1)
        per["stage2"].append(s2)
        per["ghosts"].append(gh)
    avg = {k: sum(v) / len(v) for k, v in per.items()}
    dom = max(("stage1", "stage2"), key=lambda k: avg[k])
    peak, peak_kind = peaks()
    achieved = STAGE_BYTES[dom] * cells / (avg[dom] / 1000.0) / 1e9
    return {"bound": "hbm", "kernel": "stage_kernel (%s)" % dom, "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_per_launch(dom, cells), "peak_source": peak_kind,
            "algorithmic_bytes_per_cell": STAGE_BYTES[dom], "avg_launch_ms": avg[dom],
            "kernel_ms": avg}


def run_adjoint_step(args):
    """A short run for profiling the adjoint: the n^3 Kelvin-Helmholtz state
    (default 128^3), two forward steps, then --steps calls of
    gfx_fluid_step_adjoint on the last step (U^n+1 given, features detected),
    timed with CUDA events."""
    import torch

    from genasis_b200 import problems
    from genasis_b200.adjoint import cell_volumes, step_adjoint
    from genasis_b200.fluid import FluidBox

    torch.cuda.set_device(0)
    n = args.n if args.n != 256 else 128
    cfg, prim = problems.kelvin_helmholtz(n)
    box = FluidBox(cfg, variant=args.variant)
    box.compute_from_primitive(prim)
    box.compute_from_conserved()
    dts = []
    for i in range(2):
        dts.append(box.compute_time_step(i))
        box.step(dts[-1])
    U0 = box.U.clone()
    box.step(dts[-1])
    U1 = box.U.clone()
    lam = torch.zeros_like(U1)
    lam[0] = 2.0 * U1[0] * cell_volumes(box)
    out = torch.empty_like(U1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step_adjoint(box, U0, dts[-1], lam, out, U1, True)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"workload": "kelvin_helmholtz_%d_adjoint_step" % n, "steps": args.steps,
                      "ms_per_adjoint_step": e0.elapsed_time(e1) / args.steps}), flush=True)
    box.close()


def sod_result(n=128, steps=100, variant="exact"):
    """The plain method at its small configuration: the 3-D Sod tube on n^3
    cells (left rho = 1, p = 1; right rho = 0.125, p = 0.1; diaphragm x = 0.5),
    PLM + HLL, RK2, CFL 0.8, outflow, `steps` steps (100) on the GPU and on
    the oracle side by side: per-step parity from identical inputs on the
    first steps, the final states of the two free runs, and both rates."""
    import numpy as np
    import torch

    from genasis_b200 import problems
    from genasis_b200.config import FluidConfig
    from genasis_b200.fluid import FluidBox
    from oracle.oracle import Oracle

    torch.cuda.set_device(0)
    cfg = FluidConfig(n_cells=(n, n, n), riemann_solver="HLL", courant_factor=0.8,
                      n_ramp_cycles=1)
    prim = problems.riemann(cfg, 1.0, 1.0, (0, 0, 0), 0.125, 0.1, (0, 0, 0), (0.5, 0, 0),
                            (1.0, 0, 0))
    p = cfg.proper
    box = FluidBox(cfg, variant=variant)
    box.compute_from_primitive(prim)
    o = Oracle(cfg)
    o.set_primitive(prim)

    def rel(a, b):
        return max(float(np.abs(a[f][p] - b[f][p]).max()) / max(float(np.abs(b[f][p]).max()),
                                                                 1e-300) for f in range(5))

    per_step = []
    gpu_ms = 0.0
    cpu_s = 0.0
    dts = []
    for i in range(steps):
        dt = o.timestep(i)
        dts.append(dt)
        if i < 3:  # per-step parity: the GPU step from the oracle's state
            box.set_conserved(torch.as_tensor(o.conserved(), device="cuda"))
            if i > 0:
                box.detect_features()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        box.step(dt)
        e1.record()
        t0 = time.perf_counter()
        o.step(dt)
        cpu_s += time.perf_counter() - t0
        torch.cuda.synchronize()
        gpu_ms += e0.elapsed_time(e1)
        if i < 3:
            per_step.append(rel(box.U.cpu().numpy(), o.conserved()))
    Ug = box.U.cpu().numpy()
    Uo = o.conserved()
    line = {
        "workload": "sod_%d_hll_%d_steps" % (n, steps), "cells": cfg.n_proper,
        "library": variant,
        "per_step_max_rel_diff_first_3_steps": per_step,
        "final_max_rel_diff_free_runs": rel(Ug, Uo),
        "final_bitwise_equal_fields": [bool(np.array_equal(Ug[f][p], Uo[f][p])) for f in range(6)],
        "gpu_cell_updates_per_s": cfg.n_proper * steps / (gpu_ms / 1000.0),
        "gpu_timing": "CUDA events around each gfx_fluid_step (a host synchronisation per "
                      "step for the oracle's dt)",
        "cpu_oracle_cell_updates_per_s": cfg.n_proper * steps / cpu_s,
        "cpu_threads": Oracle.n_threads(), "sim_time": float(sum(dts)),
    }
    box.close()
    return line


def rt_result(steps=200, warmup=3, adjoint_steps=10, variant="exact"):
    """3-D Rayleigh-Taylor on 384 x 384 x 768 cells ([0,0.5]^2 x [0,1]),
    gravity 0.1 along -z as a source in the RK stages, periodic x / y,
    reflecting z, PLM + HLLC, RK2, CFL 0.8: throughput over `steps` cycles
    with the HBM roofline of the stage kernel and the mass balance, then the
    adjoint of the last `adjoint_steps` steps (per-step checkpoints, stage
    recomputation) against the forward time of the same steps."""
    import torch

    from genasis_b200 import autotune, problems
    from genasis_b200.adjoint import cell_volumes, run_adjoint, run_forward

    torch.cuda.set_device(0)
    cfg, prim = problems.rayleigh_taylor()
    cells = cfg.n_proper

    box = autotune.tuned_box(cfg, adjoint=False, variant=variant)
    box.compute_from_primitive(prim)
    del prim
    dv = cell_volumes(box)
    p = cfg.proper
    mass0 = float((box.U[0][p] * dv[p]).sum())
    t_sim, cyc = box.evolve(1e30, 0.0, 0, max_cycles=max(warmup, 3))
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    l0 = box.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record()
    t_sim, cyc2 = box.evolve(1e30, t_sim, cyc, max_cycles=steps)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop(window=(w0, time.time()))
    launches = box.kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    n_done = cyc2 - cyc
    mass1 = float((box.U[0][p] * dv[p]).sum())
    dt = box.compute_time_step(cyc2)
    roof = stage_roofline(box, cells, dt, 5)
    def adjoint_cost(bx, U0, dts):
        # an untimed forward and adjoint first: the checkpoints, the adjoint's
        # workspace (20 values per cell, allocated by the handle's first
        # adjoint step) and the adjoint arrays take their memory once, so that
        # the timed run measures the steps
        final, cps = run_forward(bx, U0, dts, True)
        lam = torch.zeros_like(final)
        lam[0] = 2.0 * final[0] * dv
        grad = run_adjoint(bx, cps, dts, lam, True)
        del final, cps, lam, grad
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        final, cps = run_forward(bx, U0, dts, True)
        e[1].record()
        lam = torch.zeros_like(final)
        lam[0] = 2.0 * final[0] * dv
        grad = run_adjoint(bx, cps, dts, lam, True)
        e[2].record()
        torch.cuda.synchronize()
        out = {"library": bx.variant, "steps": len(dts), "forward_ms": e[0].elapsed_time(e[1]),
               "adjoint_ms": e[1].elapsed_time(e[2]),
               "adjoint_over_forward": e[1].elapsed_time(e[2]) / e[0].elapsed_time(e[1]),
               "objective": "sum rho^2 dV",
               "gradient_finite": bool(torch.isfinite(grad).all())}
        del cps, grad, final, lam
        return out

    adj = None
    if adjoint_steps > 0:
        U0 = box.U.clone()
        dts = []
        for i in range(adjoint_steps):
            dts.append(box.compute_time_step(cyc2 + i))
            box.step(dts[-1])
        adj = adjoint_cost(box, U0, dts)
        # the same steps' adjoint on the other library build, from the same
        # state with the same time steps
        other = "exact" if variant == "fast" else "fast"
        box.close()
        torch.cuda.empty_cache()
        box = autotune.tuned_box(cfg, adjoint=False, variant=other)
        adj["other_build"] = adjoint_cost(box, U0, dts)
        del U0
    value = cells * n_done / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": n_done,
        "warmup": max(warmup, 3), "ms_per_step": ms / n_done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "rayleigh_taylor_384x384x768", "cells": cells,
                   "riemann": "HLLC", "gravity": 0.1, "boundary": "periodic x/y, reflecting z",
                   "cfl": 0.8, "sim_time": t_sim, "library": variant,
                   "l2": "inputs larger than L2 (state %.1f GB)" % (6 * (384 + 4) ** 2 *
                                                                       (768 + 4) * 8 / 1e9),
                   "mass_rel_change": (mass1 - mass0) / mass0},
        "roofline": roof, "step_hbm_frac": STEP_BYTES * value / 1e9 / roof["peak"],
        "adjoint": adj, "gpu_launches": launches, "clocks": clocks,
    }
    box.close()
    return line


def chart_result(n=256, n_bricks=(2, 2, 2), steps=20, warmup=3, variant="exact"):
    """The sine-wave workload on n^3 cells as a chart of n_bricks bricks
    (Chart_SLD's decomposition, all bricks on this device): cycles of the
    chart's evolve timed with CUDA events, and the final state against the
    single n^3 brick after the same cycles (bit for bit)."""
    import numpy as np
    import torch

    from genasis_b200 import problems
    from genasis_b200.chart import FluidChart
    from genasis_b200.fluid import FluidBox

    torch.cuda.set_device(0)
    cfg, prim = problems.sine_wave(n, riemann_solver="HLLC", courant=0.8, n_ramp_cycles=1)
    chart = FluidChart(cfg, n_bricks, variant=variant)
    chart.from_primitive(prim)
    t_sim, cyc = chart.evolve(1e30, 0.0, 0, max_cycles=max(warmup, 3))
    l0 = chart.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    t_sim, cyc2 = chart.evolve(1e30, t_sim, cyc, max_cycles=steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = chart.kernel_launches() - l0
    got = chart.gather()
    chart.close()
    del chart
    torch.cuda.empty_cache()
    box = FluidBox(cfg, variant=variant)
    box.compute_from_primitive(prim)
    t_b, c_b = box.evolve(1e30, 0.0, 0, max_cycles=cyc2)
    ref = box.U.cpu().numpy()
    box.close()
    p = cfg.proper
    same = [bool(np.array_equal(got[f][p], ref[f][p])) for f in range(6)]
    scale = [max(float(np.abs(ref[f][p]).max()), 1e-300) for f in range(6)]
    diff = [float(np.abs(got[f][p] - ref[f][p]).max()) / scale[f] for f in range(6)]
    return {"workload": "sine_wave_%d_chart_%dx%dx%d" % ((n,) + tuple(n_bricks)),
            "max_rel_diff_to_single_brick": diff,
            "bricks": int(np.prod(n_bricks)), "brick_cells": [n // b for b in n_bricks],
            "library": variant, "value": cfg.n_proper * (cyc2 - cyc) / (ms / 1000.0),
            "unit": UNIT, "steps": cyc2 - cyc, "ms_per_step": ms / (cyc2 - cyc),
            "gpu_launches": launches, "cycles_compared": cyc2,
            "bitwise_equal_to_single_brick": same, "time_equal": t_b == t_sim}


def _adjoint_cost(cfg, prim, n_steps, variant, reps=3):
    """Forward (with per-step checkpoints) and adjoint milliseconds of
    n_steps steps from prim, J = sum rho^2 dV, on one library build: the
    medians of reps timed runs after one untimed run."""
    import torch

    from genasis_b200 import autotune
    from genasis_b200.adjoint import cell_volumes, run_adjoint, run_forward

    box = autotune.tuned_box(cfg, adjoint=True, variant=variant)
    box.compute_from_primitive(prim)
    box.compute_from_conserved()
    U0 = box.U.clone()
    dts = []
    for i in range(n_steps):
        dts.append(box.compute_time_step(i))
        box.step(dts[-1])
    dv = cell_volumes(box)
    fwd, adj = [], []
    for rep in range(reps + 1):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record()
        final, cps = run_forward(box, U0, dts, False)
        e[1].record()
        lam = torch.zeros_like(final)
        lam[0] = 2.0 * final[0] * dv
        run_adjoint(box, cps, dts, lam, False)
        e[2].record()
        torch.cuda.synchronize()
        if rep > 0:
            fwd.append(e[0].elapsed_time(e[1]))
            adj.append(e[1].elapsed_time(e[2]))
        del cps, final, lam
    box.close()
    f, a = statistics.median(fwd), statistics.median(adj)
    return {"library": variant, "forward_ms": f, "adjoint_ms": a, "adjoint_over_forward": a / f}


def _fd_check(box, cfg, U0, dts, grad, dv, directions, seed, eps=1e-6, rho_fn=None,
              flips=False):
    """Central differences (J(U0 + eps d) - J(U0 - eps d)) / (2 eps), J = sum
    rho^2 dV, along seeded unit directions over all six fields of the proper
    cells, formed cell by cell; returns the relative errors of the adjoint's
    directional derivatives and, with flips, for each direction whether the
    two forwards took different branches somewhere (their branch signatures,
    gfx_fluid_step_branches) and the kinds of decision whose counts differ."""
    import torch

    from genasis_b200.adjoint import BRANCH_KINDS, branch_signature, run_forward

    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    p = (slice(None),) + cfg.proper
    sig = {}
    if rho_fn is None:
        def rho_fn(U):
            if flips:
                sig["last"] = branch_signature(box, U, dts, False)
                return box.U[0].clone()
            return run_forward(box, U, dts, False, keep=False)[0][0]
    errs, flipped, kinds = [], [], {}
    for _ in range(directions):
        d = torch.zeros_like(U0)
        d[p] = torch.randn(d[p].shape, generator=gen, device="cuda", dtype=torch.float64)
        d /= torch.linalg.vector_norm(d)
        rp = rho_fn(U0 + eps * d)
        sp = sig.get("last")
        rm = rho_fn(U0 - eps * d)
        sm = sig.get("last")
        q = cfg.proper
        fd = float(((rp[q] - rm[q]) * (rp[q] + rm[q]) * dv[q]).sum() / (2.0 * eps))
        ad = float((grad * d).sum())
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
        if flips:
            flipped.append(sp[0] != sm[0])
            for k, name in enumerate(BRANCH_KINDS):
                if sp[1][k] != sm[1][k]:
                    kinds[name] = kinds.get(name, 0) + 1
    if flips:
        return errs, flipped, kinds
    return errs


def _fd_summary(errs, flipped, kinds):
    import numpy as np

    e = np.array(errs)
    f = np.array(flipped, dtype=bool)
    out = {"directions": int(len(e)), "within_1e-6": int((e <= 1e-6).sum()),
           "median_rel_err": float(np.median(e)), "max_rel_err": float(e.max()),
           "flipped_directions": int(f.sum()),
           "directions_by_kind_of_flip": kinds}
    if (~f).any():
        out["flip_free"] = {"directions": int((~f).sum()),
                            "within_1e-6": int((e[~f] <= 1e-6).sum()),
                            "median_rel_err": float(np.median(e[~f])),
                            "max_rel_err": float(e[~f].max())}
    if f.any():
        out["flipped"] = {"directions": int(f.sum()),
                          "within_1e-6": int((e[f] <= 1e-6).sum()),
                          "median_rel_err": float(np.median(e[f])),
                          "max_rel_err": float(e[f].max())}
    return out


def adjoint_result(n=128, directions=64, warmup=3, oracle_fd=True, variant="exact"):
    """128^3 periodic Kelvin-Helmholtz (density 2 / 1, shear +-0.5, vy =
    0.01 sin(4 pi x) + 1e-3 seeded noise, p = 2.5), PLM + HLLC, RK2, CFL 0.8,
    20 steps; J = sum rho^2 dV at the final time.  Times the forward run with
    per-step checkpoints against the adjoint run (stage recomputation), then
    checks the gradient against central differences (eps = 1e-6) along 64
    seeded directions, on this exact state and on the same state with 2e-2
    noise on every field."""
    import numpy as np
    import torch

    from genasis_b200 import autotune, problems
    from genasis_b200.adjoint import cell_volumes, run_adjoint, run_forward
    from genasis_b200.fluid import FluidBox

    torch.cuda.set_device(0)
    n_steps = 20
    out = {}
    for state in ("spec", "noisy"):
        cfg, prim = problems.kelvin_helmholtz(n)
        if state == "noisy":
            prim = problems.noisy(prim, amp=2e-2, seed=20261205)
        box = autotune.tuned_box(cfg, variant=variant)
        box.compute_from_primitive(prim)
        box.compute_from_conserved()
        U0 = box.U.clone()
        dts = []
        for i in range(n_steps):
            dts.append(box.compute_time_step(i))
            box.step(dts[-1])
        dv = cell_volumes(box)
        launches0 = box.kernel_launches()
        fwd, adj, fwd_plain = [], [], []
        for rep in range(max(warmup, 3) + 3):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            torch.cuda.synchronize()
            e[0].record()
            final, cps = run_forward(box, U0, dts, False)
            e[1].record()
            lam = torch.zeros_like(final)
            lam[0] = 2.0 * final[0] * dv
            grad = run_adjoint(box, cps, dts, lam, False)
            e[2].record()
            run_forward(box, U0, dts, False, keep=False)
            e[3].record()
            torch.cuda.synchronize()
            if rep >= max(warmup, 3):
                fwd.append(e[0].elapsed_time(e[1]))
                adj.append(e[1].elapsed_time(e[2]))
                fwd_plain.append(e[2].elapsed_time(e[3]))
            del cps
        launches = box.kernel_launches() - launches0
        errs, flipped, kinds = _fd_check(box, cfg, U0, dts, grad, dv, directions,
                                         seed=20261205, flips=True)
        errs_np = np.array(errs)
        entry = {
            "forward_ms": statistics.median(fwd), "adjoint_ms": statistics.median(adj),
            "forward_no_checkpoints_ms": statistics.median(fwd_plain),
            "adjoint_over_forward": statistics.median(adj) / statistics.median(fwd),
            "fd_directions": len(errs), "fd_within_1e-6": int((errs_np <= 1e-6).sum()),
            "fd_median_rel_err": float(np.median(errs_np)),
            "fd_max_rel_err": float(errs_np.max()),
            "fd_eps_1e-6": _fd_summary(errs, flipped, kinds),
        }
        if state == "noisy":
            # the same check at larger eps: at eps = 1e-6 a unit direction over
            # all 6 x n^3 values moves each value by ~1e-10, close to the
            # rounding floor of the differenced states
            sweep = {}
            for eps in (1e-7, 1e-5, 1e-4):
                e_s, f_s, k_s = _fd_check(box, cfg, U0, dts, grad, dv, 16, seed=20261207,
                                          eps=eps, flips=True)
                sweep["%g" % eps] = _fd_summary(e_s, f_s, k_s)
            entry["fd_eps_sweep"] = sweep
        if state == "noisy" and oracle_fd:
            # the reference-FD gradient: the oracle's step, on a 32^3 brick of
            # the same noisy state, 4 directions
            from oracle.oracle import Oracle

            cfg_s, prim_s = problems.kelvin_helmholtz(32)
            prim_s = problems.noisy(prim_s, amp=2e-2, seed=20261205)
            bs = FluidBox(cfg_s, variant=variant)
            bs.compute_from_primitive(prim_s)
            bs.compute_from_conserved()
            U0s = bs.U.clone()
            dts_s = []
            for i in range(n_steps):
                dts_s.append(bs.compute_time_step(i))
                bs.step(dts_s[-1])
            final_s, cps_s = run_forward(bs, U0s, dts_s, False)
            dvs = cell_volumes(bs)
            lam_s = torch.zeros_like(final_s)
            lam_s[0] = 2.0 * final_s[0] * dvs
            grad_s = run_adjoint(bs, cps_s, dts_s, lam_s, False)
            idx = [(np.arange(36) - 2) % 32 + 2] * 3

            def rho_oracle(U):
                Un = U.cpu().numpy()[:, idx[0]][:, :, idx[1]][:, :, :, idx[2]]
                o = Oracle(cfg_s)
                o.set_conserved(np.ascontiguousarray(Un))
                for dt in dts_s:
                    o.step(dt)
                return torch.as_tensor(o.conserved()[0], device="cuda")

            e_ref = _fd_check(bs, cfg_s, U0s, dts_s, grad_s, dvs, 4, seed=20261206,
                              rho_fn=rho_oracle)
            entry["oracle_fd_32cubed"] = {"directions": 4, "max_rel_err": max(e_ref)}
            bs.close()
        out[state] = entry
        box.close()
    spec = out["spec"]
    cfg_c, prim_c = problems.kelvin_helmholtz(n)
    other = _adjoint_cost(cfg_c, prim_c, n_steps, "exact" if variant == "fast" else "fast")
    line = {
        "metric": "adjoint/forward cost", "value": spec["adjoint_over_forward"],
        "unit": "x (adjoint ms / forward ms)", "n_gpus": 1, "steps": n_steps,
        "warmup": max(warmup, 3), "ms_per_step": spec["adjoint_ms"] / n_steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "kelvin_helmholtz_%d_adjoint" % n, "riemann": "HLLC",
                   "boundary": "periodic", "cfl": 0.8, "steps": n_steps,
                   "objective": "sum rho^2 dV", "checkpointing": "per step",
                   "fd_eps": 1e-6, "fd_seed": 20261205, "library": variant},
        "spec_state": spec, "noisy_state": out["noisy"],
        "other_build_cost": other,
        "gpu_launches": launches,
    }
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "sine":
        run_ours(args)
        return
    n = args.n if args.n != 256 else 128
    if args.workload == "bricks":
        world, rank, _ = dist_init()
        line = bricks_result(args.steps, args.warmup, args.bricks, args.variant, world, rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    elif args.workload == "adjoint":
        line = adjoint_result(n, args.directions, args.warmup, not args.no_cpu_baseline,
                              args.variant)
    elif args.workload == "adjoint_step":
        run_adjoint_step(args)
        return
    elif args.workload == "sod":
        line = sod_result(n, args.steps, args.variant)
    elif args.workload == "chart":
        line = chart_result(args.n, (2, 2, 2), args.steps, args.warmup, args.variant)
    else:
        line = rt_result(args.steps, args.warmup, args.adjoint_steps, args.variant)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
