"""Benchmark of the FSI step on the lid-driven cavity with a neo-Hookean sphere.

Workload (one "step" = one fluid_3d::step_forward of one scene): 64^3 cells,
unit cube, no-slip walls, lid u=(1,0,0) at z=1, fluid viscosity 0.01, sphere
of radius 0.2 at the centre with G=1, solid density 1, transition width
1.5 dx, 5 extrapolation layers.  Synthetic: the scene is fully defined by its
.cfg parameters.

Our arm times the plain FP64 form and the mixed form (FP32 V-cycles inside
FP64 refinement) on the device, then end to end through the C ABI with
host-side result reads.  Multi-GPU runs one independent scene per rank
(replicas: the path has no cross-scene exchange), timed as the max over ranks.

--impl reference times the reference's own CPU run_sim (oracle/_ref) on the
same .cfg, one process per host core, with the reference's own step timer.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from rmt3d_b200 import scenes  # noqa: E402

METRIC = "Mcell-steps/s"
RUN_SIM = os.path.join(ROOT, "oracle", "_ref", "run_sim")


def workload_cfg(n, steps):
    return scenes.cavity_sphere(n, steps, mu=0.01, G=1.0, rho=1.0, radius=0.2, wt_n=1.5, nlayers=5)


def config_block(n, l2):
    return {"workload": "lid-driven cavity %d^3 + neo-Hookean sphere R=0.2 G=1 (FP64 oracle parity form)" % n,
            "grid": n, "cells": n ** 3, "objects": 1, "l2": l2,
            "parallelism": "replicas (one scene per GPU)"}


# ---------------------------------------------------------------------------
# reference arm: the reference's own run_sim on the host cores
# ---------------------------------------------------------------------------
def reference_run(n, steps, procs):
    """Run `procs` copies of the reference run_sim, `steps` steps each; returns
    (cell-steps/s aggregate, per-process stepper seconds)."""
    wd = tempfile.mkdtemp(prefix="rmt3d_ref_")
    cfgs = []
    for p in range(procs):
        c = os.path.join(wd, "w%d.cfg" % p)
        scenes.write(c, workload_cfg(n, steps))
        cfgs.append(c)
    t0 = time.time()
    ps = [subprocess.Popen([RUN_SIM, c], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, cwd=wd)
          for c in cfgs]
    secs = []
    for pr in ps:
        out, _ = pr.communicate()
        m = re.search(r"Stepper: Done with everything, took a total\s+([0-9.eE+-]+) seconds", out)
        if pr.returncode != 0 or not m:
            raise RuntimeError("reference run_sim failed:\n" + out[-2000:])
        secs.append(float(m.group(1)))
    wall = time.time() - t0
    cellsteps = procs * steps * n ** 3
    return cellsteps / max(secs), secs, wall


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(RUN_SIM):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/run_sim is not built (needs the reference sources)"}))
        return
    procs = max(1, min(host_cores(), args.ref_procs))
    steps = max(1, args.ref_steps)
    rate, secs, wall = reference_run(args.size, steps, procs)
    value = rate / 1e6
    sample = "%d processes x %d steps of the %d^3 workload (reference stepper timer; set-up and the 5 pressure pre-iterations excluded)" % (
        procs, steps, args.size)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * max(secs) / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args.size, "n/a (CPU)"),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.p = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args):
    import numpy as np
    import torch

    import rmt3d_b200 as R

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n = args.size
    wd = tempfile.mkdtemp(prefix="rmt3d_bench_")
    cfg = scenes.write(os.path.join(wd, "w.cfg"), workload_cfg(n, 100000))
    stream = torch.cuda.Stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def make(precision):
        d = R.desc_from_cfg(cfg)
        d.precision = precision
        sc = R.Scene(d, stream=stream.cuda_stream)
        sc.prepare()
        return sc

    def timed(sc, k, e2e=False, bufs=None):
        for _ in range(args.warmup):
            sc.step_forward(0)
        barrier()
        l0 = sc.launches()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        start.record(stream)
        for _ in range(k):
            if e2e:
                sc.set_dt(sc.dt)  # the step's host input
            code = sc.step_forward(0)
            if code != R.NORMAL_EXIT:
                raise RuntimeError("step returned %d" % code)
            if e2e:
                for j, nm in enumerate(("u", "v", "w", "p")):
                    R.lib().rmt3d_get_field(sc._h, R.FIELD_INDEX[nm], bufs[j].data_ptr())
        stop.record(stream)
        stop.synchronize()
        wall = time.perf_counter() - t0
        ms = start.elapsed_time(stop)
        barrier()
        return max_over_ranks(ms), sc.launches() - l0, wall

    cells = n ** 3
    # plain FP64 form
    s64 = make(R.FP64)
    with ClockSampler(local) as clk:
        ms64, launches64, _ = timed(s64, args.steps)
    clocks = clk.summary()
    v64 = world * cells * args.steps / (ms64 / 1e3) / 1e6
    # mixed form (FP32 V-cycles inside FP64 iterative refinement)
    smx = make(R.MIXED)
    msmx, launchesmx, _ = timed(smx, args.steps)
    vmx = world * cells * args.steps / (msmx / 1e3) / 1e6
    sl = (slice(2, -2),) * 3
    ref = np.stack([s64.field(c)[sl] for c in "uvw"])
    got = np.stack([smx.field(c)[sl] for c in "uvw"])
    mixed_err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    p_err = float(np.linalg.norm(smx.field("p")[sl] - s64.field("p")[sl]) / np.linalg.norm(s64.field("p")[sl]))
    mixed_ok = max(mixed_err, p_err) <= 1e-5
    head_form = "mixed" if (mixed_ok and vmx > v64) else "fp64"
    value = vmx if head_form == "mixed" else v64
    ms = msmx if head_form == "mixed" else ms64
    launches = launchesmx if head_form == "mixed" else launches64
    # end to end through the C ABI: host dt in, u/v/w/p out to pinned host memory
    shp = (s64.so4, s64.sn4, s64.sm4)
    bufs = [torch.empty(shp, dtype=torch.float64, pin_memory=True) for _ in range(4)]
    sce = smx if head_form == "mixed" else s64
    mse, _, wall_e = timed(sce, args.steps, e2e=True, bufs=bufs)
    ve = world * cells * args.steps / (mse / 1e3) / 1e6
    d2h = 4 * s64.ncell * 8
    # roofline of the dominant kernel
    roof = roofline(R, sce, args)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(RUN_SIM):
        procs = max(1, min(host_cores(), args.ref_procs))
        rate, secs, wall = reference_run(n, max(1, args.ref_steps), procs)
        cpu = {"value": rate / 1e6, "unit": METRIC, "cores": procs, "kind": "reference",
               "sample": "%d processes x %d steps of the %d^3 workload, reference run_sim stepper timer" % (
                   procs, args.ref_steps, n)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if head_form == "fp64" else "f64+f32",
            "data": "synthetic (cfg-defined scene, no dataset)",
            "config": dict(config_block(n, "state %.0f MB per scene > 126 MB L2" % (state_mb(s64))),
                           headline_form=head_form),
            "forms": {"fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "gpu_launches": launches64},
                      "mixed": {"value": vmx, "ms_per_step": msmx / args.steps, "gpu_launches": launchesmx,
                                "rel_l2_vel_vs_fp64": mixed_err, "rel_l2_p_vs_fp64": p_err,
                                "steps_compared": args.warmup + args.steps}},
            "e2e": {"value": ve, "unit": METRIC, "h2d_bytes_per_step": 8, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    for s in (s64, smx):
        s.close()
    if dist is not None:
        dist.destroy_process_group()


def state_mb(sc):
    per_cell = (36 + 50 * sc.desc.n_obj) * 8
    return sc.ncell * per_cell / 1e6


TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")


def roofline(R, sc, args):
    """The dominant kernel (FEM Gauss-Seidel colour pass, finest level) timed
    live with CUDA events on the scene's stream over `steps` further steps;
    achieved = algorithmic bytes / measured duration against the measured HBM
    copy bandwidth.  traffic = DRAM bytes per launch from the committed ncu
    capture of the same kernel, when present."""
    peak, src = 6650.0, "fallback"
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
        src = "measured"
    except (OSError, ValueError, KeyError):
        pass
    sc.profile_kernel(0, 200000)
    for _ in range(args.steps):
        sc.step_forward(0)
    ms, n, byts = sc.profile_read()
    sc.profile_kernel(-1)
    achieved = (byts / n) / (ms / n * 1e-3) / 1e9 if n else None
    traffic = None
    try:
        traffic = json.load(open(TRAFFIC_FILE)).get("fem_gs_fine_%d" % args.size)
    except (OSError, ValueError):
        pass
    return {"bound": "hbm", "kernel": "k_fem_gs (finest level colour pass)", "achieved": achieved, "peak": peak,
            "peak_source": src, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": traffic, "launches_timed": n, "avg_launch_us": (1e3 * ms / n) if n else None,
            "algorithmic_bytes_per_launch": (byts / n) if n else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--ref-procs", type=int, default=16)
    ap.add_argument("--ref-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
