"""Benchmark of the FSI step on the lid-driven cavity with a neo-Hookean sphere.

Workload (one "step" = one fluid_3d::step_forward of one scene): 64^3 cells,
unit cube, no-slip walls, lid u=(1,0,0) at z=1, fluid viscosity 0.01, sphere
of radius 0.2 at the centre with G=1, solid density 1, transition width
1.5 dx, 5 extrapolation layers.  Synthetic: the scene is fully defined by its
.cfg parameters.

Our arm times the plain FP64 form and the mixed form (FP32 V-cycles inside
FP64 refinement) on the device (K steps as K step-graph launches, CUDA events
on the scene's stream), their per-step latency, then the headline form end to
end through the C ABI with host-side result reads.  Two more forms are
reported beside it: a batch of seeded scenes of uneven sizes stepped together,
and a served Poisson request stream with admission by HBM footprint (p50/p99
request and step latency) against the same stream run serially in FP64.
Multi-GPU runs one independent scene per rank (replicas: the path has no
cross-scene exchange), timed as the max over ranks.

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
def _run_sim_batch(n, steps, procs, wd, tag):
    """`procs` concurrent copies of the reference run_sim, `steps` steps each:
    per-process stepper seconds and the phase report of the slowest one."""
    cfgs = []
    for p in range(procs):
        c = os.path.join(wd, "%s%d.cfg" % (tag, p))
        scenes.write(c, workload_cfg(n, steps))
        cfgs.append(c)
    ps = [subprocess.Popen([RUN_SIM, c], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, cwd=wd)
          for c in cfgs]
    secs, outs = [], []
    for pr in ps:
        out, _ = pr.communicate()
        m = re.search(r"Stepper: Done with everything, took a total\s+([0-9.eE+-]+) seconds", out)
        if pr.returncode != 0 or not m:
            raise RuntimeError("reference run_sim failed:\n" + out[-2000:])
        secs.append(float(m.group(1)))
        outs.append(out)
    return secs, outs[secs.index(max(secs))]


def phase_report(out):
    """The reference's own phase timers (fluid_3d::watch, printed by run_sim
    at exit; they include the set-up's pressure pre-iterations), as shares of
    its tracked compute time."""
    tot = re.search(r"F3d report:\s*#\s*Total tracked compute time\s+([0-9.eE+-]+) s", out)
    if not tot:
        return None
    total = float(tot.group(1))
    rep = {"tracked_s": total}
    for name in ("Extrapolation", "Pressure Poisson", "Communication", "Stresses", "MAC"):
        m = re.search(r"#\s+%s time\s+([0-9.eE+-]+) s" % name, out)
        if m:
            rep[name.lower().replace(" ", "_") + "_share"] = float(m.group(1)) / total if total else None
    return rep


def reference_run(n, steps, procs, warmup=0):
    """Run `procs` copies of the reference run_sim; returns (cell-steps/s
    aggregate over steps warmup+1 .. warmup+steps, per-process seconds of that
    window, the slowest process's phase report).  The window is timed as the
    difference of a (warmup+steps)-step run and a warmup-step run of the same
    scene, both with the reference's stepper timer (set-up excluded)."""
    wd = tempfile.mkdtemp(prefix="rmt3d_ref_")
    long_s, out = _run_sim_batch(n, warmup + steps, procs, wd, "a")
    if warmup > 0:
        short_s, _ = _run_sim_batch(n, warmup, procs, wd, "b")
        secs = [max(1e-9, a - b) for a, b in zip(sorted(long_s), sorted(short_s))]
    else:
        secs = long_s
    cellsteps = procs * steps * n ** 3
    return cellsteps / max(secs), secs, phase_report(out)


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
    warm = max(0, args.warmup)
    rate, secs, phases = reference_run(args.size, steps, procs, warm)
    value = rate / 1e6
    sample = ("%d processes x steps %d..%d of the %d^3 workload (the reference's stepper timer: a %d-step run "
              "minus a %d-step run; set-up and the 5 pressure pre-iterations excluded)" % (
                  procs, warm + 1, warm + steps, args.size, warm + steps, warm))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": 1000 * max(secs) / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args.size, "n/a (CPU)"),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference", "sample": sample,
                         "phases": phases},
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
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return self
        # nvidia-smi takes a moment to start: the timed work begins after its
        # first sample (at most a few seconds of waiting)
        t0 = time.time()
        while time.time() - t0 < 5 and self.p.poll() is None:
            self.f.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
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


def reduce_max(dist, x, device="cuda"):
    """Max over ranks of a per-rank scalar (the replicas' timing rule); the
    identity without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, cells, steps, ms_max):
    """Whole-job throughput of `world` independent replicas, each stepping a
    scene of `cells` cells `steps` times, timed as the slowest rank."""
    return world * cells * steps / (ms_max / 1e3) / 1e6


def percentiles(xs):
    import numpy as np
    if not xs:
        return None
    return {"p50": float(np.percentile(xs, 50)), "p99": float(np.percentile(xs, 99))}


def _batch_descs(R, args, precision):
    wd = tempfile.mkdtemp(prefix="rmt3d_batch_")
    descs, cells = [], 0
    for seed in range(args.batch_scenes):
        n, text = scenes.random_scene(seed, steps=100000)
        d = R.desc_from_cfg(scenes.write(os.path.join(wd, "s%d.cfg" % seed), text))
        d.precision = precision
        d.var_den = 1  # solid densities U(0.8, 1.2): the variable-density projection
        descs.append(d)
        cells += n ** 3
    return descs, cells


def _batch_fields(b, n):
    import numpy as np
    sl = (slice(2, -2),) * 3
    return [(np.stack([b.field(i, f)[sl] for f in "uvw"]), b.field(i, "p")[sl]) for i in range(n)]


def form_batched(R, args):
    """Many independent seeded scenes (grid sizes from {32,48,64,96}, 1-8
    spheres with solid density U(0.8,1.2), lid speed U(0.5,1.5)),
    variable-density projection, mixed precision, schedules autotuned per
    kind of scene; every group's step graph in flight at once.  Wall time
    around the synchronous batch step (the scenes run on their own streams).
    After the timed steps every scene is stepped on to `batch_check_steps`
    steps and compared with the same batch run in plain FP64."""
    import numpy as np
    descs, cells = _batch_descs(R, args, R.MIXED)
    t0 = time.perf_counter()
    b = R.Batch(descs)
    b.prepare()
    prep = time.perf_counter() - t0
    tuned = b.autotune(probe_steps=2)
    st = b.step(args.warmup)
    if any(st):
        raise RuntimeError("batched warm-up status %s" % st)
    t0 = time.perf_counter()
    st = b.step(args.steps)
    wall = time.perf_counter() - t0
    if any(st):
        raise RuntimeError("batched step status %s" % st)
    out = {"value": cells * args.steps / wall / 1e6, "unit": METRIC, "scenes": len(descs), "cells": cells,
           "ms_per_batch_step": 1e3 * wall / args.steps, "timing": "wall clock around the synchronous batch step",
           "prepare_s": prep, "schedules": {str(k): list(v) for k, v in tuned.items()},
           "workload": "seeded cavities, n in {32,48,64,96}, 1-8 spheres R~U(0.08,0.15), G log-U[0.1,10], "
                       "lid U(0.5,1.5), solid density U(0.8,1.2) (variable-density projection), mixed precision"}
    total = args.batch_check_steps
    if total > args.warmup + args.steps:
        st = b.step(total - args.warmup - args.steps)
        if any(st):
            raise RuntimeError("batched status %s" % st)
        mixed = _batch_fields(b, len(descs))
        b.close()
        d64, _ = _batch_descs(R, args, R.FP64)
        b64 = R.Batch(d64)
        b64.prepare()
        st = b64.step(total)
        if any(st):
            raise RuntimeError("FP64 batch status %s" % st)
        ref = _batch_fields(b64, len(descs))
        b64.close()
        ev = [float(np.linalg.norm(m[0] - r[0]) / np.linalg.norm(r[0])) for m, r in zip(mixed, ref)]
        ep = [float(np.linalg.norm(m[1] - r[1]) / np.linalg.norm(r[1])) for m, r in zip(mixed, ref)]
        out["rel_l2_vs_fp64"] = {"steps": total, "velocity_max": max(ev), "p_max": max(ep),
                                 "velocity_median": float(np.median(ev)), "p_median": float(np.median(ep)),
                                 "reference": "the same 64 scenes as an FP64 batch (plain form) after the same steps"}
    else:
        b.close()
    return out


def form_stretched(R, args):
    """The pre-stretched sphere relaxing in a periodic box (128^3, radius 0.3,
    1.3x volume-preserving stretch, viscosity 0.005): FP64 and mixed forms,
    solid volume drift and the mixed form's error against FP64."""
    import numpy as np
    import torch
    wd = tempfile.mkdtemp(prefix="rmt3d_str_")
    n, steps = args.stretch_size, args.stretch_steps
    cfg = scenes.write(os.path.join(wd, "s.cfg"), scenes.stretched_sphere(n, steps, radius=0.3))
    out, fields = {}, {}
    for name, prec in (("fp64", R.FP64), ("mixed", R.MIXED)):
        sc = R.Scene.from_cfg(cfg, precision=prec)
        sc.prepare()
        v0 = sc.diag(1)
        sc.sync()
        t0 = time.perf_counter()
        if sc.run(steps) != R.NORMAL_EXIT:
            raise RuntimeError("stretched-sphere step failed")
        sc.sync()
        wall = time.perf_counter() - t0
        out[name] = {"value": n ** 3 * steps / wall / 1e6, "ms_per_step": 1e3 * wall / steps,
                     "volume_drift": sc.diag(1) / v0 - 1, "detF_dev": sc.diag(5)}
        sl = (slice(2, -2),) * 3
        fields[name] = {f: sc.field(f)[sl] for f in ("u", "v", "w", "p")}
        sc.close()
        torch.cuda.synchronize()
    a, b = fields["fp64"], fields["mixed"]
    va, vb = np.stack([a[f] for f in "uvw"]), np.stack([b[f] for f in "uvw"])
    out["mixed"]["rel_l2_vs_fp64"] = {"velocity": float(np.linalg.norm(vb - va) / np.linalg.norm(va)),
                                      "p": float(np.linalg.norm(b["p"] - a["p"]) / np.linalg.norm(a["p"]))}
    out["workload"] = "periodic %d^3 box, pre-stretched sphere R=0.3 (1.3x along x), G=1, mu=0.005, %d steps, " \
                      "wall-clock timed" % (n, steps)
    return out


def serve_stream(R, wd, seconds, rate, steps, seed, precision):
    import random
    rng = random.Random(seed)
    sizes = [32] * 4 + [64] * 3 + [128] * 2 + [192]
    t, reqs = 0.0, []
    while True:
        t += rng.expovariate(rate)
        if t > seconds:
            break
        k = len(reqs)
        n = rng.choice(sizes)
        _, text = scenes.random_scene(seed * 100003 + k, sizes=(n,), steps=100000)
        d = R.desc_from_cfg(scenes.write(os.path.join(wd, "r%d.cfg" % k), text))
        d.precision = precision
        d.var_den = 1
        reqs.append((t, steps, d))
    return reqs


def form_served(R, args):
    """Seeded Poisson stream (lambda = 20 requests/s), grid sizes 32/64/128/192
    in ratio 4:3:2:1, each request set up and stepped `serve_steps` steps,
    admitted by HBM footprint; against the same stream run serially in FP64."""
    import torch
    wd = tempfile.mkdtemp(prefix="rmt3d_serve_")
    free, total = torch.cuda.mem_get_info()
    budget = int(min(free * 0.8, 120e9))
    reqs = serve_stream(R, wd, args.serve_seconds, 20.0, args.serve_steps, 7, R.MIXED)
    res, summ = R.serve(reqs, budget, args.serve_slots)
    bad = [r["status"] for r in res if r["status"] != 0]
    if bad:
        raise RuntimeError("served requests failed: %s" % bad)
    # the same stream with requests of one kind stepped as one group graph
    reqs_g = serve_stream(R, wd, args.serve_seconds, 20.0, args.serve_steps, 7, R.MIXED)
    res_g, summ_g = R.serve(reqs_g, budget, args.serve_slots, grouped=True)
    if any(r["status"] != 0 for r in res_g):
        raise RuntimeError("grouped served requests failed")
    cells = sum(d.sys_size[0] * d.sys_size[1] * d.sys_size[2] * n for _, n, d in reqs)
    # the same stream, plain FP64, one request after another
    serial = serve_stream(R, wd, args.serve_seconds, 20.0, args.serve_steps, 7, R.FP64)
    for i in range(len(serial)):
        serial[i] = (0.0, serial[i][1], serial[i][2])
    res_s, summ_s = R.serve(serial, budget, 1)
    return {"value": summ["cellsteps_per_s"] / 1e6, "unit": METRIC, "requests": len(reqs),
            "request_latency_s": {"p50": summ["request_p50_s"], "p99": summ["request_p99_s"]},
            "step_latency_ms": {"p50": summ["step_p50_ms"], "p99": summ["step_p99_ms"]},
            "wall_s": summ["wall_s"], "hbm_budget_gb": budget / 1e9, "slots": args.serve_slots,
            "grouped": {"value": summ_g["cellsteps_per_s"] / 1e6, "wall_s": summ_g["wall_s"],
                        "request_latency_s": {"p50": summ_g["request_p50_s"], "p99": summ_g["request_p99_s"]},
                        "step_latency_ms": {"p50": summ_g["step_p50_ms"], "p99": summ_g["step_p99_ms"]},
                        "form": "requests of one kind stepped as one group graph (rmt3d_serve_grouped)"},
            "serial_fp64": {"value": summ_s["cellsteps_per_s"] / 1e6, "wall_s": summ_s["wall_s"],
                            "step_latency_ms": {"p50": summ_s["step_p50_ms"], "p99": summ_s["step_p99_ms"]}},
            "cellsteps": cells,
            "workload": "Poisson arrivals 20/s for %g s (the served workload's 60 s stream cut to its first %g s "
                        "so that the run ends in minutes), n in {32,64,128,192} 4:3:2:1, %d steps each (set-up "
                        "included in the latency), mixed precision; serial_fp64 = the same stream one request at "
                        "a time in FP64" % (args.serve_seconds, args.serve_seconds, args.serve_steps)}


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
        return reduce_max(dist, x)

    def make(precision, tuned=None):
        d = R.desc_from_cfg(cfg)
        d.precision = precision
        if tuned is None:
            # the multigrid schedule chosen by the project's autotuner (timing
            # candidates on a probe copy of the scene)
            b = R.Batch([d], host_threads=1)
            tuned = list(b.autotune(probe_steps=3).values())[0]
            b.close()
        sc = R.Scene(d, stream=stream.cuda_stream)
        sc.set_schedule(tuned[0], tuned[1], 0)
        sc.set_mg_launch(tuned[2])
        sc.set_smoother(tuned[3])
        sc.set_coarse_cluster(tuned[4])
        sc.set_block_shape(tuned[5])
        sc.prepare()
        sc.schedule = tuned
        return sc

    def timed(sc, k):
        """k steps as one run (k step-graph launches, one wait), CUDA events
        on the scene's stream."""
        if sc.run(args.warmup) != R.NORMAL_EXIT:
            raise RuntimeError("warm-up step failed")
        barrier()
        l0 = sc.launches()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        code = sc.run(k)
        stop.record(stream)
        stop.synchronize()
        if code != R.NORMAL_EXIT:
            raise RuntimeError("step returned %d" % code)
        ms = start.elapsed_time(stop)
        barrier()
        return max_over_ranks(ms), sc.launches() - l0

    def step_latency(sc, k):
        """per-step latency: one step per call (launch + wait), CUDA events"""
        out = []
        for _ in range(k):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            if sc.step_forward(0) != R.NORMAL_EXIT:
                raise RuntimeError("step failed")
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return percentiles(out)

    def e2e(sc, k, bufs):
        """through the public API with host buffers: dt in, and u/v/w/p out to
        pinned host memory every step (rmt3d_snapshot_fields: each step's
        fields reach the host while the next step runs; the last one is
        waited for inside the timed region)"""
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        barrier()
        t0 = time.perf_counter()
        start.record(stream)
        for _ in range(k):
            sc.set_dt(sc.dt)
            if sc.step_forward(0) != R.NORMAL_EXIT:
                raise RuntimeError("step failed")
            sc.snapshot(("u", "v", "w", "p"), bufs)
        sc.snapshot_wait()
        stop.record(stream)
        stop.synchronize()
        wall = time.perf_counter() - t0
        barrier()
        # the last host copy ends on the snapshot's copy stream: take the
        # larger of the event span and the host clock around the loop
        return max_over_ranks(max(start.elapsed_time(stop), 1e3 * wall))

    cells = n ** 3
    clk = ClockSampler(local)
    clk.__enter__()  # sampled over every timed region below
    try:
        # plain FP64 form
        s64 = make(R.FP64)
        ms64, launches64 = timed(s64, args.steps)
        v64 = replica_value(world, cells, args.steps, ms64)
        lat64 = step_latency(s64, max(5, args.steps // 2))
        # mixed form (FP32 V-cycles inside FP64 iterative refinement)
        smx = make(R.MIXED)
        msmx, launchesmx = timed(smx, args.steps)
        vmx = replica_value(world, cells, args.steps, msmx)
        latmx = step_latency(smx, max(5, args.steps // 2))
        # both scenes have now run the same number of steps from the same state
        steps_compared = args.warmup + args.steps + max(5, args.steps // 2)
        sl = (slice(2, -2),) * 3
        errs = {}
        for f in ("u", "v", "w", "p"):
            a, b = s64.field(f)[sl], smx.field(f)[sl]
            errs[f] = float(np.linalg.norm(b - a) / np.linalg.norm(a))
        va = np.stack([s64.field(f)[sl] for f in "uvw"])
        vb = np.stack([smx.field(f)[sl] for f in "uvw"])
        errs["velocity"] = float(np.linalg.norm(vb - va) / np.linalg.norm(va))
        # the FP32 advection form (opt-in): the same schedule and steps
        sbk = make(R.MIXED_BULK32, tuned=tuple(smx.schedule))
        msbk, launchesbk = timed(sbk, args.steps)
        vbk = replica_value(world, cells, args.steps, msbk)
        latbk = step_latency(sbk, max(5, args.steps // 2))
        vk = np.stack([sbk.field(f)[sl] for f in "uvw"])
        errs_bk = {"velocity": float(np.linalg.norm(vk - va) / np.linalg.norm(va)),
                   "p": float(np.linalg.norm(sbk.field("p")[sl] - s64.field("p")[sl]) / np.linalg.norm(s64.field("p")[sl]))}
        sbk.close()
        # the 1e-5 budget on the velocity field and the pressure (v alone is a
        # near-zero cross-flow whose own norm magnifies round-off; reported too)
        mixed_ok = max(errs["velocity"], errs["p"]) <= 1e-5
        head_form = "mixed" if (mixed_ok and vmx > v64) else "fp64"
        value = vmx if head_form == "mixed" else v64
        ms = msmx if head_form == "mixed" else ms64
        launches = launchesmx if head_form == "mixed" else launches64
        shp = (s64.so4, s64.sn4, s64.sm4)
        bufs = [torch.empty(shp, dtype=torch.float64, pin_memory=True) for _ in range(4)]
        sce = smx if head_form == "mixed" else s64
        roof = roofline(R, sce, args)
        head_schedule = tuple(sce.schedule)
        for s_ in (s64, smx):
            s_.close()
        # end to end on the same step window as `value`: a fresh scene of the
        # headline form, the same warm-up, then the same K steps through the
        # public API with host buffers
        sce = make(R.MIXED if head_form == "mixed" else R.FP64, tuned=head_schedule)
        if sce.run(args.warmup) != R.NORMAL_EXIT:
            raise RuntimeError("warm-up step failed")
        mse = e2e(sce, args.steps, bufs)
        ve = replica_value(world, cells, args.steps, mse)
        d2h = 4 * sce.ncell * 8
        sce.close()
        batched = served = stretched = None
        if world == 1 and not args.no_batched:
            batched = form_batched(R, args)
        if world == 1 and not args.no_stretched:
            stretched = form_stretched(R, args)
        if world == 1 and not args.no_served:
            served = form_served(R, args)
    finally:
        clk.__exit__()
    clocks = clk.summary()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and os.path.exists(RUN_SIM):
        procs = max(1, min(host_cores(), args.ref_procs))
        rate, secs, phases = reference_run(n, max(1, args.ref_steps), procs, max(0, args.warmup))
        cpu = {"value": rate / 1e6, "unit": METRIC, "cores": procs, "kind": "reference",
               "sample": "%d processes x steps %d..%d of the %d^3 workload, the reference run_sim's stepper "
                         "timer (a %d-step run minus a %d-step run)" % (
                   procs, args.warmup + 1, args.warmup + args.ref_steps, n, args.warmup + args.ref_steps,
                   args.warmup),
               "phases": phases}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if head_form == "fp64" else "f64+f32",
            "data": "synthetic (cfg-defined scene, no dataset)",
            "config": dict(config_block(n, "state %.0f MB per scene > 126 MB L2" % (state_mb_desc(R, cfg))),
                           headline_form=head_form),
            "forms": {"fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "gpu_launches": launches64,
                               "step_latency_ms": lat64, "schedule": list(s64.schedule)},
                      "mixed": {"value": vmx, "ms_per_step": msmx / args.steps, "gpu_launches": launchesmx,
                                "step_latency_ms": latmx, "rel_l2_vs_fp64": errs, "schedule": list(smx.schedule),
                                "steps_compared": steps_compared},
                      "mixed_bulk32": {"value": vbk, "ms_per_step": msbk / args.steps, "gpu_launches": launchesbk,
                                       "step_latency_ms": latbk, "rel_l2_vs_fp64": errs_bk,
                                       "steps_compared": steps_compared,
                                       "form": "RMT3D_MIXED_BULK32: the mixed form with the advection stencil in "
                                               "FP32 (opt-in; not a headline candidate)"},
                      "batched": batched, "served": served, "stretched": stretched},
            "e2e": {"value": ve, "unit": METRIC, "h2d_bytes_per_step": 8, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def state_mb_desc(R, cfg):
    return R.footprint(R.desc_from_cfg(cfg)) / 1e6


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
        traffic = json.load(open(TRAFFIC_FILE)).get(
            "fem_gs_fine_%d_%s" % (args.size, "f32" if sc.desc.precision != R.FP64 else "fp64"))
    except (OSError, ValueError):
        pass
    kname = "k_fem_gs<%s> (finest level colour pass)" % ("float" if sc.desc.precision != R.FP64 else "double")
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
            "peak_source": src, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
            "traffic": traffic, "launches_timed": n, "avg_launch_us": (1e3 * ms / n) if n else None,
            "algorithmic_bytes_per_launch": (byts / n) if n else None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--ref-procs", type=int, default=16)
    ap.add_argument("--ref-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-stretched", action="store_true")
    ap.add_argument("--stretch-size", type=int, default=128)
    ap.add_argument("--stretch-steps", type=int, default=20)
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--serve-seconds", type=float, default=1.5)
    ap.add_argument("--serve-steps", type=int, default=100)
    ap.add_argument("--batch-check-steps", type=int, default=100)
    ap.add_argument("--serve-slots", type=int, default=16)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
