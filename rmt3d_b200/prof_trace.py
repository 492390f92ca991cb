"""Kernel trace of the batched form: every kernel executed inside the group
step graphs, timed by CUPTI (through torch.profiler), summed per kernel.

    python -m rmt3d_b200.prof_trace <n> [steps=5] [smoother=-1]

Builds the scenes of the batched workload (rmt3d_b200.scenes.random_scene,
seeds 0-31) whose grid is n^3, variable density, mixed form; prepares them as
one batch (smoother -1: the autotuner's choice per scene kind; 0 colour
passes; 1 tiled sweeps), runs 3 warm-up steps, times `steps` batch steps, then traces
`steps` more.  Prints the wall time per batch step, the summed kernel time
per batch step and the largest kernels.  Kernels of concurrent scenes
overlap, so a kernel's duration includes the time it shares the device.
"""
import os
import sys
import tempfile
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import torch  # noqa: E402
from torch.profiler import ProfilerActivity, profile  # noqa: E402

import rmt3d_b200 as R  # noqa: E402
from rmt3d_b200 import scenes  # noqa: E402


def main():
    size = int(sys.argv[1]) if len(sys.argv) > 1 else 96
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 5
    smoother = int(sys.argv[3]) if len(sys.argv) > 3 else -1
    wd = tempfile.mkdtemp()
    descs = []
    for seed in range(32):
        n, text = scenes.random_scene(seed, steps=100000)
        if n != size:
            continue
        d = R.desc_from_cfg(scenes.write(os.path.join(wd, "s%d.cfg" % seed), text))
        d.precision = R.MIXED
        d.var_den = 1
        descs.append(d)
    b = R.Batch(descs)
    b.prepare()
    if smoother < 0:
        print("autotuned", b.autotune(probe_steps=2))
    else:
        b.set_smoother(smoother)
    b.step(3)
    torch.cuda.synchronize()
    t = time.perf_counter()
    b.step(steps)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t) / steps
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        b.step(steps)
        torch.cuda.synchronize()
    b.close()
    tot = {}
    for e in prof.key_averages():
        t_us = getattr(e, "self_device_time_total", None) or getattr(e, "self_cuda_time_total", 0)
        if t_us > 0:
            tot[e.key] = (t_us, e.count)
    total = sum(v[0] for v in tot.values())
    print("%d scenes of %d^3: wall %.2f ms per batch step, kernel time %.2f ms per batch step"
          % (len(descs), size, wall * 1e3, total / steps / 1e3))
    print("%-44s %12s %7s %9s %6s" % ("kernel", "us/batch step", "calls", "avg us", "share"))
    for k, (t_us, c) in sorted(tot.items(), key=lambda x: -x[1][0])[:25]:
        print("%-44s %12.1f %7d %9.1f %5.1f%%" % (k.split("(")[0][:44], t_us / steps, c, t_us / c, 100 * t_us / total))


if __name__ == "__main__":
    main()
