"""Profiling driver for the batched form: one group step between
cudaProfilerStart/Stop.

    python -m rmt3d_b200.prof_group <scenes> <n> <cavity|sphere>

Builds <scenes> equal n^3 lid-driven cavities (with one neo-Hookean sphere
each for "sphere"), prepares them, runs 3 warm-up steps, then one
rmt3d_batch_step inside the profiler range (use ncu --profile-from-start off
--graph-profiling graph: the step graph holds conditional nodes).
"""
import os
import sys
import tempfile
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import torch  # noqa: E402

import rmt3d_b200 as R  # noqa: E402
from rmt3d_b200 import scenes  # noqa: E402


def main():
    nsc, n, kind = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3]
    txt = scenes.cavity(n, steps=100) if kind == "cavity" else scenes.cavity_sphere(n, steps=100)
    path = scenes.write(os.path.join(tempfile.mkdtemp(), "pg.cfg"), txt)
    descs = [R.desc_from_cfg(path) for _ in range(nsc)]
    b = R.Batch(descs, host_threads=1)
    b.prepare()
    b.step(3)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    t = time.perf_counter()
    b.step(1)
    torch.cuda.synchronize()
    print("one group step %.2f ms" % ((time.perf_counter() - t) * 1e3))
    torch.cuda.profiler.stop()
    b.close()


if __name__ == "__main__":
    main()
