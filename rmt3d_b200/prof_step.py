"""Profiling driver: set up the bench workload, step once, then run N steps.

    RMT3D_GRAPH=0 python -m rmt3d_b200.prof_step [n=64] [steps=2] [precision=0]

Prints PREP_LAUNCHES (kernel launches before the profiled steps, for ncu -s)
and STEP_LAUNCHES (launches of the profiled steps, for ncu -c).  ncu cannot
profile kernels inside graphs that hold conditional nodes, so profiling runs
use RMT3D_GRAPH=0: the same kernels issued one by one from the host.
"""
import sys, os, tempfile
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import rmt3d_b200 as R
from rmt3d_b200 import scenes
n = int(sys.argv[1]) if len(sys.argv) > 1 else 64
steps = int(sys.argv[2]) if len(sys.argv) > 2 else 2
prec = int(sys.argv[3]) if len(sys.argv) > 3 else 0
wd = tempfile.mkdtemp()
cfg = scenes.write(os.path.join(wd, 'w.cfg'), scenes.cavity_sphere(n, 100000, radius=0.2))
d = R.desc_from_cfg(cfg); d.precision = prec
sc = R.Scene(d)
sc.prepare()
sc.step_forward(0)
sc.sync()
print('PREP_LAUNCHES=%d' % sc.launches())
l0 = sc.launches()
for _ in range(steps):
    sc.step_forward(0)
sc.sync()
print('STEP_LAUNCHES=%d' % (sc.launches() - l0))
print('MG', sc.scalar(5), sc.scalar(6))
