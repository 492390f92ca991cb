"""Profiling driver: set up the bench workload, step once, then run N steps.

    RMT3D_GRAPH=0 python -m rmt3d_b200.prof_step [n=64] [steps=2] [precision=0] [var_den=0] [objects=1]
                                                  [smoother=0] [v_down=2] [v_up=2]

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
vd = int(sys.argv[4]) if len(sys.argv) > 4 else 0
nobj = int(sys.argv[5]) if len(sys.argv) > 5 else 1
smoother = int(sys.argv[6]) if len(sys.argv) > 6 else 0
vdn = int(sys.argv[7]) if len(sys.argv) > 7 else 2
vup = int(sys.argv[8]) if len(sys.argv) > 8 else 2
wd = tempfile.mkdtemp()
text = scenes.cavity_sphere(n, 100000, radius=0.2, rho=1.2 if vd else 1.0) if nobj else scenes.cavity(n, 100000)
cfg = scenes.write(os.path.join(wd, 'w.cfg'), text)
d = R.desc_from_cfg(cfg); d.precision = prec; d.var_den = vd
sc = R.Scene(d)
sc.set_schedule(vdn, vup, 0)
sc.set_smoother(smoother)
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
