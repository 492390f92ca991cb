"""Generate the golden fixtures of the parity tests from the reference itself.

Runs the reference solver (compiled from its own sources by oracle/Makefile
into oracle/_ref/ref_driver) on small seeded workloads and stores, for each
saved step count, the state the FSI step reads and writes: velocities and
nodal pressure over the ghosted box, the primary reference maps and the
extrapolated maps.  Usage (in the build container, where the reference is
present):

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refdump  # noqa: E402
from rmt3d_b200 import scenes  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

# name -> (cfg text, saved step counts)
CASES = {
    "cavity16": (scenes.cavity(16, 8), [0, 1, 8]),
    "sphere24": (scenes.cavity_sphere(24, 4, radius=0.25), [0, 1, 4]),
    "stretch24": (scenes.stretched_sphere(24, 4, radius=0.2), [0, 1, 4]),
}
# longer runs stored as interior (u, v, w, p) only
LONG = {
    "cavity32_64": (scenes.cavity(32, 64), 64),
}


def compact(d):
    """Reduce a dump to the state the step reads and writes."""
    f, rm = d["fields"], d["refmaps"]
    prim = np.nonzero(rm["c"] != 0)[0]
    out = {
        "meta": np.array([d["m"], d["n"], d["o"], d["steps"]] + list(d["shape"]), dtype=np.int64),
        "dt_time": np.array([d["dt"], d["time"]]),
        "vel": f["vel"].T.copy(),
        "p": f["p"].copy(),
        "q": f["q"].copy(),
        "prim_index": prim.astype(np.int32),
        "prim_c": rm["c"][prim].astype(np.uint32),
        "prim_x": rm["x"][prim].copy(),
        "prim_xpred": rm["xpred"][prim].copy(),
        "ext_index": d["ext_index"].astype(np.int32),
        "ext_c": d["ext_maps"]["c"].astype(np.uint32),
        "ext_x": d["ext_maps"]["x"].copy(),
        "ext_xpred": d["ext_maps"]["xpred"].copy(),
    }
    return out


def run(cfg_text, steps, workdir):
    cfg = os.path.join(workdir, "case.cfg")
    with open(cfg, "w") as fh:
        fh.write(cfg_text)
    out = os.path.join(workdir, "s%d.bin" % steps)
    subprocess.run([DRIVER, cfg, str(steps), out], check=True, capture_output=True, cwd=workdir)
    return refdump.read(out)


def main():
    if not os.path.exists(DRIVER):
        sys.exit("build the reference first: make -C oracle")
    with tempfile.TemporaryDirectory() as wd:
        for name, (txt, steps) in CASES.items():
            arrays = {"cfg": np.frombuffer(txt.encode(), dtype=np.uint8)}
            for k in steps:
                for key, val in compact(run(txt, k, wd)).items():
                    arrays["s%d_%s" % (k, key)] = val
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            print("wrote", name)
        for name, (txt, k) in LONG.items():
            d = run(txt, k, wd)
            shp = d["shape"]
            sl = (slice(2, -2),) * 3
            vel = d["fields"]["vel"]
            arrays = {
                "cfg": np.frombuffer(txt.encode(), dtype=np.uint8),
                "meta": np.array([d["m"], d["n"], d["o"], k] + list(shp), dtype=np.int64),
                "dt_time": np.array([d["dt"], d["time"]]),
                "u": vel[:, 0].reshape(shp)[sl].copy(),
                "v": vel[:, 1].reshape(shp)[sl].copy(),
                "w": vel[:, 2].reshape(shp)[sl].copy(),
                "p": d["fields"]["p"].reshape(shp)[sl].copy(),
            }
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            print("wrote", name)


if __name__ == "__main__":
    main()
