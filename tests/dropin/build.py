"""Build tests/dropin/_bin/run_sim_gpu: the reference's run_sim sequence, its
sim_params and its unchanged stepper (Sim/stepper.hh) driving the GPU path
through include/rmt3d_fluid_3d.hh.

Test infrastructure.  It compiles against the reference's headers and links
the reference objects the oracle build made (oracle/_ref/obj: sim_params,
write_params, stepper and the single-rank MPI shim), so it needs the
reference checkout (RMT3D_REF_DIR, else the build container's copy) and
`make -C oracle` run first; the binary then travels without them.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_bin", "run_sim_gpu")
OBJ = os.path.join(ROOT, "oracle", "_ref", "obj")
LIBDIR = os.path.join(ROOT, "rmt3d_b200")


def ref_dir():
    d = os.environ.get("RMT3D_REF_DIR") or "/root/reference"
    return d if os.path.isdir(os.path.join(d, "Sim")) else None


def build():
    """Returns the binary's path, or None when the reference or the oracle's
    objects are not here."""
    ref = ref_dir()
    if ref is None or not os.path.isdir(OBJ):
        return None
    objs = sorted(glob.glob(os.path.join(OBJ, "**", "*.o"), recursive=True))
    if not objs:
        return None
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "oracle", "ref_shims"), "-I" + os.path.join(ROOT, "include")]
    inc += ["-I" + os.path.join(ref, d) for d in ("F3D_Source", "Extrapolation", "IO", "Sim", "Utilities")]
    cmd = (["g++", "-O2", "-std=c++11", "-w", "-o", OUT, os.path.join(HERE, "run_sim_gpu.cc")] + inc + objs +
           ["-L" + LIBDIR, "-lrmt3d_gpu", "-Wl,-rpath,$ORIGIN/../../../rmt3d_b200"])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-4000:])
        raise RuntimeError("run_sim_gpu build failed")
    return OUT


if __name__ == "__main__":
    print(build())
