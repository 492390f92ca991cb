"""Generate the golden fixtures of the parity tests from the reference itself.

Runs the reference solver (compiled from its own sources by oracle/Makefile
into oracle/_ref/ref_driver) on small seeded workloads and stores, for each
saved step count, the state the FSI step reads and writes: velocities and
nodal pressure over the ghosted box, the primary reference maps and the
extrapolated maps.  The oracle's Poisson solves run with RMT3D_SHIM_EXACT=1
(converged to round-off on every solve), so the fixtures carry no
residual-tolerance noise.  Usage (in the build container, where the reference
is present):

    make -C oracle REF_DIR=<reference checkout> all nofma
    make -C oracle REF_DIR=<reference checkout> VARDEN=1 all nofma
    python tests/golden/make_golden.py [case ...]

The output case out16 holds the files the reference's stepper writes for the
same workload with slice output and frame diagnostics switched on (dump_code
4 | 32): slices of all 22 output types along y (text matrices), a subset
along x (gnuplot binary) and along z (coordinate text), and macro.dat /
centroid.dat, at frames 0 and 1.

The tracer case tr16 runs the same workload with 200 passive tracers
(dump_code 1 | 8): the tracer files of frames 0 and 1, the checkpoint of
frame 1 (with its tracer file), and the tracer file after restarting from
that checkpoint and stepping 2 more steps.

The checkpoint case chk16 (16^3 cavity + sphere of radius 0.3, 2 steps per
frame) holds the reference's checkpoint after frame 1 (write_chk_pt: the
eight slice files, decompressed, and recover.cfg), the reference's state at
that point (s2_*), and its state after restarting from the checkpoint with
run_sim's sequence and stepping CHK_RESTART_STEPS more steps (s4_*).
"""
import lzma
import os
import shutil
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
RUN_SIM = os.path.join(ROOT, "oracle", "_ref", "run_sim")
# the reference rebuilt without FMA contraction (make -C oracle nofma)
DRIVER_NOFMA = os.path.join(ROOT, "oracle", "_ref", "nofma", "ref_driver")

# the variable-density build of the reference (make -C oracle VARDEN=1 all nofma)
DRIVER_VD = os.path.join(ROOT, "oracle", "_ref", "ref_driver.varden")
DRIVER_VD_NOFMA = os.path.join(ROOT, "oracle", "_ref", "nofma", "ref_driver.varden")

# name -> (cfg text, saved step counts[, variable density])
CASES = {
    "cavity16": (scenes.cavity(16, 8), [0, 1, 8]),
    "sphere24": (scenes.cavity_sphere(24, 4, radius=0.25), [0, 1, 4]),
    "stretch24": (scenes.stretched_sphere(24, 4, radius=0.2), [0, 1, 4]),
    # solid density differs from the fluid's: the reference's VAR_DEN build
    "varden24": (scenes.cavity_sphere(24, 4, radius=0.25, rho=1.5), [0, 1, 4], True),
    "multi24": (scenes.multi_sphere(24, 4, spheres=[((0.3, 0.3, 0.35), 0.15, 0.5, 0.8),
                                                  ((0.7, 0.65, 0.4), 0.15, 2.0, 1.2),
                                                  ((0.45, 0.6, 0.72), 0.15, 1.0, 1.0)]), [0, 1, 4], True),
    # two spheres 0.02 apart: their transition bands overlap, so the collision
    # stress between the two solids is active from the first step
    "collide24": (scenes.multi_sphere(24, 4, spheres=[((0.29, 0.5, 0.5), 0.2, 1.0, 1.0),
                                                    ((0.71, 0.5, 0.5), 0.2, 2.0, 1.0)]), [0, 1, 4]),
    # a sphere 0.05 above the bottom wall under gravity: wall repulsion and
    # the gravity of solid and fluid (sim_manager.cc:212-295, sim_manager.hh:400-404)
    "wall24": (scenes.wall_sphere(24, 4), [0, 1, 4]),
    # the manufactured solution (sim_ftest) on a periodic box, with its body force
    "ftest16": (scenes.ftest(16, 4), [0, 1, 4]),
}
# longer runs stored as interior (u, v, w, p) only
LONG = {
    "cavity32_64": (scenes.cavity(32, 64), 64),
}


CHK_NAMES = ["vx", "vy", "vz", "p", "X", "Y", "Z", "OID"]
CHK_RESTART_STEPS = 2


def chk_cfg():
    """16^3 cavity + sphere writing a checkpoint every frame of 2 steps."""
    txt = scenes.cavity_sphere(16, 1000, radius=0.3)
    for a, b in (("dump_code 0", "dump_code 8"), ("frames 100000", "frames 4"), ("T 100000", "T 0.05")):
        assert a in txt
        txt = txt.replace(a, b)
    return txt


def read_chk_dir(d):
    """The eight field files of a checkpoint directory (raw or .xz) as float64."""
    out = {}
    for n in CHK_NAMES:
        raw = os.path.join(d, n)
        if os.path.exists(raw):
            with open(raw, "rb") as fh:
                data = fh.read()
        else:
            with lzma.open(raw + ".xz") as fh:
                data = fh.read()
        out[n] = np.frombuffer(data, dtype=np.float64).copy()
    return out


def restart(chk_src, steps, workdir, driver, exact):
    """The reference restarted from a copy of checkpoint directory chk_src
    (c.out/chk.00001 relative to workdir, as its recover.cfg names it)."""
    dst = os.path.join(workdir, "c.out", "chk.00001")
    if os.path.exists(dst):
        shutil.rmtree(dst)
    shutil.copytree(chk_src, dst)
    out = os.path.join(workdir, "restart.bin")
    env = dict(os.environ, RMT3D_SHIM_EXACT=exact)
    subprocess.run([driver, "c.out/chk.00001/recover.cfg", str(steps), out], check=True, capture_output=True,
                   cwd=workdir, env=env)
    return refdump.read(out)


def make_chk(workdir):
    txt = chk_cfg()
    with open(os.path.join(workdir, "c.cfg"), "w") as fh:
        fh.write(txt)
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    subprocess.run([DRIVER, "c.cfg", "2", "s2.bin"], check=True, capture_output=True, cwd=workdir, env=env)
    saved = os.path.join(workdir, "saved_chk1")
    shutil.copytree(os.path.join(workdir, "c.out", "chk.00001"), saved)
    arrays = {"cfg": np.frombuffer(txt.encode(), dtype=np.uint8),
              "restart_steps": np.array(CHK_RESTART_STEPS)}
    with open(os.path.join(saved, "recover.cfg"), "rb") as fh:
        arrays["recover_cfg"] = np.frombuffer(fh.read(), dtype=np.uint8)
    for n, v in read_chk_dir(saved).items():
        arrays["chk_" + n] = v
    d2 = refdump.read(os.path.join(workdir, "s2.bin"))
    for key, val in compact(d2).items():
        arrays["s2_" + key] = val
    arrays["s2_env"] = envelope(txt, 2, d2, os.path.join(workdir, "env"))
    k = 2 + CHK_RESTART_STEPS
    dr = restart(saved, CHK_RESTART_STEPS, workdir, DRIVER, "1")
    for key, val in compact(dr).items():
        arrays["s%d_%s" % (k, key)] = val
    # rounding envelope of the restart, as envelope() does for a run
    shp = dr["shape"]
    sl = (slice(2, -2),) * 3
    vb = dr["fields"]["vel"].reshape(shp + (3,))[sl]
    pb = dr["fields"]["p"].reshape(shp)[sl]
    xb = dr["refmaps"]["x"][dr["refmaps"]["c"] != 0]
    e = np.zeros(3)
    for drv, ex in ((DRIVER_NOFMA, "1"), (DRIVER, "0")):
        dd = restart(saved, CHK_RESTART_STEPS, workdir, drv, ex)
        v = dd["fields"]["vel"].reshape(shp + (3,))[sl]
        p = dd["fields"]["p"].reshape(shp)[sl]
        xd = dd["refmaps"]["x"][dd["refmaps"]["c"] != 0]
        xe = _rel(xd, xb) if xd.shape == xb.shape and xb.size else 0.0
        e = np.maximum(e, [_rel(v, vb), _rel(p, pb), xe])
    arrays["s%d_env" % k] = e
    print("chk16 envelopes", arrays["s2_env"], e)
    np.savez_compressed(os.path.join(HERE, "chk16.npz"), **arrays)
    print("wrote chk16")


# name -> extra .cfg lines of the output case (same workload as chk16)
OUT_RUNS = {
    "y_matrix": "dump_code 36\nout_flag %d\noutput_dim 1\noutput_ind 8\ndata_fmt 0\n" % ((1 << 22) - 1),
    "x_gnuplot": "dump_code 4\nout_flag %d\noutput_dim 0\noutput_ind 5\ndata_fmt 2\n" % (
        (1 << 0) | (1 << 6) | (1 << 8) | (1 << 12) | (1 << 19)),
    "z_text": "dump_code 4\nout_flag %d\noutput_dim 2\noutput_ind 3\ndata_fmt 1\n" % (
        (1 << 1) | (1 << 9) | (1 << 13) | (1 << 20)),
}


def out_cfg(extra):
    txt = chk_cfg().replace("dump_code 8", "")
    return txt + extra


def make_out(workdir):
    arrays = {}
    for name, extra in OUT_RUNS.items():
        wd = os.path.join(workdir, name)
        os.makedirs(wd)
        txt = out_cfg(extra)
        with open(os.path.join(wd, "c.cfg"), "w") as fh:
            fh.write(txt)
        env = dict(os.environ, RMT3D_SHIM_EXACT="1")
        subprocess.run([DRIVER, "c.cfg", "2", "s2.bin"], check=True, capture_output=True, cwd=wd, env=env)
        arrays["cfg_" + name] = np.frombuffer(txt.encode(), dtype=np.uint8)
        outdir = os.path.join(wd, "c.out")
        for fn in sorted(os.listdir(outdir)):
            with open(os.path.join(outdir, fn), "rb") as fh:
                arrays["file_%s/%s" % (name, fn)] = np.frombuffer(fh.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "out16.npz"), **arrays)
    print("wrote out16", len(arrays), "arrays")


def make_tr(workdir):
    txt = chk_cfg().replace("dump_code 8", "dump_code 9") + "ntracers 200\n"
    with open(os.path.join(workdir, "c.cfg"), "w") as fh:
        fh.write(txt)
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    subprocess.run([DRIVER, "c.cfg", "2", "s2.bin"], check=True, capture_output=True, cwd=workdir, env=env)
    arrays = {"cfg": np.frombuffer(txt.encode(), dtype=np.uint8)}
    out = os.path.join(workdir, "c.out")
    for fn in ("tr.00000", "tr.00001"):
        with open(os.path.join(out, fn), "rb") as fh:
            arrays["file_" + fn] = np.frombuffer(fh.read(), dtype=np.uint8)
    chk = os.path.join(out, "chk.00001")
    saved = os.path.join(workdir, "saved_chk1")
    shutil.copytree(chk, saved)
    for n, v in read_chk_dir(saved).items():
        arrays["chk_" + n] = v
    for fn in ("recover.cfg", "tr.00001"):
        with open(os.path.join(saved, fn), "rb") as fh:
            arrays["chkfile_" + fn] = np.frombuffer(fh.read(), dtype=np.uint8)
    subprocess.run([DRIVER, "c.out/chk.00001/recover.cfg", "2", "r.bin"], check=True, capture_output=True,
                   cwd=workdir, env=env)
    with open(os.path.join(chk, "recover.out", "tr.00002"), "rb") as fh:
        arrays["file_restart_tr.00002"] = np.frombuffer(fh.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "tr16.npz"), **arrays)
    print("wrote tr16")


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


def run(cfg_text, steps, workdir, driver=DRIVER, exact="1"):
    cfg = os.path.join(workdir, "case.cfg")
    with open(cfg, "w") as fh:
        fh.write(cfg_text)
    out = os.path.join(workdir, "s%d.bin" % steps)
    env = dict(os.environ, RMT3D_SHIM_EXACT=exact)
    subprocess.run([driver, cfg, str(steps), out], check=True, capture_output=True, cwd=workdir, env=env)
    return refdump.read(out)


def _rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def envelope_parts(cfg_text, steps, base, workdir, varden=False):
    """The two parts of the rounding envelope, each as the rel-L2 change of
    (velocity vector, pressure, reference map) against the fixture state:
    (build without FMA contraction, exact solves), (the reference's own
    residual-tolerance multigrid control, FMA build); plus the first one's
    state (the no-FMA exact-mode reference)."""
    shp = base["shape"]
    sl = (slice(2, -2),) * 3
    vb = base["fields"]["vel"].reshape(shp + (3,))[sl]
    pb = base["fields"]["p"].reshape(shp)[sl]
    x_b = base["refmaps"]["x"][base["refmaps"]["c"] != 0]
    parts, nofma = [], None
    drivers = ((DRIVER_VD_NOFMA, "1"), (DRIVER_VD, "0")) if varden else ((DRIVER_NOFMA, "1"), (DRIVER, "0"))
    for drv, ex in drivers:
        d = run(cfg_text, steps, workdir, drv, ex)
        if nofma is None:
            nofma = d
        v = d["fields"]["vel"].reshape(shp + (3,))[sl]
        p = d["fields"]["p"].reshape(shp)[sl]
        x_d = d["refmaps"]["x"][d["refmaps"]["c"] != 0]
        xe = _rel(x_d, x_b) if x_b.shape == x_d.shape and x_b.size else 0.0
        parts.append(np.array([_rel(v, vb), _rel(p, pb), xe]))
    return parts[0], parts[1], nofma


def envelope(cfg_text, steps, base, workdir, varden=False):
    """Rounding envelope of the reference at this state: the largest rel-L2
    change of (velocity vector, pressure, reference map) between the fixture
    and two other valid roundings of the same computation -- the build without
    FMA contraction, and the reference's own residual-tolerance multigrid
    control instead of round-off convergence."""
    shp = base["shape"]
    sl = (slice(2, -2),) * 3
    vb = base["fields"]["vel"].reshape(shp + (3,))[sl]
    pb = base["fields"]["p"].reshape(shp)[sl]
    env = np.zeros(3)
    drivers = ((DRIVER_VD_NOFMA, "1"), (DRIVER_VD, "0")) if varden else ((DRIVER_NOFMA, "1"), (DRIVER, "0"))
    for drv, ex in drivers:
        d = run(cfg_text, steps, workdir, drv, ex)
        v = d["fields"]["vel"].reshape(shp + (3,))[sl]
        p = d["fields"]["p"].reshape(shp)[sl]
        x_b = base["refmaps"]["x"][base["refmaps"]["c"] != 0]
        x_d = d["refmaps"]["x"][d["refmaps"]["c"] != 0]
        xe = _rel(x_d, x_b) if x_b.shape == x_d.shape and x_b.size else 0.0
        env = np.maximum(env, [_rel(v, vb), _rel(p, pb), xe])
    return env


def runsim_error(cfg_text, workdir):
    """The reference run_sim's own exact-solution report (Execs/run_sim.cc:
    144-158: fluid_3d::error after the run): T, dh, dt and the mean squared
    errors of u, v, w, p, as printed (%13.10f)."""
    cfg = os.path.join(workdir, "err.cfg")
    with open(cfg, "w") as fh:
        fh.write(cfg_text)
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    out = subprocess.run([RUN_SIM, cfg], check=True, capture_output=True, text=True, cwd=workdir, env=env).stdout
    lines = out.splitlines()
    i = [j for j, ln in enumerate(lines) if ln.startswith("#T dh dt erru_sq")][0]
    return np.array([float(v) for v in lines[i + 1].split()])


def main():
    if not (os.path.exists(DRIVER) and os.path.exists(DRIVER_NOFMA)):
        sys.exit("build the reference first: make -C oracle REF_DIR=<reference checkout> all nofma")
    with tempfile.TemporaryDirectory() as wd:
        only = sys.argv[1:]
        for name, case in CASES.items():
            if only and name not in only:
                continue
            txt, steps = case[0], case[1]
            varden = len(case) > 2 and case[2]
            arrays = {"cfg": np.frombuffer(txt.encode(), dtype=np.uint8), "varden": np.array(int(varden))}
            for k in steps:
                d = run(txt, k, wd, DRIVER_VD if varden else DRIVER)
                for key, val in compact(d).items():
                    arrays["s%d_%s" % (k, key)] = val
                envf, envt, dn = envelope_parts(txt, k, d, wd, varden)
                arrays["s%d_env" % k] = np.maximum(envf, envt)
                arrays["s%d_envf" % k] = envf
                arrays["s%d_envt" % k] = envt
                # the same state from the build without FMA contraction, exact
                # solves: the rounding the CUDA path (built without contraction)
                # follows
                for key, val in compact(dn).items():
                    arrays["n%d_%s" % (k, key)] = val
                print(name, k, "envelope (nofma, tolerance)", envf, envt)
            if "has_exact 1" in txt:
                arrays["runsim_err"] = runsim_error(txt, wd)
                print(name, "run_sim exact-solution errors", arrays["runsim_err"])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            print("wrote", name)
        if not only or "out16" in only:
            os.makedirs(os.path.join(wd, "out"))
            make_out(os.path.join(wd, "out"))
        if not only or "tr16" in only:
            os.makedirs(os.path.join(wd, "tr"))
            make_tr(os.path.join(wd, "tr"))
        if not only or "chk16" in only:
            os.makedirs(os.path.join(wd, "chk", "env"))
            make_chk(os.path.join(wd, "chk"))
        for name, (txt, k) in LONG.items():
            if only and name not in only:
                continue
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
            envf, envt, dn = envelope_parts(txt, k, d, wd)
            arrays["env"] = np.maximum(envf, envt)
            arrays["envf"] = envf
            arrays["envt"] = envt
            vn = dn["fields"]["vel"]
            for c, nm in enumerate("uvw"):
                arrays["n" + nm] = vn[:, c].reshape(shp)[sl].copy()
            arrays["np"] = dn["fields"]["p"].reshape(shp)[sl].copy()
            print(name, "envelope (nofma, tolerance)", envf, envt)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            print("wrote", name)


if __name__ == "__main__":
    main()
