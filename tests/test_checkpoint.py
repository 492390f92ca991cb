"""Checkpoint/restart in the reference's format (F3D_Source/fluid_3d_chk_pt.cc).

The fixture chk16 holds the reference's checkpoint of a 16^3 cavity + sphere
after frame 1 (2 steps), its state there (s2) and its state after restarting
from that checkpoint and stepping 2 more steps (s4).  The restart's dt is the
reference's: recover.cfg stores dt with %g, so the restarted stepper fits 3
steps per frame instead of 2 (dt 0.00555... instead of 0.00833...).

* CPU: recover.cfg parsing (run controls, the restart point, the dropped
  restart when the checkpoint directory is absent) and the restart's dt fit.
* GPU: our restart from the reference's checkpoint against the reference's
  restart (rel-L2 1e-10); our checkpoint files against the reference's; the
  reference restarted from our checkpoint; write -> read -> write round trips
  at 16^3 and 64^3; missing and empty files.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

NAMES = ["vx", "vy", "vz", "p", "X", "Y", "Z", "OID"]
TOL = 1e-10
ENV_FACTOR = 20
REF_DRIVER = os.path.join(H.ROOT, "oracle", "_ref", "ref_driver")


def fixture():
    return H.load_fixture("chk16")


def put_checkpoint(root, fx, files=None):
    """The fixture's checkpoint as root/c.out/chk.00001 (uncompressed)."""
    d = os.path.join(str(root), "c.out", "chk.00001")
    os.makedirs(d, exist_ok=True)
    for n in NAMES:
        (files or {}).get(n, fx["chk_" + n]).tofile(os.path.join(d, n))
    with open(os.path.join(d, "recover.cfg"), "wb") as fh:
        fh.write(bytes(fx["recover_cfg"]))
    return d


def read_dir(d):
    out = {}
    for n in NAMES:
        p = os.path.join(d, n)
        if os.path.exists(p):
            out[n] = np.fromfile(p, dtype=np.float64)
        else:
            import lzma
            with lzma.open(p + ".xz") as fh:
                out[n] = np.frombuffer(fh.read(), dtype=np.float64).copy()
    return out


def bound(fx, *ks):
    return max(TOL, ENV_FACTOR * max(float(np.max(fx["s%d_env" % k])) for k in ks))


# --------------------------------------------------------------------------
# CPU: recover.cfg and the restart's stepper arithmetic
# --------------------------------------------------------------------------
def test_recover_cfg_parses(tmp_path, monkeypatch):
    fx = fixture()
    put_checkpoint(tmp_path, fx)
    monkeypatch.chdir(tmp_path)
    d = R.desc_from_cfg("c.out/chk.00001/recover.cfg")
    run = d.run
    assert (run.chk_num, run.chk_step) == (1, 2)
    assert run.current_time == 0.0166667
    assert run.recover_dirname == b"c.out"
    assert run.dirname == b"c.out/chk.00001/recover.out"
    assert run.dump_code == 8 and run.chkpt_freq == 1 and run.output_ind == 8
    assert d.dt == 0.00833333
    # the physics keywords come back as the original .cfg gave them
    src = tmp_path / "c.cfg"
    src.write_bytes(bytes(fx["cfg"]))
    d0 = R.desc_from_cfg(str(src))
    for k in ("sys_size", "bounds", "periodic", "walls", "wall_pos"):
        assert list(getattr(d, k)) == list(getattr(d0, k)), k
    for k in ("fmu", "frho", "wall_dist", "T", "frames", "n_obj", "nlayers", "wt_n", "sim_type", "godunov"):
        assert getattr(d, k) == getattr(d0, k), k
    assert [list(r) for r in d.bct] == [list(r) for r in d0.bct]
    assert [list(r) for r in d.bcv] == [list(r) for r in d0.bcv]
    o, o0 = d.obj[0], d0.obj[0]
    assert (o.type, o.rho, o.G, list(o.basic), list(o.extra)) == (o0.type, o0.rho, o0.G, list(o0.basic),
                                                                 list(o0.extra))
    assert d0.run.chk_num == 0 and d0.run.dirname == str(tmp_path / "c.out").encode()


def test_restart_dropped_without_checkpoint(tmp_path, monkeypatch):
    """sim_params drops the restart when recover_dirname/chk.<n>/recover.cfg
    is absent (sim_params.cc:374-397)."""
    fx = fixture()
    put_checkpoint(tmp_path, fx)
    other = tmp_path / "elsewhere"
    other.mkdir()
    monkeypatch.chdir(other)
    d = R.desc_from_cfg(str(tmp_path / "c.out" / "chk.00001" / "recover.cfg"))
    assert (d.run.chk_num, d.run.chk_step) == (0, 0)


def test_restart_dt_fit(tmp_path, monkeypatch):
    """The restarted stepper refits the %g-rounded dt: 3 steps per frame."""
    fx = fixture()
    put_checkpoint(tmp_path, fx)
    monkeypatch.chdir(tmp_path)
    d = R.desc_from_cfg("c.out/chk.00001/recover.cfg")
    dt, steps = R.stepper_dt(d, 1.0)
    assert steps == 3
    assert dt == 0.0055555555555555549
    assert R.stepper_dt(d, 1.0)[0] != pytest.approx(float(fx["s2_dt_time"][0]), rel=1e-3)


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def restart_scene(monkeypatch, root, fx, steps):
    """run_sim on the checkpoint's recover.cfg, stopping after `steps` steps."""
    monkeypatch.chdir(root)
    return R.run_sim("c.out/chk.00001/recover.cfg", stop_short=steps, mg_exact=1)


def state_errors(sc, st):
    e = H.compare_state(sc, st, 1)
    shp = st["shape"]
    ref = np.stack([st["vel"][c].reshape(shp)[H.INTERIOR] for c in range(3)])
    got = np.stack([sc.field(n)[H.INTERIOR] for n in "uvw"])
    e["vel"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return e


@pytest.mark.gpu
def test_restart_from_reference_checkpoint(tmp_path, monkeypatch):
    fx = fixture()
    put_checkpoint(tmp_path, fx)
    k = int(fx["restart_steps"])
    sc = restart_scene(monkeypatch, tmp_path, fx, k)
    try:
        st = H.state(fx, 2 + k)
        assert sc.scalar(13) == 0  # init_err: restarted
        assert sc.dt == st["dt"]
        assert sc.time == pytest.approx(st["time"], rel=1e-15)
        assert sc.scalar(4) == 2 + k  # step count continues from chk_step
        e = state_errors(sc, st)
        assert e["prim_mismatch"] == 0 and e["ext_mismatch"] == 0, e
        assert e["vel"] < TOL and e["p"] < TOL and e["xi"] < TOL, e
    finally:
        sc.close()


def run_to_checkpoint(root, monkeypatch, fx):
    """run_sim on the original .cfg for frame 1 (2 steps): the stepper writes
    c.out/chk.00000 and c.out/chk.00001."""
    (root / "c.cfg").write_bytes(bytes(fx["cfg"]))
    monkeypatch.chdir(root)
    return R.run_sim("c.cfg", stop_short=2, mg_exact=1)


def compare_files(ours, ref, tol, m, n, o):
    """Field files against the reference's: values within tol (velocity
    components relative to the whole velocity field, as the parity tests),
    owners and the 100 markers of cells without a map exactly.  Positions
    past m*n of a slice hold pressure in the map files and are compared as
    values."""
    L = (m + 1) * (n + 1)
    for k in NAMES:
        assert ours[k].shape == ref[k].shape == (o * L,), k
    vo = np.stack([ours[k] for k in ("vx", "vy", "vz")])
    vr = np.stack([ref[k] for k in ("vx", "vy", "vz")])
    assert H.rel_l2(vo, vr) < tol, H.rel_l2(vo, vr)
    for k in NAMES[3:]:
        assert H.rel_l2(ours[k], ref[k]) < tol, (k, H.rel_l2(ours[k], ref[k]))
    cells = lambda a: a.reshape(o, L)[:, :m * n]  # noqa: E731
    assert np.array_equal(cells(ours["OID"]), cells(ref["OID"]))
    for k in ("X", "Y", "Z"):
        assert np.array_equal(cells(ours[k]) == 100.0, cells(ref[k]) == 100.0), k


@pytest.mark.gpu
def test_checkpoint_files_match_reference(tmp_path, monkeypatch):
    fx = fixture()
    sc = run_to_checkpoint(tmp_path, monkeypatch, fx)
    try:
        d = tmp_path / "c.out" / "chk.00001"
        ours = read_dir(str(d))
        assert os.path.exists(str(d / "vx.xz"))  # compressed as the reference does
        ref = {n: fx["chk_" + n] for n in NAMES}
        compare_files(ours, ref, bound(fx, 2), 16, 16, 16)
        # recover.cfg: the reference's text line for line
        assert (d / "recover.cfg").read_bytes() == bytes(fx["recover_cfg"])
    finally:
        sc.close()


@pytest.mark.gpu
def test_reference_restarts_from_gpu_checkpoint(tmp_path, monkeypatch):
    """The reference's own restart (oracle/_ref/ref_driver) reads our
    checkpoint and lands on its restart from its own checkpoint."""
    if not os.path.exists(REF_DRIVER):
        pytest.skip("oracle/_ref/ref_driver is not built")
    fx = fixture()
    sc = run_to_checkpoint(tmp_path, monkeypatch, fx)
    sc.close()
    k = int(fx["restart_steps"])
    out = str(tmp_path / "r.bin")
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    subprocess.run([REF_DRIVER, "c.out/chk.00001/recover.cfg", str(k), out], check=True, capture_output=True,
                   cwd=str(tmp_path), env=env, timeout=300)
    from oracle import refdump
    from golden.make_golden import compact
    got = compact(refdump.read(out))
    st = H.state(fx, 2 + k)
    shp = st["shape"]
    tol = bound(fx, 2, 2 + k)
    for c in range(3):
        assert H.rel_l2(got["vel"][c], st["vel"][c]) < tol
    assert H.rel_l2(got["p"].reshape(shp)[H.INTERIOR], st["p"].reshape(shp)[H.INTERIOR]) < tol
    assert np.array_equal(got["prim_index"], st["prim_index"])


def roundtrip(tmp_path, cfg_text, steps):
    """Run, checkpoint, restart a fresh scene from it, checkpoint again."""
    cfg = tmp_path / "rt.cfg"
    cfg.write_text(cfg_text)
    sc = R.Scene.from_cfg(str(cfg))
    sc.prepare()
    assert sc.run(steps) == R.NORMAL_EXIT
    a = tmp_path / "a"
    sc.write_chk_pt(steps, 1, str(a), compress=False)
    t_a = sc.time
    sc2 = R.Scene.from_cfg(str(cfg))
    st = sc2.read_chk_pt(str(a))
    assert st == 0
    sc2.init_iter()
    b = tmp_path / "b"
    sc2.write_chk_pt(steps, 1, str(b), compress=False)
    dims = (sc.desc.sys_size[0], sc.desc.sys_size[1], sc.desc.sys_size[2])
    fm, fn = sc.fm, sc.fn
    sc.close()
    sc2.close()
    return read_dir(str(a)), read_dir(str(b)), dims, fm, fn, t_a


@pytest.mark.gpu
@pytest.mark.parametrize("n,steps", [(16, 3), (64, 2)])
def test_checkpoint_roundtrip(tmp_path, n, steps):
    """write -> read -> write: velocities, owners and primary maps come back
    bit for bit; the pressure comes back through the reference's stride-m
    row read (p2[i + fm j] = p1[i + m j])."""
    from rmt3d_b200 import scenes
    A, B, (m, nn, o), fm, fn, _ = roundtrip(tmp_path, scenes.cavity_sphere(n, 100, radius=0.3), steps)
    L = (m + 1) * (nn + 1)
    for k in ("vx", "vy", "vz"):
        assert np.array_equal(A[k], B[k]), k
    # the map files' positions past m*n hold the last pressure slice
    cells = lambda a: a.reshape(o, L)[:, :m * nn]  # noqa: E731
    assert np.array_equal(cells(A["OID"]), cells(B["OID"]))
    prim = cells(A["OID"]) > 0
    assert prim.sum() > 0
    for k in ("X", "Y", "Z"):
        assert np.array_equal(cells(A[k])[prim], cells(B[k])[prim]), k
    pa = A["p"].reshape(o, L)
    pb = B["p"].reshape(o, L)
    i, j = np.meshgrid(np.arange(fm), np.arange(fn), indexing="ij")
    np.testing.assert_array_equal(pb[:, (i + fm * j).ravel()], pa[:, (i + m * j).ravel()])


@pytest.mark.gpu
def test_missing_and_empty_files(tmp_path):
    fx = fixture()
    d = put_checkpoint(tmp_path, fx)
    cfg = tmp_path / "c.cfg"
    cfg.write_bytes(bytes(fx["cfg"]))
    sc = R.Scene.from_cfg(str(cfg), mg_exact=1)
    try:
        sc.prepare()
        t0 = sc.time
        u0 = sc.field("u").copy()
        shutil.move(os.path.join(d, "Y"), os.path.join(d, "Y.bak"))
        assert sc.read_chk_pt(d) == 1
        open(os.path.join(d, "Y"), "wb").close()
        assert sc.read_chk_pt(d) == 2
        assert sc.time == t0 and np.array_equal(sc.field("u"), u0)
        shutil.move(os.path.join(d, "Y.bak"), os.path.join(d, "Y"))
        assert sc.read_chk_pt(d) == 0
        assert sc.time == 0.0  # current_time of this scene's own run block
    finally:
        sc.close()


@pytest.mark.gpu
def test_initialize_falls_back_when_files_missing(tmp_path, monkeypatch):
    """A checkpoint directory whose field files are gone: initialize starts
    from scratch (init_err 1) and clears chk_num, as fluid_3d::initialize."""
    fx = fixture()
    d = put_checkpoint(tmp_path, fx)
    os.remove(os.path.join(d, "OID"))
    monkeypatch.chdir(tmp_path)
    sc = R.Scene.from_cfg("c.out/chk.00001/recover.cfg", mg_exact=1)
    try:
        assert sc.initialize() == 1
        assert sc.time == 0.0
    finally:
        sc.close()
