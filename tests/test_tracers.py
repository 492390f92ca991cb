"""Passive tracers (Utilities/tracers.{hh,cc}) against the reference.

The fixture tr16 is the 16^3 cavity + sphere of chk16 with 200 tracers
(dump_code 1 | 8): the reference's tracer files at frames 0 and 1, its
checkpoint of frame 1 (fields, recover.cfg, tr.00001), and its tracer file
after restarting from that checkpoint and stepping 2 more steps.

Tracer files hold float32 coordinates, so positions are compared to 1e-6
(a few float ulps on a unit box; the fields agree to 1e-10).  A fresh start
cannot be compared directly: the reference scatters the tracers with GSL's
generator and this implementation with its own, so the fresh-run test
places the tracers at the reference's frame-0 positions first.
"""
import os

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

NAMES = ["vx", "vy", "vz", "p", "X", "Y", "Z", "OID"]
POS_TOL = 1e-6


def fixture():
    return H.load_fixture("tr16")


def tr_file(data):
    b = bytes(data)
    n = int(np.frombuffer(b[:4], dtype=np.int32)[0])
    return np.frombuffer(b[4:], dtype=np.float32).reshape(n, 3).astype(np.float64)


def test_tracer_cfg_and_footprint(tmp_path):
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg"]))
    d = R.desc_from_cfg(str(p))
    assert d.run.ntracers == 200 and d.run.dump_code == 9
    with_tr = R.footprint(d)
    d.run.dump_code = 8
    assert with_tr - R.footprint(d) == 200 * (3 * 4 + 6 * 8 + 1)


@pytest.mark.gpu
def test_fresh_run_tracers_match_reference(tmp_path):
    """From the reference's frame-0 positions, two steps land on its frame-1
    positions."""
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg"]))
    sc = R.Scene.from_cfg(str(p), mg_exact=1)
    try:
        sc.prepare()
        start = tr_file(fx["file_tr.00000"])
        sc.place_tracers(start)
        got0 = sc.tracers()
        assert np.abs(got0 - start).max() < 1e-7
        assert sc.run(2) == R.NORMAL_EXIT
        got = sc.tracers().astype(np.float64)
        ref = tr_file(fx["file_tr.00001"])
        assert np.abs(got - ref).max() < POS_TOL, np.abs(got - ref).max()
        assert np.abs(ref - start).max() > 10 * POS_TOL  # the tracers did move
    finally:
        sc.close()


@pytest.mark.gpu
def test_restart_tracers_match_reference(tmp_path, monkeypatch):
    """The reference's checkpoint with its tracer file; run_sim on its
    recover.cfg for 2 steps writes the reference's tr.00002."""
    fx = fixture()
    d = tmp_path / "c.out" / "chk.00001"
    d.mkdir(parents=True)
    for n in NAMES:
        fx["chk_" + n].tofile(str(d / n))
    (d / "recover.cfg").write_bytes(bytes(fx["chkfile_recover.cfg"]))
    (d / "tr.00001").write_bytes(bytes(fx["chkfile_tr.00001"]))
    monkeypatch.chdir(tmp_path)
    sc = R.run_sim("c.out/chk.00001/recover.cfg", stop_short=2, mg_exact=1)
    try:
        out = d / "recover.out"
        first = tr_file((out / "tr.00001").read_bytes())
        assert np.abs(first - tr_file(fx["chkfile_tr.00001"])).max() < 1e-7
        got = tr_file((out / "tr.00002").read_bytes())
        ref = tr_file(fx["file_restart_tr.00002"])
        assert np.abs(got - ref).max() < POS_TOL, np.abs(got - ref).max()
        text = np.loadtxt(str(out / "tr_st.00002"))
        assert np.abs(text - got).max() < 1e-5  # "%g" text of the same positions
    finally:
        sc.close()


@pytest.mark.gpu
def test_tracers_graph_and_eager_identical(tmp_path, monkeypatch):
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg"]))
    res = []
    for graph in ("1", "0"):
        monkeypatch.setenv("RMT3D_GRAPH", graph)
        sc = R.Scene.from_cfg(str(p), mg_exact=1)
        try:
            sc.prepare()
            for _ in range(3):
                assert sc.step_forward(0) == R.NORMAL_EXIT
            res.append(sc.tracers())
        finally:
            sc.close()
    assert np.array_equal(res[0], res[1])


@pytest.mark.gpu
def test_tracers_stay_inside(tmp_path):
    """Walled cavity: every tracer stays inside the box (tracers::dx keeps a
    tracer that moves towards a no-slip wall 1% of the box away from it);
    periodic box: no tracer is lost."""
    from rmt3d_b200 import scenes
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg"]))
    sc = R.Scene.from_cfg(str(p), mg_exact=0)
    try:
        sc.prepare()
        assert sc.run(20) == R.NORMAL_EXIT
        t = sc.tracers()
        assert t.shape == (200, 3)
        assert (t > 0).all() and (t < 1).all()
    finally:
        sc.close()
    q = tmp_path / "p.cfg"
    q.write_text(scenes.stretched_sphere(24, 100, radius=0.2) + "ntracers 300\n")
    dd = R.desc_from_cfg(str(q))
    dd.run.dump_code = 1
    sc = R.Scene(dd)
    try:
        sc.prepare()
        assert sc.run(10) == R.NORMAL_EXIT
        t = sc.tracers()
        assert t.shape == (300, 3) and not (t == 0).all(axis=1).any()
    finally:
        sc.close()
