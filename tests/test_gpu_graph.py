"""The step as one CUDA graph against the step issued kernel by kernel.

The graph form captures the same kernels in the same order, with the
multigrid cycle control and the step's branches evaluated on the device
(WHILE and IF graph nodes).  Both forms must give bit-identical states,
times, step counts and cycle counts, and the graph form must stop a run at
the failing step exactly as the eager form does.
"""
import os

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R
from rmt3d_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene(desc, graph):
    old = os.environ.get("RMT3D_GRAPH")
    os.environ["RMT3D_GRAPH"] = "1" if graph else "0"
    try:
        return R.Scene(desc)
    finally:
        if old is None:
            del os.environ["RMT3D_GRAPH"]
        else:
            os.environ["RMT3D_GRAPH"] = old


def _run(desc, graph, steps, chunks=1):
    sc = _scene(desc, graph)
    try:
        sc.prepare()
        l0 = sc.launches()
        for _ in range(chunks):
            assert sc.run(steps // chunks) == R.NORMAL_EXIT
        out = {f: sc.field(f) for f in ("u", "v", "w", "p", "q", "dp")}
        out["scalars"] = [sc.scalar(i) for i in (0, 1, 4, 5, 6, 7, 8)]
        out["launches"] = sc.launches() - l0
        if desc.n_obj:
            out["x"] = sc.refmap(0)[1]
        return out
    finally:
        sc.close()


@pytest.mark.parametrize("kind", ["cavity", "sphere", "periodic_sphere", "mixed"])
def test_graph_equals_eager(tmp_path, kind):
    if kind == "cavity":
        text = scenes.cavity(16, steps=6)
    elif kind == "periodic_sphere":
        text = scenes.stretched_sphere(24, steps=6, radius=0.2)
    else:
        text = scenes.cavity_sphere(24, steps=6, radius=0.25)
    desc = R.desc_from_cfg(scenes.write(str(tmp_path / "g.cfg"), text))
    if kind == "mixed":
        desc.precision = R.MIXED
    eager = _run(desc, False, 6)
    graph = _run(desc, True, 6, chunks=2)
    for k in eager:
        if k == "launches":
            continue
        a, b = np.asarray(eager[k]), np.asarray(graph[k])
        assert np.array_equal(a, b, equal_nan=True), k
    # the graph adds its gate, branch and status kernels to every step
    per_step = (graph["launches"] - eager["launches"]) / 6
    assert per_step == (3 if desc.n_obj else 2), per_step


def test_graph_run_stops_at_failing_step(tmp_path):
    fx = H.load_fixture("cavity16")
    sc = R.Scene.from_cfg(H.fixture_cfg(fx, str(tmp_path / "c16.cfg")))
    try:
        sc.prepare()
        st0 = H.state(fx, 0)
        fa, ra, ei, em = H.to_aos(st0)
        so4, sn4, sm4 = st0["shape"]
        fa["vel"][10 + sm4 * (10 + sn4 * 10), 0] = np.nan  # an interior cell
        sc.import_reference(fa, ra, ei, em, H.state(fx, 1)["dt"], 0.0)
        nt0 = sc.scalar(4)
        assert sc.run(4) == R.PROJECTION_ERR
        assert sc.scalar(4) == nt0 + 1  # the later steps did not run
    finally:
        sc.close()


@pytest.mark.parametrize("kind", ["sphere", "mixed", "varden"])
def test_cluster_solve_matches_phase_launches(tmp_path, kind):
    """The whole-solve cluster kernel and the per-phase launches apply the
    same operators and control; solved to round-off they agree closely."""
    text = scenes.cavity_sphere(24, steps=4, radius=0.25, rho=1.4 if kind == "varden" else 1.0)
    desc = R.desc_from_cfg(scenes.write(str(tmp_path / "c.cfg"), text))
    desc.mg_exact = 1
    if kind == "mixed":
        desc.precision = R.MIXED
    if kind == "varden":
        desc.var_den = 1
    out = []
    for cluster in (1, 0):
        sc = R.Scene(desc)
        try:
            sc.set_mg_launch(cluster)
            sc.prepare()
            assert sc.run(4) == R.NORMAL_EXIT
            out.append({f: sc.field(f)[H.INTERIOR] for f in ("u", "v", "w", "p")})
        finally:
            sc.close()
    for f in out[0]:
        e = H.rel_l2(out[0][f], out[1][f])
        assert e < 1e-10, (f, e)


@pytest.mark.parametrize("form", [R.MIXED, R.MIXED_BULK32])
def test_mixed_form_accuracy(tmp_path, form):
    """The mixed forms (FP32 V-cycles inside FP64 refinement, solves ended at
    mixed_rtol x max|rhs|; the second also with the advection stencil in FP32)
    stay within their 1e-5 rel-L2 budget against the FP64 form over 60 steps
    of a 32^3 cavity with a sphere.  Velocity is measured against the norm of
    the whole velocity field (v alone is a near-zero cross-flow whose own norm
    magnifies round-off), pressure against its own."""
    path = scenes.write(str(tmp_path / "m.cfg"), scenes.cavity_sphere(32, steps=60, radius=0.25))
    out = {}
    for prec in (R.FP64, form):
        sc = R.Scene.from_cfg(path, precision=prec)
        try:
            sc.prepare()
            assert sc.run(60) == R.NORMAL_EXIT
            out[prec] = ({f: sc.field(f)[H.INTERIOR] for f in ("u", "v", "w", "p")}, sc.scalar(7) + sc.scalar(8))
        finally:
            sc.close()
    a, b = out[R.FP64][0], out[form][0]
    va, vb = np.stack([a[f] for f in "uvw"]), np.stack([b[f] for f in "uvw"])
    assert np.linalg.norm(vb - va) / np.linalg.norm(va) < 1e-5
    assert H.rel_l2(b["p"], a["p"]) < 1e-5
    # the relaxed solves need fewer V-cycles
    assert out[form][1] < out[R.FP64][1]


def test_fp32_face_states_read_back(tmp_path):
    """The FP32 advection form keeps the face states in FP32 on the device;
    reading them widens them to FP64 (the values the step computed, finite,
    close to the FP64 form's), and a snapshot, which copies FP64 arrays,
    refuses them."""
    path = scenes.write(str(tmp_path / "f.cfg"), scenes.cavity_sphere(24, steps=4, radius=0.25))
    faces = {}
    for prec in (R.FP64, R.MIXED_BULK32):
        sc = R.Scene.from_cfg(path, precision=prec)
        try:
            sc.prepare()
            assert sc.run(2) == R.NORMAL_EXIT
            faces[prec] = np.stack([sc.field(9 + a) for a in range(18)])
            if prec == R.MIXED_BULK32:
                import torch
                buf = torch.empty((sc.so4, sc.sn4, sc.sm4), dtype=torch.float64, pin_memory=True)
                with pytest.raises(R.RMT3DError):
                    sc.snapshot((9,), [buf])
        finally:
            sc.close()
    f64, f32 = faces[R.FP64], faces[R.MIXED_BULK32]
    assert np.all(np.isfinite(f32))
    assert np.array_equal(f32, f32.astype(np.float32).astype(np.float64))
    assert np.linalg.norm(f32 - f64) / np.linalg.norm(f64) < 1e-4


def test_graph_rebuilt_after_dt_change(tmp_path):
    """dt is a captured parameter of the step graph: after set_dt the graph is
    captured again, and the run matches the eager form through the change."""
    path = scenes.write(str(tmp_path / "d.cfg"), scenes.cavity_sphere(24, steps=8, radius=0.25))
    desc = R.desc_from_cfg(path)
    res = []
    for graph in (False, True):
        sc = _scene(desc, graph)
        try:
            sc.prepare()
            assert sc.run(2) == R.NORMAL_EXIT
            sc.set_dt(sc.dt * 0.7)
            assert sc.run(3) == R.NORMAL_EXIT
            res.append(({f: sc.field(f) for f in ("u", "v", "w", "p")}, sc.time, sc.dt))
        finally:
            sc.close()
    for f in res[0][0]:
        assert np.array_equal(res[0][0][f], res[1][0][f]), f
    assert res[0][1] == res[1][1] and res[0][2] == res[1][2]
