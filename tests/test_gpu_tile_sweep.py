"""The tiled multigrid sweep (one launch per whole Gauss-Seidel sweep on
shared-memory tiles, mg_tile.cuh) gives exactly the bits of the colour-pass
smoother (one launch per colour): every point's update reads the same
operands in the same order.  Checked over whole steps -- set-up, both
Poisson solves on every level, all the rest of the step -- for walled and
periodic boxes, constant and variable density, FP64 and the mixed form, a
scene alone and a batch group, with the boxes of the tiled sweep cut by the level's edges in every way the
grid sizes 16, 24 and their coarse levels give."""
import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "q", "dp")


def run(tmp_path, name, precision, smoother, steps=3, v=(2, 2)):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / (name + ".cfg")))
    sc = R.Scene.from_cfg(cfg, precision=precision, var_den=int(fx.get("varden", 0)))
    try:
        sc.set_schedule(v[0], v[1], 0)
        sc.set_smoother(smoother)
        sc.prepare()
        assert sc.run(steps) == R.NORMAL_EXIT
        return {f: sc.field(f).copy() for f in FIELDS}, sc.launches()
    finally:
        sc.close()


@pytest.mark.parametrize("name", ["cavity16", "stretch24", "varden24", "multi24"])
@pytest.mark.parametrize("precision", [R.FP64, R.MIXED])
def test_tiled_sweep_bit_identical(tmp_path, name, precision):
    ref, l0 = run(tmp_path, name, precision, 0)
    got, l1 = run(tmp_path, name, precision, 1)
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), (name, precision, f)
    assert l1 < l0  # one launch per sweep instead of one per colour


@pytest.mark.parametrize("v", [(1, 2), (1, 1)])
def test_tiled_sweep_odd_sweep_counts(tmp_path, v):
    """An odd number of sweeps leaves a level's solution in its residual
    array; the cycle follows it there and the fine level copies it back."""
    for prec in (R.FP64, R.MIXED):
        ref, _ = run(tmp_path, "sphere24", prec, 0, v=v)
        got, _ = run(tmp_path, "sphere24", prec, 1, v=v)
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), (v, prec, f)


def test_tiled_sweep_in_batch_group(tmp_path):
    names = ["sphere24", "varden24", "multi24"]
    descs = []
    for n in names:
        fx = H.load_fixture(n)
        d = R.desc_from_cfg(H.fixture_cfg(fx, str(tmp_path / (n + ".cfg"))))
        d.precision = R.MIXED
        d.var_den = 1
        descs.append(d)
    out = []
    for mode in (0, 1):
        b = R.Batch(descs + descs)  # two scenes of each: groups of two
        try:
            b.prepare()
            b.set_smoother(mode)
            assert b.step(3) == [R.NORMAL_EXIT] * (2 * len(descs))
            out.append([{f: b.field(i, f).copy() for f in ("u", "p")} for i in range(2 * len(descs))])
        finally:
            b.close()
    for a, c in zip(out[0], out[1]):
        for f in a:
            assert np.array_equal(a[f], c[f]), f


def run_cc(tmp_path, name, precision, pts, steps=3):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / (name + ".cfg")))
    sc = R.Scene.from_cfg(cfg, precision=precision, var_den=int(fx.get("varden", 0)))
    try:
        sc.set_coarse_cluster(pts)
        sc.prepare()
        assert sc.run(steps) == R.NORMAL_EXIT
        return {f: sc.field(f).copy() for f in FIELDS}, sc.launches()
    finally:
        sc.close()


@pytest.mark.parametrize("name", ["sphere24", "stretch24", "varden24"])
@pytest.mark.parametrize("precision", [R.FP64, R.MIXED])
def test_coarse_cluster_bit_identical(tmp_path, name, precision):
    """The coarse part of each V-cycle as one thread-block-cluster launch
    (the same phase bodies, separated by cluster barriers) gives the bits of
    the per-phase launches, with fewer launches."""
    ref, l0 = run_cc(tmp_path, name, precision, 0)
    got, l1 = run_cc(tmp_path, name, precision, 5000)
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f]), (name, precision, f)
    assert l1 < l0


def test_coarse_cluster_in_batch_group(tmp_path):
    descs = []
    for n in ("sphere24", "varden24"):
        fx = H.load_fixture(n)
        d = R.desc_from_cfg(H.fixture_cfg(fx, str(tmp_path / (n + ".cfg"))))
        d.precision = R.MIXED
        d.var_den = 1
        descs.append(d)
    out = []
    for pts in (0, 5000):
        b = R.Batch(descs + descs)
        try:
            b.prepare()
            for i in range(2 * len(descs)):
                R.lib().rmt3d_scene_set_coarse_cluster(b.scene_handle(i), pts)
            b.set_smoother(0)  # rebuilds the groups with the new schedules
            assert b.step(3) == [R.NORMAL_EXIT] * (2 * len(descs))
            out.append([{f: b.field(i, f).copy() for f in ("u", "p")} for i in range(2 * len(descs))])
        finally:
            b.close()
    for a, c in zip(out[0], out[1]):
        for f in a:
            assert np.array_equal(a[f], c[f]), f
