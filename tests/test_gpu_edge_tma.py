"""The velocity edge states with TMA-staged velocity tiles (k_edge_vel_tma:
planes of u, v, w brought into shared memory by cp.async.bulk.tensor copies
that complete on mbarriers) give exactly the bits of the plain-load kernel
(k_edge_vel, chosen with RMT3D_EDGE_TMA=0 when a scene is created): each
cell's slopes read the same operands in the same order.  Checked over whole
steps for walled and periodic boxes, with and without objects, for a grid
whose x extent is not a multiple of the 32-cell tile (24^3) and one that is
(32^3 cavity)."""
import os

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R
from rmt3d_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p") + tuple("fvel%d%d" % (f, c) for f in range(6) for c in range(3))


def run(cfg, tma, precision=R.FP64, steps=3):
    old = os.environ.get("RMT3D_EDGE_TMA")
    os.environ["RMT3D_EDGE_TMA"] = "1" if tma else "0"
    try:
        sc = R.Scene.from_cfg(cfg, precision=precision)
    finally:
        if old is None:
            del os.environ["RMT3D_EDGE_TMA"]
        else:
            os.environ["RMT3D_EDGE_TMA"] = old
    try:
        sc.prepare()
        assert sc.run(steps) == R.NORMAL_EXIT
        return {f: sc.field(f).copy() for f in FIELDS}
    finally:
        sc.close()


@pytest.mark.parametrize("name", ["cavity16", "sphere24", "stretch24", "wall24"])
def test_edge_tma_bit_identical(tmp_path, name):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / (name + ".cfg")))
    a, b = run(cfg, False), run(cfg, True)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (name, f)


def test_edge_tma_cavity32_mixed(tmp_path):
    cfg = scenes.write(str(tmp_path / "c32.cfg"), scenes.cavity_sphere(32, 100000, radius=0.2))
    a, b = run(cfg, False, R.MIXED, 5), run(cfg, True, R.MIXED, 5)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f
