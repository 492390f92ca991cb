"""Solid diagnostics (compute_centroid, total_dev_in_detF) against a numpy
restatement on the exported state, and the size-independent invariants they
track: solid volume conservation and det F = 1 for volume-preserving maps."""
import math

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R
from rmt3d_b200 import scenes

pytestmark = pytest.mark.gpu


def heaviside(phi, eps):
    """sim_manager::heaviside (Sim/sim_manager.hh:259-268)."""
    h = 0.5 - phi / (2 * eps) - np.sin(math.pi * phi / eps) / (2 * math.pi)
    h = np.clip(h, 0.0, 1.0)
    h = np.where(phi >= eps, 0.0, h)
    return np.where(phi <= -eps, 1.0, h)


def test_volume_and_centroid_match_numpy(tmp_path):
    fx = H.load_fixture("sphere24")
    sc = R.Scene.from_cfg(H.fixture_cfg(fx, str(tmp_path / "s.cfg")))
    try:
        sc.prepare()
        assert sc.run(2) == R.NORMAL_EXIT
        code, x, _ = sc.refmap(0)
        sl = (slice(2, -2),) * 3
        prim = code[sl] == 0
        d = sc.desc
        ob = d.obj[0]
        c, r = ob.basic[:3], ob.basic[3]
        xi = np.stack([x[a][sl][prim] for a in range(3)])
        phi = np.sqrt(((xi - np.array(c)[:, None]) ** 2).sum(0)) - r
        dx = (d.bounds[1] - d.bounds[0]) / d.sys_size[0]
        hs = heaviside(phi, d.wt_n * dx)
        vol = hs.sum() * dx ** 3
        assert sc.diag(1) == pytest.approx(vol, rel=1e-12)
        n = d.sys_size[0]
        coords = d.bounds[0] + (np.arange(n) + 0.5) * dx
        kk, jj, ii = np.nonzero(prim)
        for a, idx in zip((2, 3, 4), (ii, jj, kk)):
            assert sc.diag(a) == pytest.approx((coords[idx] * hs).sum() / hs.sum(), rel=1e-12)
        # the sphere sits at the centre of the cavity
        assert sc.diag(2) == pytest.approx(0.5, abs=2e-2)
    finally:
        sc.close()


def test_stretched_sphere_volume_and_detF(tmp_path):
    """The pre-stretched sphere's map is volume preserving (det F = 1) and the
    solid volume is conserved while it relaxes."""
    cfg = scenes.write(str(tmp_path / "st.cfg"), scenes.stretched_sphere(32, 20, radius=0.25))
    sc = R.Scene.from_cfg(cfg)
    try:
        sc.prepare()
        v0 = sc.diag(1)
        # H(phi) summed over the primary maps only (phi < 0): the outer half of
        # the smeared interface is not counted, so the sum sits below the
        # ellipsoid's volume by about the interface width
        assert 0.85 < v0 / (4 / 3 * math.pi * 0.25 ** 3) < 1.0
        assert sc.diag(5) < 5e-3 and sc.diag(6) < 5e-2
        assert sc.run(20) == R.NORMAL_EXIT
        assert abs(sc.diag(1) / v0 - 1) < 5e-3
        assert sc.diag(5) < 5e-2
    finally:
        sc.close()
