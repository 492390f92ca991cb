"""The oracle: the reference's own sources compiled with single-rank MPI and
PGMG-compatible shims (oracle/Makefile).  These tests pin the committed golden
fixtures to that binary and check the fixture contents are self-consistent."""
import os
import subprocess

import numpy as np
import pytest

import helpers as H
from oracle import refdump

DRIVER = os.path.join(H.ROOT, "oracle", "_ref", "ref_driver")
DRIVER_VD = os.path.join(H.ROOT, "oracle", "_ref", "ref_driver.varden")
needs_ref = pytest.mark.skipif(not (os.path.exists(DRIVER) and os.path.exists(DRIVER_VD)),
                               reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("name,k", [("cavity16", 1), ("sphere24", 1), ("stretch24", 0), ("varden24", 1),
                                    ("multi24", 1), ("collide24", 1), ("wall24", 1), ("ftest16", 1)])
def test_fixture_reproduces_from_reference(tmp_path, name, k):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / "case.cfg"))
    out = str(tmp_path / "o.bin")
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    drv = DRIVER_VD if int(fx.get("varden", 0)) else DRIVER
    subprocess.run([drv, cfg, str(k), out], check=True, capture_output=True, cwd=str(tmp_path), env=env)
    d = refdump.read(out)
    st = H.state(fx, k)
    assert d["dt"] == st["dt"] and d["time"] == st["time"]
    # bit-identical: the fixture is this binary's output
    assert np.array_equal(d["fields"]["vel"].T, st["vel"])
    assert np.array_equal(d["fields"]["p"], st["p"])
    assert np.array_equal(d["ext_index"], st["ext_index"])


def test_nofma_states_reproduce_from_reference(tmp_path):
    """The no-FMA states (n<k>_*) are that build's exact-mode output."""
    drv = os.path.join(H.ROOT, "oracle", "_ref", "nofma", "ref_driver")
    if not os.path.exists(drv):
        pytest.skip("oracle/_ref/nofma not built here")
    fx = H.load_fixture("sphere24")
    cfg = H.fixture_cfg(fx, str(tmp_path / "case.cfg"))
    out = str(tmp_path / "o.bin")
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    subprocess.run([drv, cfg, "1", out], check=True, capture_output=True, cwd=str(tmp_path), env=env)
    d = refdump.read(out)
    st = H.state(fx, 1, "n")
    assert np.array_equal(d["fields"]["vel"].T, st["vel"]) and np.array_equal(d["fields"]["p"], st["p"])


def test_fixture_invariants():
    for name in ("cavity16", "sphere24", "stretch24", "varden24", "multi24", "collide24", "wall24", "ftest16"):
        fx = H.load_fixture(name)
        for k in (0, 1):
            st = H.state(fx, k)
            n = int(np.prod(st["shape"]))
            assert st["vel"].shape == (3, n) and np.isfinite(st["vel"]).all()
            # at most one map per object per cell
            keys = st["ext_index"].astype(np.int64) * 1024 + (st["ext_c"] & 1023)
            assert len(np.unique(keys)) == len(keys)
            # an object never has both its primary map and an extrapolated
            # map in one cell (other objects' maps may share the cell)
            for oid in set((st["prim_c"] & 1023).tolist()) - {0}:
                prim = set(st["prim_index"][(st["prim_c"] & 1023) == oid].tolist())
                ext = set(st["ext_index"][(st["ext_c"] & 1023) == oid].tolist())
                assert not prim & ext, (name, oid)
        # lid-driven cavity: walls hold the Dirichlet values through the ghost mirror
    fx = H.load_fixture("cavity16")
    st = H.state(fx, 8)
    shp = st["shape"]
    u = st["vel"][0].reshape(shp)
    # ghost + first interior layer at the lid average to the lid speed 1
    assert np.allclose(0.5 * (u[-2, 2:-2, 2:-2] + u[-3, 2:-2, 2:-2]), 1.0, atol=1e-12)


def test_long_cavity_fixture_shape():
    fx = H.load_fixture("cavity32_64")
    assert fx["u"].shape == (32, 32, 32)
    assert np.abs(fx["u"]).max() < 1.0 + 1e-9


def test_ftest_error_restatement_matches_reference_report():
    """The numpy restatement of fluid_3d::error (tests/helpers.py) gives the
    reference run_sim's own printed exact-solution errors for its state."""
    fx = H.load_fixture("ftest16")
    st = H.state(fx, 4)
    shp = st["shape"]
    e = H.ftest_error(*[st["vel"][c].reshape(shp)[H.INTERIOR] for c in range(3)],
                      st["p"].reshape(shp)[H.INTERIOR], st["time"], 1.0 / 16, 0.01)
    printed = fx["runsim_err"]
    assert st["time"] == pytest.approx(printed[0], rel=1e-12)
    assert np.allclose(e, printed[3:], rtol=0, atol=6e-11), (e, printed)


@needs_ref
def test_compact_field_dumps_match_full_dumps(tmp_path):
    """The compact dumps the configuration-size GPU tests read
    (`ref_driver ... fields k1,k2,...`) carry the same velocity and pressure
    bits as the full dumps the fixtures were made from, at every listed step."""
    fx = H.load_fixture("cavity16")
    cfg = H.fixture_cfg(fx, str(tmp_path / "case.cfg"))
    env = dict(os.environ, RMT3D_SHIM_EXACT="1")
    subprocess.run([DRIVER, cfg, "8", "out", "fields", "1,8"], check=True, capture_output=True, cwd=str(tmp_path),
                   env=env)
    for k in (1, 8):
        d = refdump.read_fields(str(tmp_path / ("out_s%d.f64" % k)))
        st = H.state(fx, k)
        assert d["steps"] == k and d["dt"] == st["dt"] and d["time"] == st["time"]
        for c, name in enumerate("uvw"):
            assert np.array_equal(d[name].ravel(), st["vel"][c]), (k, name)
        assert np.array_equal(d["p"].ravel(), st["p"]), k
