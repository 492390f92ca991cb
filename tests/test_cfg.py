"""Host-side .cfg front end and stepper arithmetic (Sim/sim_params.cc,
Sim/stepper.hh), checked against the reference's own dt from the fixtures."""
import os

import numpy as np
import pytest

import rmt3d_b200 as R
from rmt3d_b200 import scenes
import helpers as H


def test_defaults_match_reference():
    d = R.desc_defaults()
    assert list(d.sys_size) == [96, 96, 96]
    assert d.fmu == 0.002 and d.nlayers == 8 and d.max_extrap_rs == 5
    assert d.wt_n == 2.5 and d.weight_fac == 0.25 and d.num_iters == 5


def test_cavity_cfg(tmp_path):
    p = scenes.write(str(tmp_path / "c.cfg"), scenes.cavity(32, 64))
    d = R.desc_from_cfg(p)
    assert list(d.sys_size) == [32, 32, 32]
    assert list(d.periodic) == [0, 0, 0]
    assert d.bcv[0][5] == 1.0 and d.bct[0][5] == 1
    assert list(d.walls) == [1] * 6
    assert d.wall_dist == pytest.approx(1 / 32)
    assert d.stop_short == 64 and d.n_obj == 0


def test_periodicity_from_bc_sums(tmp_path):
    p = scenes.write(str(tmp_path / "s.cfg"), scenes.stretched_sphere(32, 4))
    d = R.desc_from_cfg(p)
    assert list(d.periodic) == [1, 1, 1]
    assert d.n_obj == 1 and d.obj[0].type == 1
    assert d.obj[0].extra[1] == pytest.approx(1.3 ** 0.5)


def test_unknown_keyword_is_an_error(tmp_path):
    p = str(tmp_path / "bad.cfg")
    with open(p, "w") as f:
        f.write("sys_size 8 8 8\nnot_a_keyword 3\n")
    with pytest.raises(R.RMT3DError) as e:
        R.desc_from_cfg(p)
    assert "not_a_keyword" in str(e.value)


def test_cfg_name_must_end_in_cfg(tmp_path):
    with pytest.raises(R.RMT3DError):
        R.desc_from_cfg(str(tmp_path / "x.txt"))


@pytest.mark.parametrize("name", ["cavity16", "sphere24", "stretch24"])
def test_stepper_dt_matches_reference(tmp_path, name):
    fx = H.load_fixture(name)
    d = R.desc_from_cfg(H.fixture_cfg(fx, str(tmp_path / "f.cfg")))
    dt_reg = H.state(fx, 0)["dt"]  # init_iter leaves dt = dt_reg
    dt, steps = R.stepper_dt(d, dt_reg)
    # the reference build lets GCC contract a*b+c into FMA (its C++ default), so
    # agreement is to the last bit or two
    assert dt == pytest.approx(H.state(fx, 1)["dt"], rel=5e-16, abs=0)
    assert steps >= 1


def test_random_scene_is_seeded_and_disjoint(tmp_path):
    n1, t1 = scenes.random_scene(7)
    n2, t2 = scenes.random_scene(7)
    assert (n1, t1) == (n2, t2)
    d = R.desc_from_cfg(scenes.write(str(tmp_path / "r.cfg"), t1))
    assert 1 <= d.n_obj <= 8
    dx = 1.0 / n1
    for a in range(d.n_obj):
        for b in range(a):
            ca, cb = np.array(d.obj[a].basic[:3]), np.array(d.obj[b].basic[:3])
            gap = np.linalg.norm(ca - cb) - d.obj[a].basic[3] - d.obj[b].basic[3]
            assert gap >= 2 * dx


def test_precision_forms(tmp_path):
    """The extension keywords select the arithmetic form and the mixed forms'
    solve tolerance; a form outside the three is refused before any device
    work."""
    text = scenes.cavity(16, 4) + "precision 2\nmixed_rtol 1e-6\n"
    d = R.desc_from_cfg(scenes.write(str(tmp_path / "p.cfg"), text))
    assert d.precision == R.MIXED_BULK32 and d.mixed_rtol == 1e-6
    assert R.desc_from_cfg(scenes.write(str(tmp_path / "q.cfg"), scenes.cavity(16, 4))).precision == R.FP64
    d.precision = 3
    with pytest.raises(R.RMT3DError) as e:
        R.Scene(d)
    assert "precision" in str(e.value)
