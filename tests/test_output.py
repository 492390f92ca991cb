"""Frame diagnostics and slice output against the reference's own files.

The fixture out16 holds what the reference's stepper wrote for the 16^3
cavity + sphere (frames 0 and 1, 2 steps per frame) with slice output and
frame diagnostics on (Sim/stepper.hh:378-474, 583-610;
F3D_Source/fluid_3d_io.cc:3-434): all 22 output types as y-slices in text
matrices, a subset as x-slices in gnuplot binary and as z-slices in
coordinate text, and macro.dat / centroid.dat.  run_sim here writes the same
files from the CUDA path; the values must agree to 1e-6 of each file's
scale (the reference's rounding envelope of this state is about 5e-8 of the
velocity field), owners, layers and the 100 markers of cells without a map
exactly.  A file's scale is its largest magnitude, and at least the
problem's own scale for the velocity components (the lid speed, 1) and
their differences (1/dx = 16), so that a nearly zero component is not
compared at its own tiny magnitude.
Quantities at round-off level (the divergence of projected face velocities,
the momentum across a symmetric plane) are compared with an absolute
1e-12.
"""
import os

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

REL = 1e-6
ABS = 1e-12
RUNS = ("y_matrix", "x_gnuplot", "z_text")
DISCRETE = ("OID", "LID", "J")
SCALE_FLOOR = {"vx": 1.0, "vy": 1.0, "vz": 1.0, "w": 1.0, "wx": 16.0, "wy": 16.0, "wz": 16.0, "div_eu": 16.0}


def fixture():
    return H.load_fixture("out16")


def files_of(fx, run):
    pre = "file_%s/" % run
    return {k[len(pre):]: bytes(fx[k]) for k in fx if k.startswith(pre)}


def parse(run, name, data):
    if name in ("macro.dat", "centroid.dat"):
        lines = data.decode().split("\n", 1)
        return np.array([float(t) for t in lines[1].split()])
    if run == "x_gnuplot":
        return np.frombuffer(data, dtype=np.float32).astype(np.float64)
    return np.array([float(t) for t in data.decode().split()])


def test_output_cfg_parses(tmp_path):
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg_x_gnuplot"]))
    r = R.desc_from_cfg(str(p)).run
    assert (r.dump_code, r.output_dim, r.output_ind, r.data_fmt) == (4, 0, 5, 2)
    assert r.out_flag == (1 << 0) | (1 << 6) | (1 << 8) | (1 << 12) | (1 << 19)


@pytest.mark.gpu
@pytest.mark.parametrize("run", RUNS)
def test_files_match_reference(tmp_path, monkeypatch, run):
    fx = fixture()
    wd = tmp_path / run
    wd.mkdir()
    (wd / "c.cfg").write_bytes(bytes(fx["cfg_" + run]))
    monkeypatch.chdir(wd)
    sc = R.run_sim("c.cfg", stop_short=2, mg_exact=1)
    sc.close()
    ref = files_of(fx, run)
    ours = sorted(os.listdir(str(wd / "c.out")))
    assert ours == sorted(ref), (ours, sorted(ref))
    for name, data in ref.items():
        got_raw = (wd / "c.out" / name).read_bytes()
        a = parse(run, name, got_raw)
        b = parse(run, name, data)
        assert a.shape == b.shape, name
        stem = name.split(".")[0]
        if stem in DISCRETE:
            assert np.array_equal(a, b), name
            continue
        assert np.array_equal(a == 100.0, b == 100.0), name
        scale = max(float(np.max(np.abs(b))) if b.size else 0.0, SCALE_FLOOR.get(stem, 0.0))
        err = np.abs(a - b)
        assert np.all(err <= REL * scale + ABS), (name, float(err.max()), scale)
        if name == "macro.dat":
            # frame and step columns, and the rank columns
            for col in (1, 2, 4, 6):
                assert np.array_equal(a[col::18], b[col::18]), col


@pytest.mark.gpu
def test_macro_values(tmp_path):
    """rmt3d_macro against direct host sums over the exported fields."""
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg_z_text"]))
    sc = R.Scene.from_cfg(str(p), mg_exact=1)
    try:
        sc.prepare()
        assert sc.run(3) == R.NORMAL_EXIT
        m = sc.macro()
        u = np.stack([sc.field(n)[H.INTERIOR] for n in "uvw"])
        d = sc.desc
        dv = (1.0 / d.sys_size[0]) * (1.0 / d.sys_size[1]) * (1.0 / d.sys_size[2])
        np.testing.assert_allclose([m.momentum[c] for c in range(3)], u.reshape(3, -1).sum(1) * dv, rtol=1e-12,
                                   atol=1e-18)
        assert m.kinetic == pytest.approx(0.5 * float((u * u).sum()) * dv, rel=1e-12)
        assert m.energy == pytest.approx(m.elastic + m.kinetic + m.potential, rel=1e-15)
        assert m.elastic > 0 and m.power == 0
        # face-velocity divergence extremes from the exported face velocities
        f = [sc.field("fvel%d%d" % (2 * a + 1, a))[H.INTERIOR] - sc.field("fvel%d%d" % (2 * a, a))[H.INTERIOR]
             for a in range(3)]
        div = d.sys_size[0] * f[0] + d.sys_size[1] * f[1] + d.sys_size[2] * f[2]
        assert m.div_u_max == pytest.approx(float(div.max()), abs=1e-13)
        assert m.div_u_min == pytest.approx(float(div.min()), abs=1e-13)
        assert m.div_u_l2 == pytest.approx(sc.diag(0), rel=1e-14)
        assert m.dev_detF == pytest.approx(sc.diag(5), rel=1e-14)
        # a single object's centroid agrees with compute_centroid
        for c in range(3):
            assert m.centroid[0][c] == pytest.approx(sc.diag(2 + c), rel=1e-13)
    finally:
        sc.close()


@pytest.mark.gpu
def test_slice_shapes_and_bounds(tmp_path):
    fx = fixture()
    p = tmp_path / "c.cfg"
    p.write_bytes(bytes(fx["cfg_z_text"]))
    sc = R.Scene.from_cfg(str(p), mg_exact=1)
    try:
        sc.prepare()
        assert sc.slice(0, 2, 3).shape == (16, 16)
        assert sc.slice(7, 2, 3).shape == (17, 17)  # pressure on the 17^2 nodes
        assert sc.slice(7, 0, 3).shape == (17, 17)
        assert not sc.slice(0, 1, 16).any()  # outside the cell range: zeros
        u = sc.field("u")
        np.testing.assert_array_equal(sc.slice(0, 1, 5), u[2:-2, 7, 2:-2])
        pr = sc.field("p")
        np.testing.assert_array_equal(sc.slice(7, 2, 4), pr[6, 2:-1, 2:-1])
        with pytest.raises(R.RMT3DError):
            sc.slice(22, 0, 0)
        with pytest.raises(R.RMT3DError):
            sc.slice(9, 0, 0, obj_id=2)
    finally:
        sc.close()
