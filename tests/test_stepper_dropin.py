"""The drop-in seam: the reference's own stepper (Sim/stepper.hh, unchanged)
and run_sim sequence driving the GPU path through rmt3d_fluid_3d
(include/rmt3d_fluid_3d.hh).

tests/dropin/run_sim_gpu.cc is run_sim's sequence with rmt3d_fluid_3d in
place of fluid_3d; tests/dropin/build.py compiles it against the reference's
headers and links the reference's sim_params / write_params / stepper
objects from the oracle build.  On the GPU it runs the output workload of the
out16 fixture (16^3 cavity + sphere, 2 steps per frame, slices and macro.dat
on) and its files must match the reference's own files as the Python
run_sim's do (tests/test_output.py's rules).
"""
import os
import subprocess

import numpy as np
import pytest

import helpers as H
import test_output as T

BIN = os.path.join(H.HERE, "dropin", "_bin", "run_sim_gpu")


def test_dropin_builds_against_reference_stepper():
    import importlib.util
    spec = importlib.util.spec_from_file_location("dropin_build", os.path.join(H.HERE, "dropin", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    if b.ref_dir() is None or not os.path.isdir(b.OBJ):
        pytest.skip("the reference checkout or the oracle objects are not here")
    assert b.build() == BIN and os.access(BIN, os.X_OK)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(BIN), reason="run_sim_gpu not built (tests/dropin/build.py)")
@pytest.mark.parametrize("run", ["y_matrix", "z_text"])
def test_dropin_run_matches_reference_files(tmp_path, run):
    fx = T.fixture()
    txt = bytes(fx["cfg_" + run]).decode()
    assert "stop_short 1000" in txt
    (tmp_path / "c.cfg").write_text(txt.replace("stop_short 1000", "stop_short 2"))
    env = dict(os.environ, RMT3D_MG_EXACT="1")
    r = subprocess.run([BIN, "c.cfg"], cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ref = T.files_of(fx, run)
    ours = sorted(os.listdir(str(tmp_path / "c.out")))
    assert ours == sorted(ref), (ours, sorted(ref))
    worst = 0.0
    for name, data in ref.items():
        a = T.parse(run, name, (tmp_path / "c.out" / name).read_bytes())
        b = T.parse(run, name, data)
        assert a.shape == b.shape, name
        stem = name.split(".")[0]
        if stem in T.DISCRETE:
            assert np.array_equal(a, b), name
            continue
        assert np.array_equal(a == 100.0, b == 100.0), name
        scale = max(float(np.max(np.abs(b))) if b.size else 0.0, T.SCALE_FLOOR.get(stem, 0.0))
        err = np.abs(a - b)
        worst = max(worst, float(err.max()) / scale if scale else 0.0)
        assert np.all(err <= T.REL * scale + T.ABS), (name, float(err.max()), scale)
    print("\nrun_sim_gpu %s: %d files, largest error %.3g of the file's scale" % (run, len(ref), worst))
