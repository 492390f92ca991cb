"""Parity of the CUDA FSI step with the reference (the oracle's golden states).

Every Poisson solve on both sides is converged to round-off (mg_exact on the
GPU, RMT3D_SHIM_EXACT in the oracle), so the comparison is not limited by the
reference's residual tolerance.  The CUDA path is built without floating-point
contraction, so its states are compared with the reference built the same way
(the fixtures' ``n<k>_*`` states); the reference's own build (FMA contraction
on, ``s<k>_*``) is a second, equally valid rounding of the same computation.

* One step from the reference's own state must agree to rel-L2 1e-10.
* varden24 (one sphere of density 1.5) and multi24 (three spheres of
  densities 0.8, 1.2, 1.0) are states of the reference's VAR_DEN build and
  run the variable-density form (1/rho-weighted MAC and FEM operators).
* collide24 holds two spheres 0.02 apart, whose transition bands overlap:
  the collision stress between solids (fluid_3d.cc:1465-1773) is active.
* wall24 holds a sphere 0.05 above the bottom wall under gravity: the wall
  repulsion and gravity terms of the accelerations are active.
* ftest16 is the manufactured solution on a periodic box (sim_ftest), whose
  body force drives the flow.
* Over several steps two roundings of the reference drift apart by an amount
  stored in each fixture (``s<k>_envf``: the rel-L2 difference between the
  reference built with and without FMA contraction, both solving exactly).
  Where that difference is above round-off, discrete branches of the
  algorithm (limiter cases, upwinding signs, extrapolation weights) meet
  quantities that are zero in exact arithmetic and take either side, and the
  difference, once opened, stays in the state (it need not grow: the wall24
  envelope is 1.3e-5 after one step and 1.7e-6 after four).  Multi-step
  results must lie within ENV_FACTOR times the largest envelope up to that
  step (up to step 1 for the state after the set-up, whose pressure
  pre-iterations run with the velocity at rest), or 1e-10, whichever is
  larger.  Measured on a B200 the CUDA path's error is 0.5 to 2.5 times that
  envelope in most cases; the largest ratio, 8.5, is sphere24 after one step,
  which starts from a set-up whose pressure (after five pressure
  pre-iterations solved to round-off by both sides, each with its own
  multigrid) differs from the reference's by 1e-9.  1e-10 holds through one
  step from the reference's state (to 3e-13), and through every step where
  the reference's own two roundings agree to 1e-12: multi24, collide24,
  ftest16.  The residual-tolerance part of the
  envelope (``s<k>_envt``) does not apply: both sides solve exactly.

Velocity components are compared relative to the norm of the whole velocity
field; pressure and the reference map relative to their own norms.  Every
test prints the measured errors.
"""
import os

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

pytestmark = pytest.mark.gpu

TOL = 1e-10       # rel-L2 per field, FP64 plain form
ENV_FACTOR = 10   # multi-step bound in units of the reference's own rounding envelope

CASES = ["cavity16", "sphere24", "stretch24", "varden24", "multi24", "collide24", "wall24", "ftest16"]


def envelope(fx, k):
    """The reference's rounding envelope (no-FMA against FMA build, exact
    solves) of its whole state -- the largest of its per-group envelopes, since
    a perturbation of one group feeds the others within a step -- largest over
    the saved steps up to k (up to 1 for k = 0)."""
    saved = sorted(int(key[1:].split("_")[0]) for key in fx if key.startswith("s") and key.endswith("_envf"))
    return max(float(np.max(fx["s%d_envf" % j])) for j in saved if j <= max(k, 1))


def bound(fx, k):
    """Tolerance at step k: ENV_FACTOR times the envelope, or TOL."""
    return max(TOL, ENV_FACTOR * envelope(fx, k))


def vec_errors(scene, st):
    shp = st["shape"]
    ref = np.stack([st["vel"][c].reshape(shp)[H.INTERIOR] for c in range(3)])
    got = np.stack([scene.field(n)[H.INTERIOR] for n in "uvw"])
    scale = np.linalg.norm(ref)
    scale = scale if scale > 0 else 1.0  # the initial state is at rest
    out = {n: float(np.linalg.norm(got[c] - ref[c]) / scale) for c, n in enumerate("uvw")}
    out["p"] = H.rel_l2(scene.field("p")[H.INTERIOR], st["p"].reshape(shp)[H.INTERIOR])
    return out


def map_errors(scene, st):
    e = H.compare_state(scene, st, 1)
    return {k: e[k] for k in ("prim_mismatch", "ext_mismatch", "xi")}


def make_scene(tmp_path, name, exact=1, prepare=True):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / (name + ".cfg")))
    # fixtures made with the reference's VAR_DEN build run the variable-density form
    sc = R.Scene.from_cfg(cfg, mg_exact=exact, var_den=int(fx.get("varden", 0)))
    if prepare:
        sc.prepare()
    return fx, sc


STEPS = {"cavity16": [1, 8]}


@pytest.mark.parametrize("name", CASES)
def test_full_path_matches_reference(tmp_path, name):
    """run_sim's set-up (initialize, dt fit, 5 pressure pre-iterations) and
    the first steps, against the reference's states."""
    fx, sc = make_scene(tmp_path, name)
    steps = STEPS.get(name, [1, 4])
    try:
        st0 = H.state(fx, 0, "n")
        assert sc.dt == pytest.approx(H.state(fx, 1, "n")["dt"], rel=5e-16)
        e = vec_errors(sc, st0)
        print("\n%s step 0: %s (bound %.3g)" % (name, e, bound(fx, 0)))
        assert e["p"] < bound(fx, 0), e
        if sc.desc.n_obj:
            m = map_errors(sc, st0)
            assert m["prim_mismatch"] == 0 and m["ext_mismatch"] == 0 and m["xi"] < bound(fx, 0), m
        done = 0
        for k in steps:
            assert sc.run(k - done) == R.NORMAL_EXIT
            done = k
            st = H.state(fx, k, "n")
            e = vec_errors(sc, st)
            m = map_errors(sc, st) if sc.desc.n_obj else {}
            print("%s step %d: %s %s (bound %.3g, envelope %.3g)" % (name, k, e, m, bound(fx, k),
                                                                     envelope(fx, k)))
            assert max(e["u"], e["v"], e["w"]) < bound(fx, k), (k, e)
            assert e["p"] < bound(fx, k), (k, e)
            if sc.desc.n_obj:
                assert m["prim_mismatch"] == 0 and m["ext_mismatch"] == 0, (k, m)
                assert m["xi"] < bound(fx, k), (k, m)
    finally:
        sc.close()


@pytest.mark.parametrize("name", CASES)
def test_single_step_from_reference_state(tmp_path, name):
    """One step from the reference's own state (imported in its AoS layout)."""
    fx, sc = make_scene(tmp_path, name)
    try:
        st0, st1 = H.state(fx, 0, "n"), H.state(fx, 1, "n")
        fa, ra, ei, em = H.to_aos(st0)
        sc.import_reference(fa, ra, ei, em, st1["dt"], st0["time"])
        assert sc.step_forward(0) == R.NORMAL_EXIT
        e = vec_errors(sc, st1)
        m = map_errors(sc, st1) if sc.desc.n_obj else {}
        print("\n%s one step from the reference state: %s %s" % (name, e, m))
        assert max(e.values()) < TOL, e
        if sc.desc.n_obj:
            assert m["prim_mismatch"] == 0 and m["ext_mismatch"] == 0 and m["xi"] < TOL, m
    finally:
        sc.close()


def test_varden_fixture_discriminates(tmp_path):
    """The variable-density fixtures really test the 1/rho-weighted operators:
    the constant-density projection misses them by far more than TOL."""
    fx = H.load_fixture("varden24")
    cfg = H.fixture_cfg(fx, str(tmp_path / "v.cfg"))
    sc = R.Scene.from_cfg(cfg, mg_exact=1, var_den=0)
    try:
        st0, st1 = H.state(fx, 0), H.state(fx, 1)
        fa, ra, ei, em = H.to_aos(st0)
        sc.import_reference(fa, ra, ei, em, st1["dt"], st0["time"])
        assert sc.step_forward(0) == R.NORMAL_EXIT
        e = vec_errors(sc, st1)
        assert max(e.values()) > 1e3 * TOL, e
    finally:
        sc.close()


def test_cavity32_64_steps(tmp_path):
    """The plain FP64 lid-driven cavity: 32^3, 64 steps, against the reference."""
    fx = H.load_fixture("cavity32_64")
    cfg = H.fixture_cfg(fx, str(tmp_path / "c32.cfg"))
    sc = R.Scene.from_cfg(cfg, mg_exact=1)
    try:
        sc.prepare()
        assert sc.run(64) == R.NORMAL_EXIT
        ref = np.stack([fx["nu"], fx["nv"], fx["nw"]])
        got = np.stack([sc.field(n)[H.INTERIOR] for n in "uvw"])
        scale = np.linalg.norm(ref)
        env = fx["envf"]
        e = {c: float(np.linalg.norm(got[i] - ref[i]) / scale) for i, c in enumerate("uvw")}
        e["p"] = H.rel_l2(sc.field("p")[H.INTERIOR], fx["np"])
        b = max(TOL, ENV_FACTOR * float(np.max(env)))
        print("\ncavity32_64 after 64 steps: %s (bound %.3g, envelope %s)" % (e, b, env))
        assert max(e.values()) < b, e
        assert sc.time == pytest.approx(float(fx["dt_time"][1]), rel=1e-14)
    finally:
        sc.close()


def test_reference_tolerance_noise_floor(tmp_path):
    """With the reference's own V-cycle control the answer differs from the
    round-off-converged one only at the tolerance-level noise floor (measured
    for the reference against itself: ~3e-7 after 8 steps at 16^3)."""
    fx, sc = make_scene(tmp_path, "cavity16", exact=0)
    try:
        assert sc.run(8) == R.NORMAL_EXIT
        e = vec_errors(sc, H.state(fx, 8))
        assert max(e.values()) < 1e-5, e
    finally:
        sc.close()


def test_incompressibility_and_symmetry(tmp_path):
    """Size-independent properties: the cavity set-up is mirror-symmetric in y
    (u, w even, v odd); round-off breaks the symmetry only as much as it does
    in the reference itself, and the FEM divergence norm stays small."""
    fx, sc = make_scene(tmp_path, "cavity16")
    try:
        sc.run(8)
        st = H.state(fx, 8)
        shp = st["shape"]

        def asym(u, v, w):
            return max(np.abs(u - u[:, ::-1, :]).max(), np.abs(w - w[:, ::-1, :]).max(),
                       np.abs(v + v[:, ::-1, :]).max())

        ref = asym(*[st["vel"][c].reshape(shp)[H.INTERIOR] for c in range(3)])
        got = asym(*[sc.field(n)[H.INTERIOR] for n in "uvw"])
        assert got <= 10 * ref + 1e-12, (got, ref)
        assert sc.diag(0) < 5e-3
    finally:
        sc.close()


def test_nan_input_is_reported(tmp_path):
    """A NaN planted in the host-side input surfaces as the reference's error
    path: the upwinding's averaging branch zeroes NaN normal face velocities
    (fluid_3d.cc:2167-2174), the MAC solve stays finite, and the NaN reaches
    the FEM projection, which step_forward reports as PROJECTION_ERR
    (fluid_3d.cc:543-553)."""
    fx, sc = make_scene(tmp_path, "cavity16")
    try:
        st0 = H.state(fx, 0)
        fa, ra, ei, em = H.to_aos(st0)
        so4, sn4, sm4 = st0["shape"]
        fa["vel"][10 + sm4 * (10 + sn4 * 10), 0] = np.nan  # an interior cell
        sc.import_reference(fa, ra, ei, em, H.state(fx, 1)["dt"], 0.0)
        assert sc.step_forward(0) == R.PROJECTION_ERR
    finally:
        sc.close()


def test_ftest_exact_solution(tmp_path):
    """The manufactured solution (sim_ftest, periodic 16^3, 4 steps): the
    mean squared errors against the exact solution, fluid_3d::error's report,
    match the reference's own report (run_sim's printed line, 10 decimals)
    and the same errors of the reference's state."""
    fx, sc = make_scene(tmp_path, "ftest16")
    try:
        assert sc.run(4) == R.NORMAL_EXIT
        mu, dx = 0.01, 1.0 / 16
        got = H.ftest_error(*[sc.field(c)[H.INTERIOR] for c in "uvwp"], sc.time, dx, mu)
        st = H.state(fx, 4, "n")
        shp = st["shape"]
        ref = H.ftest_error(*[st["vel"][c].reshape(shp)[H.INTERIOR] for c in range(3)],
                            st["p"].reshape(shp)[H.INTERIOR], st["time"], dx, mu)
        printed = fx["runsim_err"]
        print("\nftest16 errors (u, v, w, p) after 4 steps: ours %s, reference %s, run_sim printed %s"
              % (got, ref, printed[3:]))
        assert sc.time == pytest.approx(printed[0], rel=1e-13)
        assert np.allclose(got, ref, rtol=1e-8, atol=0), (got, ref)
        assert np.allclose(got, printed[3:], rtol=0, atol=6e-11), (got, printed)
        assert got.max() < 1e-3  # the scheme tracks the exact solution
    finally:
        sc.close()
