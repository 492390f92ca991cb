"""Batched form and serving loop against scenes stepped alone.

A batch steps independent scenes of uneven grid sizes together (each on its
own stream, kernels overlapping on the device); the serving loop admits
requests over time under an HBM budget.  Each scene's result must be the same
as when the scene runs alone.  Every reduction (the step's and the
checksum's) sums in a fixed order.  A scene stepped inside a group of
several scenes -- in a batch, or served as a group with requests of its kind
-- runs its least-squares extrapolation with 4 lanes per frontier cell instead
of a warp (more cells in flight when the GPU is shared), which regroups
those sums: grouped scenes match to round-off (SAME_TOL).
"""
import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R
from rmt3d_b200 import _lib, scenes

pytestmark = pytest.mark.gpu

SAME_TOL = 1e-10      # grouped versus alone (round-off, through the solver's stopping test)


def _same(got, ref):
    """Per-field errors of a grouped scene against its solo run: velocity
    components against the whole velocity (a near-zero cross-flow component's
    own norm magnifies round-off), pressure against its own norm."""
    vn = np.sqrt(sum(np.linalg.norm(ref[f][H.INTERIOR]) ** 2 for f in "uvw")) or 1.0
    e = {f: float(np.linalg.norm(got[f][H.INTERIOR] - ref[f][H.INTERIOR]) / vn) for f in "uvw"}
    e["p"] = H.rel_l2(got["p"][H.INTERIOR], ref["p"][H.INTERIOR])
    return e


def _same_checksum(got, ref):
    """Checksums (sums of u^2, v^2, w^2, p^2): velocity terms against their
    total, pressure against itself."""
    vt = abs(ref[0]) + abs(ref[1]) + abs(ref[2])
    return [abs(got[c] - ref[c]) / (vt if c < 3 else abs(ref[3])) for c in range(4)]



def _descs(tmp_path):
    cfgs = [
        scenes.cavity(16, steps=4),
        scenes.cavity_sphere(24, steps=4, radius=0.25),
        scenes.cavity(32, steps=4, lid=0.7),
        scenes.cavity_sphere(16, steps=4, radius=0.3, G=3.0),
    ]
    out = []
    for i, c in enumerate(cfgs):
        out.append(R.desc_from_cfg(scenes.write(str(tmp_path / ("b%d.cfg" % i)), c)))
    return out


def _alone(desc, steps):
    sc = R.Scene(desc)
    try:
        sc.prepare()
        assert sc.run(steps) == R.NORMAL_EXIT
        return {f: sc.field(f) for f in ("u", "v", "w", "p")}, sc.checksum()
    finally:
        sc.close()


def test_alone_is_deterministic(tmp_path):
    """Every reduction sums in a fixed order: two runs agree bit for bit."""
    d = _descs(tmp_path)[1]
    a, ca = _alone(d, 3)
    b, cb = _alone(d, 3)
    for f in a:
        assert (a[f] == b[f]).all(), f
    assert list(ca) == list(cb)


def test_batch_matches_alone(tmp_path):
    descs = _descs(tmp_path)
    b = R.Batch(descs, host_threads=3)
    try:
        b.prepare()
        st = b.step(3)
        assert st == [R.NORMAL_EXIT] * len(descs)
        for i, d in enumerate(descs):
            ref, rc = _alone(d, 3)
            e = _same({f: b.field(i, f) for f in ref}, ref)
            assert max(e.values()) < SAME_TOL, (i, e)
            assert max(_same_checksum(b.checksum(i), rc)) < SAME_TOL, (i, b.checksum(i), rc)
    finally:
        b.close()


def test_autotune_choices_and_results(tmp_path):
    descs = _descs(tmp_path)[:3]
    b = R.Batch(descs, host_threads=2)
    try:
        b.prepare()
        tuned = b.autotune(probe_steps=2)
        sizes = sorted({d.sys_size[0] * d.sys_size[1] * d.sys_size[2] for d in descs})
        assert sorted(tuned) == sizes
        for vd, vu, cl, sm, cc, bs in tuned.values():
            assert (vd, vu) in [(2, 2), (1, 1), (1, 2), (2, 1), (3, 3)]
            assert cl in (0, 1) and sm in (0, 1) and cc in (0, 5000, 40000)
            assert 0 <= bs < R._lib.BLOCK_SHAPES
        assert b.step(3) == [R.NORMAL_EXIT] * len(descs)
        # another smoothing schedule converges to the same tolerance: the
        # fields agree with the default schedule at the solver's tolerance
        for i, d in enumerate(descs):
            ref, _ = _alone(d, 3)
            e = H.rel_l2(b.field(i, "u")[H.INTERIOR], ref["u"][H.INTERIOR])
            assert e < 1e-6, (i, e)
    finally:
        b.close()


def test_footprint_is_what_a_scene_allocates(tmp_path):
    for d in _descs(tmp_path):
        for prec in (R.FP64, R.MIXED, R.MIXED_BULK32):
            d.precision = prec
            sc = R.Scene(d)
            try:
                assert R.footprint(d) == sc.device_bytes
            finally:
                sc.close()


@pytest.mark.parametrize("grouped", [False, True])
def test_serve_same_alone_and_in_mix(tmp_path, grouped):
    """Each served request's result is its solo run's: bit for bit on
    streams, to round-off when requests of a kind step as a group."""
    descs = _descs(tmp_path)
    steps = 3
    # staggered arrivals: later requests arrive while earlier ones run
    reqs = [(0.0, steps, descs[0]), (0.0, steps, descs[1]), (0.02, steps, descs[2]),
            (0.05, steps, descs[3]), (0.05, steps, descs[1]), (0.1, steps, descs[2])]
    budget = sum(R.footprint(d) for _, _, d in reqs)
    res, summ = R.serve(reqs, budget, max_slots=3, grouped=grouped)
    assert summ["requests"] == len(reqs)
    assert 0 < summ["request_p50_s"] <= summ["request_p99_s"]
    assert 0 < summ["step_p50_ms"] <= summ["step_p99_ms"]
    assert summ["cellsteps_per_s"] > 0
    # the work overlapped: some request was admitted before another finished
    spans = sorted((r["admit_s"], r["finish_s"]) for r in res)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    for (arr, n, d), r in zip(reqs, res):
        assert r["status"] == R.NORMAL_EXIT and r["steps_done"] == n
        assert r["admit_s"] >= arr - 1e-6
        _, alone = _alone(d, n)
        if grouped:  # requests of one kind step as a group: round-off against alone
            assert max(_same_checksum(r["checksum"], alone)) < SAME_TOL, (r["checksum"], alone)
        else:
            assert list(r["checksum"]) == list(alone), (r["checksum"], alone)


@pytest.mark.parametrize("grouped", [False, True])
def test_serve_admission_by_budget(tmp_path, grouped):
    descs = _descs(tmp_path)
    big = max(R.footprint(d) for d in descs)
    reqs = [(0.0, 2, d) for d in descs]
    # room for one scene at a time (any two footprints exceed the budget
    # except pairs of small scenes): overlapping spans must fit together
    budget = int(big * 1.5)
    res, _ = R.serve(reqs, budget, max_slots=4, grouped=grouped)
    used = [R.footprint(d) for d in descs]
    assert all(r["status"] == R.NORMAL_EXIT for r in res)
    for i in range(len(res)):
        for j in range(i + 1, len(res)):
            overlap = res[i]["admit_s"] < res[j]["finish_s"] and res[j]["admit_s"] < res[i]["finish_s"]
            if overlap:
                assert used[i] + used[j] <= budget, (i, j)
    # a request larger than the whole budget is refused up front
    with pytest.raises(_lib.RMT3DError) as ei:
        R.serve(reqs, big // 2, max_slots=2, grouped=grouped)
    assert ei.value.code == _lib.ERR_TOO_LARGE


def _group_descs(tmp_path, precision=R.FP64, var_den=0):
    """Three 24^3 scenes that differ in their objects and lid speed (one group)
    and one 16^3 scene (a group of its own)."""
    cfgs = [
        scenes.cavity_sphere(24, steps=4, radius=0.25, rho=1.3),
        scenes.multi_sphere(24, 4, spheres=[((0.3, 0.3, 0.35), 0.15, 0.5, 0.8), ((0.7, 0.65, 0.4), 0.15, 2.0, 1.2)],
                            lid=0.7),
        scenes.cavity(24, steps=4, lid=1.3),
        scenes.cavity_sphere(16, steps=4, radius=0.3),
    ]
    out = []
    for i, c in enumerate(cfgs):
        d = R.desc_from_cfg(scenes.write(str(tmp_path / ("g%d.cfg" % i)), c))
        d.precision = precision
        d.var_den = var_den
        out.append(d)
    return out


@pytest.mark.parametrize("form", ["fp64", "mixed_vd", "bulk32_vd"])
def test_group_matches_alone(tmp_path, form):
    """Equally sized scenes step as one group (batched multigrid over the
    group); each scene's result is its solo result to round-off."""
    prec = {"fp64": R.FP64, "mixed_vd": R.MIXED, "bulk32_vd": R.MIXED_BULK32}[form]
    descs = _group_descs(tmp_path, prec, 0 if form == "fp64" else 1)
    b = R.Batch(descs, host_threads=2)
    try:
        b.prepare()
        assert b.step(2) == [R.NORMAL_EXIT] * len(descs)
        assert b.step(3) == [R.NORMAL_EXIT] * len(descs)
        for i, d in enumerate(descs):
            ref, _ = _alone(d, 5)
            e = _same({f: b.field(i, f) for f in ref}, ref)
            assert max(e.values()) < SAME_TOL, (i, e)
    finally:
        b.close()


def test_group_failure_is_isolated(tmp_path):
    """A scene of a group that fails stops at its failing step; the others of
    the group keep stepping and match their solo runs to round-off."""
    import ctypes

    descs = _group_descs(tmp_path)[:3]
    b = R.Batch(descs, host_threads=1)
    try:
        b.prepare()
        # plant a NaN in an interior cell of scene 2's velocity
        h = b.scene_handle(2)
        L = R.lib()
        dims = (ctypes.c_int * 6)()
        L.rmt3d_get_dims(h, dims)
        sm4, sn4, so4 = dims[0], dims[1], dims[2]
        from rmt3d_b200.layout import FIELD_DT, REFMAP_DT
        fa = np.zeros(sm4 * sn4 * so4, dtype=FIELD_DT)
        ra = np.zeros(sm4 * sn4 * so4, dtype=REFMAP_DT)
        cnt = ctypes.c_int()
        L.rmt3d_export_reference(h, fa.ctypes.data_as(ctypes.c_void_p), ra.ctypes.data_as(ctypes.c_void_p), None,
                                 None, 0, ctypes.byref(cnt))
        fa["vel"][10 + sm4 * (10 + sn4 * 10), 0] = np.nan
        dt = ctypes.c_double()
        L.rmt3d_get_scalar(h, 0, ctypes.byref(dt))
        ei = np.zeros(1, dtype=np.int32)
        em = np.zeros(1, dtype=REFMAP_DT)
        assert L.rmt3d_import_reference(h, fa.ctypes.data_as(ctypes.c_void_p), ra.ctypes.data_as(ctypes.c_void_p),
                                        ei.ctypes.data_as(ctypes.c_void_p), em.ctypes.data_as(ctypes.c_void_p), 0,
                                        dt.value, 0.0) == 0
        st = b.step(3)
        assert st[2] == R.PROJECTION_ERR and st[:2] == [R.NORMAL_EXIT] * 2
        for i in range(2):
            ref, _ = _alone(descs[i], 3)
            e = _same({f: b.field(i, f) for f in ref}, ref)
            assert max(e.values()) < SAME_TOL, (i, e)
    finally:
        b.close()
