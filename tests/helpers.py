"""Shared test helpers: golden-fixture loading and field comparison."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from rmt3d_b200.layout import FIELD_DT, REFMAP_DT  # noqa: E402


def load_fixture(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def fixture_cfg(fx, path):
    with open(path, "w") as f:
        f.write(bytes(fx["cfg"]).decode())
    return path


def state(fx, k, prefix="s"):
    """State k of a fixture as a dict (shape, dt, time, fields...).  prefix
    "s": the reference as built by its own flags (FMA contraction on), exact
    solves; "n": the reference built without FMA contraction, exact solves --
    the rounding the CUDA path, built without contraction, follows."""
    g = lambda key: fx["%s%d_%s" % (prefix, k, key)]  # noqa: E731
    meta = g("meta")
    shp = tuple(int(v) for v in meta[4:7])
    return {
        "shape": shp,
        "dt": float(g("dt_time")[0]),
        "time": float(g("dt_time")[1]),
        "vel": g("vel"),
        "p": g("p"),
        "q": g("q"),
        "prim_index": g("prim_index"),
        "prim_c": g("prim_c"),
        "prim_x": g("prim_x"),
        "prim_xpred": g("prim_xpred"),
        "ext_index": g("ext_index"),
        "ext_c": g("ext_c"),
        "ext_x": g("ext_x"),
        "ext_xpred": g("ext_xpred"),
    }


def to_aos(st):
    """Rebuild the reference's AoS arrays from a compact state."""
    n = int(np.prod(st["shape"]))
    fields = np.zeros(n, dtype=FIELD_DT)
    fields["vel"] = st["vel"].T
    fields["p"] = st["p"]
    fields["q"] = st["q"]
    rm = np.zeros(n, dtype=REFMAP_DT)
    rm["grad_phi"] = -1e200
    rm["c"][st["prim_index"]] = st["prim_c"]
    rm["x"][st["prim_index"]] = st["prim_x"]
    rm["xpred"][st["prim_index"]] = st["prim_xpred"]
    ext = np.zeros(len(st["ext_index"]), dtype=REFMAP_DT)
    ext["grad_phi"] = -1e200
    ext["c"] = st["ext_c"]
    ext["x"] = st["ext_x"]
    ext["xpred"] = st["ext_xpred"]
    return fields, rm, st["ext_index"].astype(np.int32), ext


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


INTERIOR = (slice(2, -2),) * 3


def compare_state(scene, st, nobj):
    """Per-field rel-L2 errors of a GPU scene against a reference state, plus
    reference-map bookkeeping mismatches."""
    shp = st["shape"]
    out = {}
    for c, nm in enumerate("uvw"):
        out[nm] = rel_l2(scene.field(nm)[INTERIOR], st["vel"][c].reshape(shp)[INTERIOR])
    out["p"] = rel_l2(scene.field("p")[INTERIOR], st["p"].reshape(shp)[INTERIOR])
    if nobj:
        code, x, _ = scene.refmap(0)
        code = code.ravel()
        prim_ref = np.zeros(code.size, bool)
        prim_ref[st["prim_index"][(st["prim_c"] & 1023) == 1]] = True
        out["prim_mismatch"] = int((prim_ref != (code == 0)).sum())
        ext_ref = np.zeros(code.size, bool)
        sel = (st["ext_c"] & 1023) == 1
        ext_ref[st["ext_index"][sel]] = True
        out["ext_mismatch"] = int((ext_ref != (code > 0)).sum())
        xr = np.zeros((3, code.size))
        xr[:, st["prim_index"]] = st["prim_x"].T
        xr[:, st["ext_index"][sel]] = st["ext_x"][sel].T
        both = (code >= 0) & (prim_ref | ext_ref)
        xs = x.reshape(3, -1)
        out["xi"] = max(rel_l2(xs[c][both], xr[c][both]) for c in range(3))
    return out


# ---- the manufactured solution of sim_ftest (Sim/sim_manager.cc:139-167) ----
def ftest_velocity(x, y, z):
    tp = 2 * np.pi
    u = -np.sin(tp * x) * np.cos(tp * y) * np.cos(tp * z)
    v = 0.5 * np.cos(tp * x) * np.sin(tp * y) * np.cos(tp * z)
    w = 0.5 * np.cos(tp * x) * np.cos(tp * y) * np.sin(tp * z)
    return u, v, w


def ftest_exact(x, y, z, t, h, mu):
    """sim_ftest::exact: velocity at the cell centre (x, y, z), pressure at the
    cell's lower corner, at time t."""
    tp = 2 * np.pi
    u, v, w = ftest_velocity(x, y, z)
    c = np.cos(tp * t)
    xc, yc, zc = x - 0.5 * h, y - 0.5 * h, z - 0.5 * h
    p = 3 * np.pi * mu * np.cos(tp * xc) * np.cos(tp * yc) * np.cos(tp * zc)
    return u * c, v * c, w * c, p * (c - np.sin(tp * t) / (6 * np.pi * mu))


def ftest_error(u, v, w, p, t, dx, mu, x0=0.0):
    """fluid_3d::error (F3D_Source/fluid_3d.cc:2810-2858) on a periodic box
    (node grid = cell grid): the mean squared error of u, v, w over the cells
    and of p over the nodes.  u, v, w, p: interior arrays indexed [k, j, i]."""
    o, n, m = u.shape
    xs = x0 + (np.arange(m) + 0.5) * dx
    ys = x0 + (np.arange(n) + 0.5) * dx
    zs = x0 + (np.arange(o) + 0.5) * dx
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    eu, ev, ew, ep = ftest_exact(X, Y, Z, t, dx, mu)
    cnt = m * n * o
    return np.array([((eu - u) ** 2).sum() / cnt, ((ev - v) ** 2).sum() / cnt, ((ew - w) ** 2).sum() / cnt,
                     ((ep - p) ** 2).sum() / cnt])
