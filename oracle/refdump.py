"""Reader for the oracle driver's state dumps (oracle/ref_driver.cc).

Test infrastructure: returns the reference's AoS arrays (struct field and
struct ref_map, F3D_Source/fields.hh:34-646) and the extrapolated-map list.
"""
import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from rmt3d_b200.layout import FIELD_DT, REFMAP_DT  # noqa: E402  (the records the dump holds)


def read(path):
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:4] == b"RMTD", "not an oracle dump"
    hdr = np.frombuffer(raw, "<i4", 11, 4)
    ver, m, n, o, sm4, sn4, so4, steps, n_ext, fsz, rsz = [int(v) for v in hdr]
    assert ver == 1 and fsz == 360 and rsz == 488
    off = 4 + 44
    dt, time = np.frombuffer(raw, "<f8", 2, off)
    off += 16
    nc = sm4 * sn4 * so4
    fields = np.frombuffer(raw, FIELD_DT, nc, off).copy()
    off += 360 * nc
    refmaps = np.frombuffer(raw, REFMAP_DT, nc, off).copy()
    off += 488 * nc
    rec = np.dtype([("index", "<i4"), ("pad", "<i4"), ("map", REFMAP_DT)])
    ext = np.frombuffer(raw, rec, n_ext, off).copy()
    return {"m": m, "n": n, "o": o, "shape": (so4, sn4, sm4), "steps": steps, "dt": float(dt), "time": float(time),
            "fields": fields, "refmaps": refmaps, "ext_index": ext["index"].copy(), "ext_maps": ext["map"].copy()}


def read_fields(path):
    """A compact dump (ref_driver ... fields k1,k2,...): dt, time and the
    velocity components and pressure over the ghosted box, as
    {"shape": (so4, sn4, sm4), "steps", "dt", "time", "u", "v", "w", "p"}."""
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:4] == b"RMTF", "not a compact oracle dump"
    ver, m, n, o, sm4, sn4, so4, steps = [int(v) for v in np.frombuffer(raw, "<i4", 8, 4)]
    assert ver == 1
    dt, time = np.frombuffer(raw, "<f8", 2, 36)
    nc = sm4 * sn4 * so4
    arr = np.frombuffer(raw, "<f8", 4 * nc, 52).reshape(4, so4, sn4, sm4)
    out = {"m": m, "n": n, "o": o, "shape": (so4, sn4, sm4), "steps": steps, "dt": float(dt), "time": float(time)}
    for c, name in enumerate("uvwp"):
        out[name] = arr[c].copy()
    return out
