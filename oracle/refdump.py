"""Reader for the oracle driver's state dumps (oracle/ref_driver.cc).

Test infrastructure: returns the reference's AoS arrays (struct field and
struct ref_map, F3D_Source/fields.hh:34-646) and the extrapolated-map list.
"""
import numpy as np

FIELD_DT = np.dtype([("vel", "<f8", 3), ("p", "<f8"), ("dp", "<f8"), ("q", "<f8"), ("dvel", "<f8", 3),
                     ("nv_der", "<f8", (3, 3)), ("fvel", "<f8", (6, 3)), ("sigma", "<f8", (3, 3))])
REFMAP_DT = np.dtype([("c", "<u4"), ("pad", "<u4"), ("x", "<f8", 3), ("xpred", "<f8", 3), ("nv_der", "<f8", (3, 3)),
                      ("fx", "<f8", (6, 3)), ("sigma", "<f8", (3, 3)), ("elastic_energy", "<f8", 3),
                      ("detF", "<f8", 3), ("grad_phi", "<f8", (3, 3)), ("act_power", "<f8", 3)])
assert FIELD_DT.itemsize == 360 and REFMAP_DT.itemsize == 488


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
