"""The reference's per-cell AoS records as numpy dtypes.

``FIELD_DT`` is ``struct field`` (F3D_Source/fields.hh:34-282): velocity,
pressure, pressure correction, MAC potential, velocity change, the limited
normal derivatives, the six face velocities and the lower-face stress rows,
360 bytes per cell.  ``REFMAP_DT`` is ``struct ref_map`` (fields.hh:285-646),
with its packed ``c`` word (object id and layer, F3D_Source/defs.hh:12-14),
488 bytes per cell.  ``rmt3d_import_reference`` and ``rmt3d_export_reference``
read and write arrays of exactly these records over the ghosted box.
"""
import numpy as np

FIELD_DT = np.dtype([("vel", "<f8", 3), ("p", "<f8"), ("dp", "<f8"), ("q", "<f8"), ("dvel", "<f8", 3),
                     ("nv_der", "<f8", (3, 3)), ("fvel", "<f8", (6, 3)), ("sigma", "<f8", (3, 3))])
REFMAP_DT = np.dtype([("c", "<u4"), ("pad", "<u4"), ("x", "<f8", 3), ("xpred", "<f8", 3), ("nv_der", "<f8", (3, 3)),
                      ("fx", "<f8", (6, 3)), ("sigma", "<f8", (3, 3)), ("elastic_energy", "<f8", 3),
                      ("detF", "<f8", 3), ("grad_phi", "<f8", (3, 3)), ("act_power", "<f8", 3)])
assert FIELD_DT.itemsize == 360 and REFMAP_DT.itemsize == 488
