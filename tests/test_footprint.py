"""Admission footprint (host-only arithmetic; no device calls).

rmt3d_scene_footprint mirrors the allocations of rmt3d_scene_create and the
multigrid set-up; the GPU tests check it equals what a scene holds.  Here:
the per-cell arithmetic and the multigrid hierarchy terms for the grids of
the synthetic workloads.
"""
import rmt3d_b200 as R
from rmt3d_b200 import scenes


def _desc(tmp_path, text, name):
    return R.desc_from_cfg(scenes.write(str(tmp_path / name), text))


def test_fluid_only_bytes(tmp_path):
    d = _desc(tmp_path, scenes.cavity(32), "c32.cfg")
    n = 36 ** 3
    fp = R.footprint(d)
    # 36 doubles per ghosted cell dominate; multigrid adds about 8/7 x 3
    # doubles per MAC cell and per FEM node
    mg = 3 * 8 * (32 ** 3 + 33 ** 3) * 8 / 7
    assert 36 * 8 * n < fp < 36 * 8 * n + 1.1 * mg + (1 << 20)


def test_objects_precision_and_size_order(tmp_path):
    base = _desc(tmp_path, scenes.cavity(64), "c64.cfg")
    sph = _desc(tmp_path, scenes.cavity_sphere(64), "s64.cfg")
    n = 68 ** 3
    # one object: 51 doubles + 2 ints of map state, frontier scratch of
    # 13 bytes per cell and object, the frontier lengths, and the list of
    # cells holding a map with its length; each array of the per-cell slab
    # takes a 256-byte multiple
    pad = lambda b: (b + 255) // 256 * 256
    assert R.footprint(sph) - R.footprint(base) == (n * (51 * 8 + 8) + pad(n) + 3 * n * 4 + pad(2 * 16 * 4) + n * 4 +
                                                    pad(4))
    mixed = _desc(tmp_path, scenes.cavity_sphere(64), "m64.cfg")
    mixed.precision = R.MIXED
    # the mixed form adds FP32 copies of the multigrid hierarchies; its FP32
    # advection form keeps the 18 face-state arrays in FP32
    assert R.footprint(mixed) > R.footprint(sph)
    bulk = _desc(tmp_path, scenes.cavity_sphere(64), "b64.cfg")
    bulk.precision = R.MIXED_BULK32
    assert R.footprint(mixed) - R.footprint(bulk) == 18 * n * 4
    sizes = [R.footprint(_desc(tmp_path, scenes.cavity(k), "k%d.cfg" % k)) for k in (32, 48, 64, 96, 128)]
    assert sizes == sorted(sizes)


def test_uncoarsenable_grid_has_no_footprint(tmp_path):
    d = _desc(tmp_path, scenes.cavity(32), "c.cfg")
    d.sys_size[0] = d.sys_size[1] = d.sys_size[2] = 31 * 37  # odd, large: no hierarchy
    assert R.footprint(d) == 0
