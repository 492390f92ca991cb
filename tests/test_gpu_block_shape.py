"""The block shape of the bulk stencil kernels (rmt3d_scene_set_block_shape)
changes only which block computes a cell, never a cell's arithmetic: whole
steps give the same bits under every shape, for walled and periodic boxes,
constant and variable density, FP64 and the mixed form."""
import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "q", "dp")


def run(tmp_path, name, precision, shape, steps=3):
    fx = H.load_fixture(name)
    cfg = H.fixture_cfg(fx, str(tmp_path / (name + ".cfg")))
    sc = R.Scene.from_cfg(cfg, precision=precision, var_den=int(fx.get("varden", 0)))
    try:
        sc.set_block_shape(shape)
        sc.prepare()
        assert sc.run(steps) == R.NORMAL_EXIT
        return {f: sc.field(f).copy() for f in FIELDS}
    finally:
        sc.close()


@pytest.mark.parametrize("name", ["cavity16", "stretch24", "varden24", "multi24"])
@pytest.mark.parametrize("precision", [R.FP64, R.MIXED])
def test_block_shapes_bit_identical(tmp_path, name, precision):
    ref = run(tmp_path, name, precision, 0)
    for shape in range(1, R._lib.BLOCK_SHAPES):
        got = run(tmp_path, name, precision, shape)
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), (name, precision, shape, f)


def test_block_shape_out_of_range(tmp_path):
    fx = H.load_fixture("cavity16")
    sc = R.Scene.from_cfg(H.fixture_cfg(fx, str(tmp_path / "c.cfg")))
    try:
        for bad in (-1, R._lib.BLOCK_SHAPES):
            with pytest.raises(R.RMT3DError):
                sc.set_block_shape(bad)
    finally:
        sc.close()
