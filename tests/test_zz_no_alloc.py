"""The allocation-free divergence diagnostic, rmt3d_div_u_noalloc.

It serves hosts that cannot allocate device memory at the moment they need
the diagnostic (a host confined to a memory pool it must not grow, or a plugin
that is only handed device pointers): its scratch is a fixed array inside the
library instead of per-call or per-scene allocations.  This file is named so
that pytest collects it last.  The test calls the entry point through the C
ABI twice in a row on the same state and checks both results against the
allocating path, rmt3d_diag(kind 0), within the parity tolerance of the
single-step tests.
"""
import ctypes

import numpy as np
import pytest

import helpers as H
import rmt3d_b200 as R
from rmt3d_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _call(lib, desc, dt_basis, dvel, faces):
    size = (ctypes.c_int * 3)(*desc.sys_size)
    prd = (ctypes.c_int * 3)(*desc.periodic)
    bounds = (ctypes.c_double * 6)(*desc.bounds)
    dv = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in dvel])
    fv = (ctypes.c_void_p * 6)(*[t.data_ptr() if t is not None else None for t in faces])
    out = ctypes.c_double()
    code = lib.rmt3d_div_u_noalloc(size, prd, bounds, dt_basis, dv, fv, None, ctypes.byref(out))
    return code, out.value


@pytest.mark.parametrize("name", ["cavity16", "stretch24"])
def test_noalloc_div_u_matches_allocating_path(tmp_path, name):
    """cavity16 has walls on every face; stretch24 is periodic on every axis,
    where the right-hand side reads the periodic images in the ghost layers."""
    import torch

    lib = R.lib()
    fx = H.load_fixture(name)
    sc = R.Scene.from_cfg(H.fixture_cfg(fx, str(tmp_path / (name + ".cfg"))))
    try:
        sc.prepare()
        assert sc.run(2) == R.NORMAL_EXIT
        expected = sc.diag(0)
        assert expected > 0
        dvel = [torch.from_numpy(sc.field(n).copy()).cuda() for n in ("du", "dv", "dw")]
        faces = [None if sc.desc.periodic[f // 2] else
                 torch.from_numpy(sc.field("fvel%d%d" % (f, f // 2)).copy()).cuda() for f in range(6)]
        torch.cuda.synchronize()
        for _ in range(2):  # two calls in a row share the same scratch array
            code, got = _call(lib, sc.desc, sc.dt_reg, dvel, faces)
            assert code == _lib.OK, lib.rmt3d_last_error()
            assert abs(got - expected) <= TOL * abs(expected), (got, expected)
        # grids beyond the fixed scratch are refused, not truncated
        big = R.desc_from_cfg(H.fixture_cfg(fx, str(tmp_path / (name + "b.cfg"))))
        big.sys_size[0] = big.sys_size[1] = big.sys_size[2] = 96
        code, _ = _call(lib, big, sc.dt_reg, dvel, faces)
        assert code == _lib.ERR_TOO_LARGE
    finally:
        sc.close()
