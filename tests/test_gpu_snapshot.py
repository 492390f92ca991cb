"""rmt3d_snapshot_fields: each step's fields reach pinned host buffers
asynchronously while the next step runs; after rmt3d_snapshot_wait they equal
the synchronous rmt3d_get_field of the same state, step after step."""
import numpy as np
import pytest
import torch

import helpers as H
import rmt3d_b200 as R

pytestmark = pytest.mark.gpu


def test_snapshot_equals_sync_reads(tmp_path):
    fx = H.load_fixture("sphere24")
    sc = R.Scene.from_cfg(H.fixture_cfg(fx, str(tmp_path / "s.cfg")))
    try:
        sc.prepare()
        names = ("u", "v", "w", "p", "q")
        shp = (sc.so4, sc.sn4, sc.sm4)
        bufs = [torch.empty(shp, dtype=torch.float64, pin_memory=True) for _ in names]
        for step in range(3):
            assert sc.step_forward(0) == R.NORMAL_EXIT
            sc.snapshot(names, bufs)
            sc.snapshot_wait()
            for n, b in zip(names, bufs):
                assert np.array_equal(b.numpy(), sc.field(n)), (step, n)
        # two snapshots in flight: the second waits for the first's host copy
        assert sc.step_forward(0) == R.NORMAL_EXIT
        sc.snapshot(names, bufs)
        first = [sc.field(n).copy() for n in names]
        assert sc.step_forward(0) == R.NORMAL_EXIT
        second_bufs = [torch.empty(shp, dtype=torch.float64, pin_memory=True) for _ in names]
        sc.snapshot(names, second_bufs)
        sc.snapshot_wait()
        for n, b, f in zip(names, bufs, first):
            assert np.array_equal(b.numpy(), f), n
        for n, b in zip(names, second_bufs):
            assert np.array_equal(b.numpy(), sc.field(n)), n
    finally:
        sc.close()
