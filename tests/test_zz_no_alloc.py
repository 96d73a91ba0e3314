"""The allocation-free entry point, mc3d_run_noalloc.

Some callers of this library cannot call cudaMalloc: code inside a framework whose
caching allocator owns the device memory, or a loop with a fixed memory budget.  For
them there is one extern "C" call whose working memory is a static device array of
fixed size.  This test hands it device buffers it allocated itself (the test may
allocate; the entry point does not), runs the same job twice in a row and compares
both results word for word with mc3d_run's.  The file sorts last so that a run
stopping at its first failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_mc3d_run_twice(engine, table):
    import torch

    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry

    g = layered_vessel_geometry(48, 40, 24, 0.1)
    p = engine.OpticalProps.from_tissues(LAYER_ROWS)
    tab = np.ascontiguousarray(table[:230401])  # MC3D_NOALLOC_MAX_TABLE lines
    job = engine.Job(0, 0, 300_000, 24681357, "uniform")
    ref = engine.run([g], [p], [job], table=tab, steps="voxel")[0]

    nx, ny, nz = g.shape
    dev = torch.device("cuda", 0)
    tissue = torch.from_numpy(g.tissue.reshape(-1).copy()).to(dev)
    outs = [torch.zeros(nx * ny, dtype=torch.int64, device=dev) for _ in range(3)]
    totals = torch.zeros(14, dtype=torch.int64, device=dev)
    cg = engine.CGeom(nx, ny, nz, 0, g.dx, g.dy, g.dz, tissue.data_ptr())
    cp, cj = p.c(), job.c()
    lib = engine.lib()
    for _ in range(2):
        st = lib.mc3d_run_noalloc(C.byref(cg), C.byref(cp), C.byref(cj), tab.ctypes.data,
                                  len(tab), 0, None, *[o.data_ptr() for o in outs],
                                  totals.data_ptr())
        assert st == 0, lib.mc3d_last_error()
        torch.cuda.synchronize(dev)
        drs, sq, tr = [o.cpu().numpy().view(np.uint64).reshape(ny, nx) for o in outs]
        tot = dict(zip(engine.TOTAL_FIELDS, map(int, totals.cpu().numpy().view(np.uint64))))
        assert tot == ref.totals
        assert np.array_equal(drs, ref.drs) and np.array_equal(sq, ref.drs_sq)
        assert np.array_equal(tr, ref.trans)

    # beyond the static array's limits the call refuses instead of allocating
    too_long = np.ascontiguousarray(table[:230402])
    st = lib.mc3d_run_noalloc(C.byref(cg), C.byref(cp), C.byref(cj), too_long.ctypes.data,
                              len(too_long), 0, None, *[o.data_ptr() for o in outs],
                              totals.data_ptr())
    assert st == -11  # MC3D_ERR_CAPACITY
