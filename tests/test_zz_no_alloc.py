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


def _rejected_streams(table, seed, streams):
    """streams whose seeding needed more than one attempt, by the loop of init_RNG
    (gpumcml_rng/gpumcml_rng.cu:95-114)"""
    begin, x, n = int(table[0]), int(seed), 0
    for i in range(streams):
        fora = int(table[1 + i % (len(table) - 1)])
        first = True
        while True:
            x1 = (x & 0xFFFFFFFF) * begin + (x >> 32)
            carry = int((x1 & 0xFFFFFFFF) / 4294967296.0 * fora)
            x = (x1 & 0xFFFFFFFF) * begin + (x1 >> 32)
            st = (carry << 32) + (x & 0xFFFFFFFF)
            if st != 0 and (st >> 32) < fora - 1 and (st & 0xFFFFFFFF) < 0xFFFFFFFF:
                break
            if first:
                n += 1
                first = False
    return n


def test_noalloc_with_rejected_seeds(engine):
    """a table of tiny multipliers makes init_RNG reject seeding attempts; the
    rejection list lives in the static array too, and both calls still match
    mc3d_run word for word.  Past MC3D_NOALLOC_MAX_REJECTIONS rejected streams the
    call refuses before it launches anything."""
    import torch

    small = np.array([4294967118] + [3, 5, 7, 11, 13, 17] * 50, np.uint32)
    g = engine.Geometry(np.ones((16, 16, 16), np.uint8), 0.1, 0.1, 0.1)
    p = engine.OpticalProps.from_tissues([(0.1, 10.0, 0.9, 1.4)])
    job = engine.Job(0, 0, 1500, 55555, "uniform")
    nrej = _rejected_streams(small, job.seed, job.num_streams())
    assert 0 < nrej <= 4096
    ref = engine.run([g], [p], [job], table=small, steps="voxel")[0]

    dev = torch.device("cuda", 0)
    tissue = torch.from_numpy(g.tissue.reshape(-1).copy()).to(dev)
    outs = [torch.zeros(256, dtype=torch.int64, device=dev) for _ in range(3)]
    totals = torch.zeros(14, dtype=torch.int64, device=dev)
    cg = engine.CGeom(16, 16, 16, 0, g.dx, g.dy, g.dz, tissue.data_ptr())
    cp, cj = p.c(), job.c()
    lib = engine.lib()
    for _ in range(2):
        st = lib.mc3d_run_noalloc(C.byref(cg), C.byref(cp), C.byref(cj), small.ctypes.data,
                                  len(small), 0, None, *[o.data_ptr() for o in outs],
                                  totals.data_ptr())
        assert st == 0, lib.mc3d_last_error()
        torch.cuda.synchronize(dev)
        drs, sq, tr = [o.cpu().numpy().view(np.uint64).reshape(16, 16) for o in outs]
        tot = dict(zip(engine.TOTAL_FIELDS, map(int, totals.cpu().numpy().view(np.uint64))))
        assert tot == ref.totals
        assert np.array_equal(drs, ref.drs) and np.array_equal(sq, ref.drs_sq)
        assert np.array_equal(tr, ref.trans)

    many = engine.Job(0, 0, 40_000, 55555, "uniform")
    assert _rejected_streams(small, many.seed, many.num_streams()) > 4096
    cm = many.c()
    st = lib.mc3d_run_noalloc(C.byref(cg), C.byref(cp), C.byref(cm), small.ctypes.data,
                              len(small), 0, None, *[o.data_ptr() for o in outs],
                              totals.data_ptr())
    assert st == -11  # MC3D_ERR_CAPACITY
