"""The reference-shaped entry point run to success.

mc3d_run_3dmc_gpu takes run_3dmc_gpu's arguments (src/mc3d_gpu.h:16) as
src/mc3d_main.cu:44-61 passes them: the geometry_t / opticalprops_t layouts by
value, caller-zeroed R and T of nx*ny doubles, A of nx*ny*nz floats.  It reads
./safeprimes_base32.txt like rng_init (src/mc3d_rng.cu:16) and the seed from
MC3D_SEED.  Its R, T, totals and finished count must be mc3d_run's tallies of the
same job divided by 2^32, accumulated onto what the caller passed, and A must come
back untouched."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_run_3dmc_gpu_matches_mc3d_run(engine, table, tmp_path, monkeypatch):
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    monkeypatch.chdir(tmp_path)
    tab = np.ascontiguousarray(table[:230401])
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", tab)
    seed = 1796308352
    monkeypatch.setenv("MC3D_SEED", str(seed))

    g = layered_vessel_geometry(40, 36, 20, 0.1)
    g.tissue[12:14, 5:9, 5:9] = 0  # in-volume air: photons freeze below the surface
    p = engine.OpticalProps.from_tissues(LAYER_ROWS)
    nx, ny, nz = g.shape
    photons = 150_000

    tt = np.ascontiguousarray(g.tissue.astype(np.int32))
    geo = engine.CRefGeometry(np.float32(g.dx), np.float32(g.dy), np.float32(g.dz),
                              np.float32(g.dx) * nx, np.float32(g.dy) * ny,
                              np.float32(g.dz) * nz, nx, ny, nz, tt.ctypes.data)
    props = engine.CRefOptProps(p.num_tissue_types, p.n.ctypes.data, p.mua.ctypes.data,
                                p.mus.ctypes.data, p.g.ctypes.data, 0)
    # the caller's arrays already hold something: the entry point accumulates
    R = np.full((ny, nx), 0.25)
    T = np.full((ny, nx), 0.5)
    A = np.arange(nx * ny * nz, dtype=np.float32)
    A0 = A.copy()
    r_tot, t_tot = C.c_double(1.0), C.c_double(2.0)
    fin = C.c_int(-1)
    st = engine.lib().mc3d_run_3dmc_gpu(geo, props, photons, R.ctypes.data, C.byref(r_tot),
                                        T.ctypes.data, C.byref(t_tot), A.ctypes.data,
                                        C.byref(fin))
    assert st == 0, engine.lib().mc3d_last_error()

    ref = engine.run([g], [p], [engine.Job(0, 0, photons, seed, "uniform")], table=tab)[0]
    q = 1.0 / engine.WEIGHT_SCALE
    assert fin.value == ref.photons == photons
    assert np.array_equal(R, 0.25 + ref.drs.astype(np.float64) * q)
    assert np.array_equal(T, 0.5 + ref.trans.astype(np.float64) * q)
    t = ref.totals
    assert r_tot.value == 1.0 + (t["r_in"] + t["r_out"]) * q
    assert t_tot.value == 2.0 + (t["t_in"] + t["t_out"]) * q
    assert t["t_in"] > 0 and t["r_in"] > 0
    assert np.array_equal(A, A0)


def test_run_3dmc_gpu_seed_changes_result(engine, table, tmp_path, monkeypatch):
    """two MC3D_SEED values give two different (valid) runs of the same job"""
    monkeypatch.chdir(tmp_path)
    tab = np.ascontiguousarray(table[:230401])
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", tab)
    g = engine.Geometry(np.ones((16, 16, 16), np.uint8), 0.1, 0.1, 0.1)
    p = engine.OpticalProps.from_tissues([(0.1, 10.0, 0.9, 1.4)])
    tt = np.ascontiguousarray(g.tissue.astype(np.int32))
    geo = engine.CRefGeometry(0.1, 0.1, 0.1, 1.6, 1.6, 1.6, 16, 16, 16, tt.ctypes.data)
    props = engine.CRefOptProps(2, p.n.ctypes.data, p.mua.ctypes.data, p.mus.ctypes.data,
                                p.g.ctypes.data, 0)
    outs = []
    for seed in (11, 12):
        monkeypatch.setenv("MC3D_SEED", str(seed))
        R = np.zeros(256)
        fin = C.c_int(0)
        assert engine.lib().mc3d_run_3dmc_gpu(geo, props, 20_000, R.ctypes.data, None, None,
                                              None, None, C.byref(fin)) == 0
        assert fin.value == 20_000
        outs.append(R)
    assert not np.array_equal(outs[0], outs[1])
