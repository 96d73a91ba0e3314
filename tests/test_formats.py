"""File formats against the reference's own readers and writer (src/mc3d_io.cu,
compiled into oracle/_ref/libref_io.so), and the engine's error behaviour."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import ROOT
from ymc3d_b200.workloads import (read_drs_file, write_geometry_file, write_optprops_file)

REF_IO = ROOT / "oracle" / "_ref" / "libref_io.so"


def ref_io():
    if not REF_IO.exists():
        pytest.skip("reference I/O not built (oracle/build_ref.py needs the reference checkout)")
    h = C.CDLL(str(REF_IO))
    h.ref_read_geometry.restype = C.c_int
    h.ref_read_geometry.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]
    h.ref_read_optprops.restype = C.c_int
    h.ref_read_optprops.argtypes = [C.c_char_p, C.c_void_p] + [C.c_void_p] * 4 + [C.c_int]
    h.ref_save_diff_refl.restype = None
    h.ref_save_diff_refl.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p, C.c_int,
                                     C.c_char_p]
    return h


def random_geometry(rng, nx=17, ny=11, nz=9):
    t = rng.integers(0, 6, size=(nz, ny, nx)).astype(np.uint8)
    return t, 0.013, 0.021, 0.017


def test_geometry_reader_matches_reference(engine, tmp_path):
    rng = np.random.default_rng(1)
    t, dx, dy, dz = random_geometry(rng)
    t[0, 0, :3] = 0  # air voxels: stored as 255 in the file
    path = tmp_path / "g.bin"
    write_geometry_file(path, t, dx, dy, dz)
    n3, d3 = np.zeros(3, np.int32), np.zeros(3, np.float32)
    ref_t = np.zeros(t.size, np.int32)
    assert ref_io().ref_read_geometry(str(path).encode(), n3.ctypes.data, d3.ctypes.data,
                                      ref_t.ctypes.data, ref_t.size) == 0
    g = engine.geometry_read_from_file(path)
    assert list(n3) == list(g.shape)
    assert np.array_equal(np.float32([g.dx, g.dy, g.dz]), d3)
    assert np.array_equal(g.tissue.reshape(-1).astype(np.int32), ref_t)
    assert np.array_equal(g.tissue, t)


def test_optprops_reader_matches_reference(engine, tmp_path):
    rows = [(0.5, 20, 0.8, 1.44), (0.05, 15, 0.85, 1.37), (0.011, 12.5, 0.9, 1.44)]
    path = tmp_path / "p.bid"
    write_optprops_file(path, rows)
    nt = C.c_int()
    arrs = [np.zeros(8, np.float32) for _ in range(4)]
    assert ref_io().ref_read_optprops(str(path).encode(), C.byref(nt),
                                      *[a.ctypes.data for a in arrs], 8) == 0
    p = engine.opticalprops_read_from_file(path)
    assert p.num_tissue_types == nt.value == 4
    for ours, ref in zip((p.mua, p.mus, p.g, p.n), arrs):
        assert np.array_equal(ours, ref[:4])


def test_drs_writer_matches_reference_bytes(engine, tmp_path):
    rng = np.random.default_rng(3)
    g = engine.Geometry(np.ones((4, 13, 19), np.uint8), 0.02, 0.03, 0.05)
    R = rng.uniform(0, 50, size=(13, 19))
    engine.save_diff_refl(str(tmp_path / "ours"), g, R, 12345)
    ref_io().ref_save_diff_refl(19, 13, 0.02, 0.03, R.ctypes.data, 12345,
                                str(tmp_path / "ref").encode())
    a = (tmp_path / "ours_drs.bin").read_bytes()
    b = (tmp_path / "ref_drs.bin").read_bytes()
    assert a == b
    data, dx, dy = read_drs_file(tmp_path / "ours_drs.bin")
    assert np.allclose(data, R / 12345) and dx == float(np.float32(0.02))


def test_error_behaviour(engine, tmp_path):
    with pytest.raises(engine.Mc3dError) as e:
        engine.geometry_read_from_file(tmp_path / "missing.bin")
    assert e.value.status == -9  # MC3D_ERR_IO (the reference calls fclose(NULL))
    bad = tmp_path / "2d.bin"
    np.array([2, 4, 4, 1], "<i4").tofile(bad)
    with pytest.raises(engine.Mc3dError) as e:
        engine.geometry_read_from_file(bad)
    assert e.value.status == -10  # "Binary is not 3D."
    t = np.ones((3, 4, 5), np.uint8)
    path = tmp_path / "trunc.bin"
    write_geometry_file(path, t, 0.1, 0.1, 0.1)
    path.write_bytes(path.read_bytes()[:-7])
    with pytest.raises(engine.Mc3dError) as e:
        engine.geometry_read_from_file(path)
    assert e.value.status == -10
    p = tmp_path / "big.bin"
    with open(p, "wb") as f:
        np.array([3, 2, 1, 1], "<i4").tofile(f)
        np.array([0.1, 0.1, 0.1], "<f8").tofile(f)
        np.array([7, 300], "<i4").tofile(f)  # 301 does not fit a uint8 tissue index
    with pytest.raises(engine.Mc3dError) as e:
        engine.geometry_read_from_file(p)
    assert e.value.status == -3
    q = tmp_path / "short.bid"
    np.array([2], "<i4").tofile(q)
    with pytest.raises(engine.Mc3dError) as e:
        engine.opticalprops_read_from_file(q)
    assert e.value.status == -10
