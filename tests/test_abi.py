"""The C ABI library loads without a GPU, exports every function include/*.h
declares, and rejects bad inputs on the host with the documented status codes."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np

from conftest import ROOT, has_gpu


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^[A-Za-z_][\w \*]*?\b(mc3d_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_every_declared_symbol_is_exported(engine):
    names = declared_functions()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", str(engine.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(\w+)$", out, flags=re.M))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = C.CDLL(str(engine.LIB_PATH))
    for n in names:
        getattr(lib, n)
    assert lib.mc3d_abi_version() == 2


def _inputs(engine):
    g = engine.Geometry(np.ones((4, 4, 4), np.uint8), 0.1, 0.1, 0.1)
    p = engine.OpticalProps.from_tissues([(0.1, 10, 0.9, 1.4)])
    return g, p


def _status(engine, fn):
    try:
        fn()
    except engine.Mc3dError as e:
        return e.status
    return 0


def test_host_side_validation(engine, table):
    g, p = _inputs(engine)
    run = engine.run
    J = engine.Job
    assert _status(engine, lambda: run([g], [p], [J(photons=10, seed=0)], table)) == -5
    assert _status(engine, lambda: run([g], [p], [J(photons=10, seed=(4294967117 << 32))],
                                       table)) == -5
    assert _status(engine, lambda: run([g], [p], [J(photons=10)], table[:1])) == -6
    bad_tab = table[:10].copy()
    bad_tab[3] = 1
    assert _status(engine, lambda: run([g], [p], [J(photons=10)], bad_tab)) == -6
    g2 = engine.Geometry(np.full((4, 4, 4), 3, np.uint8), 0.1, 0.1, 0.1)
    assert _status(engine, lambda: run([g2], [p], [J(photons=10)], table)) == -3
    only_air = engine.OpticalProps(np.zeros(1), np.zeros(1), np.zeros(1), np.ones(1))
    assert _status(engine, lambda: run([g], [only_air], [J(photons=10)], table)) == -4
    g0 = engine.Geometry(np.ones((4, 4, 4), np.uint8), 0.0, 0.1, 0.1)
    assert _status(engine, lambda: run([g0], [p], [J(photons=10)], table)) == -2
    assert _status(engine, lambda: run([g], [p], [J(geom=1, photons=10)], table)) == -1
    assert _status(engine, lambda: run([g], [p], [J(photons=10, streams=5, stream_first=3,
                                                    stream_count=4)], table)) == -1
    assert _status(engine, lambda: run([g], [p], [J(photons=10)], table, block=100)) == -1
    big = [engine.OpticalProps.from_tissues([(0.1, 10, 0.9, 1.4)] * 255)] * 60
    assert _status(engine, lambda: run([g], big, [J(photons=10)], table)) == -11
    if not has_gpu():
        assert _status(engine, lambda: run([g], [p], [J(photons=10)], table)) == -8
    opt = engine._options()
    opt.steps = 7  # neither MC3D_STEPS_MERGED nor MC3D_STEPS_VOXEL
    gg, pp, jj = engine._arrays([g], [p], [J(photons=10)])
    _, outs = engine._outs([g], [J(photons=10)])
    assert engine.lib().mc3d_run(gg, 1, pp, 1, jj, 1, table.ctypes.data, len(table),
                                 C.byref(opt), outs) == -1


def test_reference_shaped_entry_needs_table(engine, tmp_path, monkeypatch):
    """mc3d_run_3dmc_gpu reads ./safeprimes_base32.txt like rng_init
    (src/mc3d_rng.cu:16) and reports a missing file instead of exiting"""
    monkeypatch.chdir(tmp_path)
    g, p = _inputs(engine)
    tt = g.tissue.astype(np.int32)
    geo = engine.CRefGeometry(0.1, 0.1, 0.1, 0.4, 0.4, 0.4, 4, 4, 4, tt.ctypes.data)
    props = engine.CRefOptProps(2, p.n.ctypes.data, p.mua.ctypes.data, p.mus.ctypes.data,
                                p.g.ctypes.data, 0)
    R = np.zeros(16)
    fin = C.c_int(0)
    st = engine.lib().mc3d_run_3dmc_gpu(geo, props, 100, R.ctypes.data, None, None, None, None,
                                        C.byref(fin))
    assert st == -6


def test_noalloc_rejects_non_finite_values(engine, table):
    """mc3d_run_noalloc checks voxel sizes and optical values like mc3d_run, before
    it touches the device (the pointers below are never dereferenced)"""
    g, p = _inputs(engine)
    lib = engine.lib()
    fake = C.c_void_p(0x1000)  # non-null stand-in for device buffers
    tab = np.ascontiguousarray(table[:1000])
    cj = engine.Job(0, 0, 10, 1796308352, "uniform").c()

    def call(cg, cp):
        return lib.mc3d_run_noalloc(C.byref(cg), C.byref(cp), C.byref(cj), tab.ctypes.data,
                                    len(tab), 0, None, fake, fake, fake, fake)

    cp = p.c()
    for bad in (float("inf"), float("nan")):
        for axis in range(3):
            d = [0.1, 0.1, 0.1]
            d[axis] = bad
            assert call(engine.CGeom(4, 4, 4, 0, *d, 0x1000), cp) == -2
    cg = engine.CGeom(4, 4, 4, 0, 0.1, 0.1, 0.1, 0x1000)
    for field in ("mua", "mus", "g", "n"):
        for bad in (float("inf"), float("nan")):
            q = engine.OpticalProps(p.mua.copy(), p.mus.copy(), p.g.copy(), p.n.copy())
            getattr(q, field)[1] = bad
            assert call(cg, q.c()) == -4
