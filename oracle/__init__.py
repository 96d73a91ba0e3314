"""CPU oracle for YMC3D's photon-tracking path -- TEST INFRASTRUCTURE ONLY.

ctypes face of liboracle.so (mc3d_oracle.c, a line-by-line C restatement of the
reference; see its header for the file:line map).  Only tests/, the smoke test
and bench.py's CPU-baseline leg use it, as the checker; the engine never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
LIB64_PATH = HERE / "liboracle64.so"  # the same loop in FP64 with libm functions
TOTAL_FIELDS = ("photons", "steps", "w_launched", "r_in", "r_out", "t_in", "t_out", "absorbed",
                "rr_killed", "rr_created", "lost", "capped", "quickfix", "fresnel")
REC_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("ux", "<f4"), ("uy", "<f4"),
                      ("uz", "<f4"), ("W", "<f4"), ("s", "<f4"), ("steps", "<u4"),
                      ("tissue", "<u4"), ("rng", "<u8")])


class OGeom(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("pad", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("tissue", C.c_void_p)]


class OProps(C.Structure):
    _fields_ = [("ntypes", C.c_int32), ("pad", C.c_int32), ("mua", C.c_void_p),
                ("mus", C.c_void_p), ("g", C.c_void_p), ("n", C.c_void_p)]


class OJob(C.Structure):
    _fields_ = [("photons", C.c_int64), ("streams", C.c_int64), ("seed", C.c_uint64),
                ("beam", C.c_int32), ("pad", C.c_int32), ("max_steps", C.c_int64)]


_lib = None
_lib64 = None


def lib(f64: bool = False):
    global _lib, _lib64
    if (_lib64 if f64 else _lib) is None:
        path = LIB64_PATH if f64 else LIB_PATH
        if not path.exists():
            from . import build as _b
            _b.build()
        h = C.CDLL(str(path))
        h.orc_init_rng.restype = C.c_int
        h.orc_init_rng.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_int64, C.c_void_p,
                                   C.c_void_p]
        h.orc_rand_co.restype = None
        h.orc_rand_co.argtypes = [C.c_void_p, C.c_uint32, C.c_int64, C.c_void_p]
        h.orc_run.restype = C.c_int
        h.orc_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int,
                              C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p]
        for f in ("orc_logf", "orc_acosf", "orc_sinf"):
            getattr(h, f).restype = C.c_float
            getattr(h, f).argtypes = [C.c_float]
        h.orc_sincospif.restype = None
        h.orc_sincospif.argtypes = [C.c_float, C.c_void_p, C.c_void_p]
        h.orc_grid_coord_x.restype = C.c_int
        h.orc_grid_coord_x.argtypes = [C.c_float, C.c_float, C.c_float]
        if f64:
            _lib64 = h
        else:
            _lib = h
    return _lib64 if f64 else _lib


def init_rng(table: np.ndarray, seed: int, n: int):
    """init_RNG restated: (x, a) of streams 0..n-1; raises on an invalid seed."""
    table = np.ascontiguousarray(table, np.uint32)
    x = np.zeros(max(n, 1), np.uint64)
    a = np.zeros(max(n, 1), np.uint32)
    st = lib().orc_init_rng(table.ctypes.data, len(table), seed, n, x.ctypes.data, a.ctypes.data)
    if st:
        raise ValueError(f"orc_init_rng status {st}")
    return x[:n], a[:n]


def rand_co(x: int, a: int, n: int) -> np.ndarray:
    st = C.c_uint64(x)
    out = np.zeros(n, np.float32)
    lib().orc_rand_co(C.byref(st), a, n, out.ctypes.data)
    return out


def run(tissue: np.ndarray, dx: float, dy: float, dz: float, mua, mus, g, n, photons: int,
        streams: int, seed: int, table: np.ndarray, beam: int = 0, threads: int = 0,
        first: int = 0, count: int = -1, max_steps: int = 0, photon_log: bool = False,
        absorption_map: bool = False, f64: bool = False):
    """Simulate streams [first, first+count) of a job; returns dict with drs, drs_sq,
    trans ([ny, nx] uint64), totals and the optional per-photon log.  f64 runs the
    FP64 build of the same loop (geometry in the file's double voxel sizes)."""
    tissue = np.ascontiguousarray(tissue, np.uint8)
    nz, ny, nx = tissue.shape
    arrs = [np.ascontiguousarray(v, np.float32) for v in (mua, mus, g, n)]
    table = np.ascontiguousarray(table, np.uint32)
    geom = OGeom(nx, ny, nz, 0, dx, dy, dz, tissue.ctypes.data)
    props = OProps(len(arrs[0]), 0, *[a.ctypes.data for a in arrs])
    job = OJob(photons, streams, seed, beam, 0, max_steps)
    drs = np.zeros((ny, nx), np.uint64)
    drs_sq = np.zeros((ny, nx), np.uint64)
    trans = np.zeros((ny, nx), np.uint64)
    tot = np.zeros(len(TOTAL_FIELDS), np.uint64)
    log = np.zeros(max(photons, 1), REC_DTYPE) if photon_log else None
    amap = np.zeros((nz, ny, nx), np.uint64) if absorption_map else None
    st = lib(f64).orc_run(C.byref(geom), C.byref(props), C.byref(job), table.ctypes.data,
                       len(table), threads, first, count, drs.ctypes.data, drs_sq.ctypes.data,
                       trans.ctypes.data, tot.ctypes.data,
                       None if log is None else log.ctypes.data,
                       None if amap is None else amap.ctypes.data)
    if st:
        raise ValueError(f"orc_run status {st}")
    return {"drs": drs, "drs_sq": drs_sq, "trans": trans,
            "totals": {k: int(v) for k, v in zip(TOTAL_FIELDS, tot)},
            "photon_log": None if log is None else log[:photons], "absorption": amap}
