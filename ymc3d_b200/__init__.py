"""ymc3d_b200 -- B200-native photon tracking for YMC3D.

Python face of libmc3d.so (C ABI in include/mc3d.h).  The names follow the
reference: ``run_3dmc_gpu`` (src/mc3d_gpu.cu:388), ``geometry_read_from_file``
and ``opticalprops_read_from_file`` (src/mc3d_io.cu:16-169), ``save_diff_refl``
(src/mc3d_io.cu:218-227).  Everything runs through the CUDA library; there is no
CPU fallback, and a missing library raises at import of the first call.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
# MC3D_LIBRARY points the package at another build of the library (debug builds,
# A/B measurements); the default is the in-tree build
LIB_PATH = Path(os.environ.get("MC3D_LIBRARY", HERE / "libmc3d.so"))
WEIGHT_SCALE = 4294967296.0  # fixed point: Q(W) = round(W * 2^32)

MC3D_OK = 0
STATUS_NAMES = {
    0: "MC3D_OK", -1: "MC3D_ERR_ARG", -2: "MC3D_ERR_GEOMETRY", -3: "MC3D_ERR_TISSUE_RANGE",
    -4: "MC3D_ERR_PROPS", -5: "MC3D_ERR_SEED", -6: "MC3D_ERR_TABLE", -7: "MC3D_ERR_CUDA",
    -8: "MC3D_ERR_NO_DEVICE", -9: "MC3D_ERR_IO", -10: "MC3D_ERR_FORMAT",
    -11: "MC3D_ERR_CAPACITY", -12: "MC3D_ERR_CANCELLED",
}
BEAMS = {"uniform": 0, "pencil": 1}
MATH = {"fast": 0, "exact": 1, "f64": 2}
STEPS = {"merged": 0, "voxel": 1}
TOTAL_FIELDS = ("photons", "steps", "w_launched", "r_in", "r_out", "t_in", "t_out", "absorbed",
                "rr_killed", "rr_created", "lost", "capped", "quickfix", "fresnel")
DEFAULT_STREAMS = 1 << 40  # include/mc3d.h: one photon per stream unless a job says otherwise


class Mc3dError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


# ----------------------------------------------------------------- C structs
class CGeom(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("pad", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("tissue", C.c_void_p)]


class CProps(C.Structure):
    _fields_ = [("num_tissue_types", C.c_int32), ("pad", C.c_int32), ("mua", C.c_void_p),
                ("mus", C.c_void_p), ("g", C.c_void_p), ("n", C.c_void_p)]


class CJob(C.Structure):
    _fields_ = [("geom", C.c_int32), ("props", C.c_int32), ("beam", C.c_int32),
                ("pad", C.c_int32), ("photons", C.c_int64), ("streams", C.c_int64),
                ("seed", C.c_uint64), ("stream_first", C.c_int64), ("stream_count", C.c_int64)]


class CTotals(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in TOTAL_FIELDS]


class COut(C.Structure):
    _fields_ = [("drs", C.c_void_p), ("drs_sq", C.c_void_p), ("trans", C.c_void_p),
                ("absorption", C.c_void_p), ("totals", CTotals)]


PHOTON_RECORD_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("ux", "<f4"),
                                ("uy", "<f4"), ("uz", "<f4"), ("W", "<f4"), ("s", "<f4"),
                                ("steps", "<u4"), ("tissue", "<u4"), ("rng", "<u8")])


class COptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("math", C.c_int32), ("block", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("absorption_map", C.c_int32),
                ("use_graph", C.c_int32), ("max_steps", C.c_int64),
                ("photon_log", C.c_void_p), ("cancel", C.c_void_p), ("steps", C.c_int32),
                ("pad", C.c_int32)]


class CRefGeometry(C.Structure):
    _fields_ = [("sample_dx", C.c_float), ("sample_dy", C.c_float), ("sample_dz", C.c_float),
                ("length_x", C.c_float), ("length_y", C.c_float), ("length_z", C.c_float),
                ("num_x", C.c_int), ("num_y", C.c_int), ("num_z", C.c_int),
                ("tissue_type", C.c_void_p)]


class CRefOptProps(C.Structure):
    _fields_ = [("num_tissue_types", C.c_int), ("n", C.c_void_p), ("mua", C.c_void_p),
                ("mus", C.c_void_p), ("g", C.c_void_p), ("alloc_where", C.c_int)]


# ----------------------------------------------------------------- library
_lib = None

EXPORTS = {
    "mc3d_last_error": (C.c_char_p, []),
    "mc3d_abi_version": (C.c_int, []),
    "mc3d_default_options": (None, [C.c_void_p]),
    "mc3d_run": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                           C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "mc3d_plan_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                   C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p]),
    "mc3d_plan_execute": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc3d_plan_read": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc3d_plan_shape": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mc3d_plan_device_totals": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mc3d_plan_destroy": (None, [C.c_void_p]),
    "mc3d_stream_seeds": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                    C.c_void_p, C.c_void_p, C.c_int32]),
    "mc3d_mwc_draws": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                 C.c_int32]),
    "mc3d_safe_distance": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                     C.c_int32]),
    "mc3d_run_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                   C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "mc3d_run_3dmc_gpu": (C.c_int, [CRefGeometry, CRefOptProps, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    "mc3d_safeprime_table": (C.c_int, [C.c_void_p, C.c_int64, C.c_uint64, C.c_int32]),
    "mc3d_safeprimes_write": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int64]),
    "mc3d_safeprimes_read": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "mc3d_read_geometry_header": (C.c_int, [C.c_char_p] + [C.c_void_p] * 6),
    "mc3d_read_geometry": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int64]),
    "mc3d_read_optprops": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_int32]),
    "mc3d_save_property": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                     C.c_double, C.c_double, C.c_double, C.c_void_p]),
    "mc3d_save_diff_refl": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                      C.c_void_p, C.c_int64]),
}


def lib():
    """Load libmc3d.so (built in-tree by ymc3d_b200.build); raise if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m ymc3d_b200.build`"
                               " (there is no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _check(status: int) -> None:
    if status != MC3D_OK:
        raise Mc3dError(status, lib().mc3d_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------------- inputs
@dataclass
class Geometry:
    """geometry_t (src/mc3d_types.h:38-43): tissue[nz, ny, nx] uint8, 0 = air."""
    tissue: np.ndarray
    dx: float
    dy: float
    dz: float

    def __post_init__(self):
        self.tissue = np.ascontiguousarray(self.tissue, dtype=np.uint8)
        if self.tissue.ndim != 3:
            raise ValueError("tissue must be [nz, ny, nx]")

    @property
    def shape(self):
        nz, ny, nx = self.tissue.shape
        return nx, ny, nz

    def c(self) -> CGeom:
        nx, ny, nz = self.shape
        return CGeom(nx, ny, nz, 0, self.dx, self.dy, self.dz, self.tissue.ctypes.data)


@dataclass
class OpticalProps:
    """opticalprops_t (src/mc3d_types.h:28-36); index 0 is air (0, 0, 0, 1)."""
    mua: np.ndarray
    mus: np.ndarray
    g: np.ndarray
    n: np.ndarray

    def __post_init__(self):
        for k in ("mua", "mus", "g", "n"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.float32))

    @classmethod
    def from_tissues(cls, rows: Sequence[Sequence[float]]) -> "OpticalProps":
        """rows of (mua, mus, g, n) per tissue type 1..T; air is prepended."""
        a = np.array([(0.0, 0.0, 0.0, 1.0)] + [tuple(r) for r in rows], dtype=np.float64)
        return cls(a[:, 0], a[:, 1], a[:, 2], a[:, 3])

    @property
    def num_tissue_types(self) -> int:
        return int(self.mua.shape[0])

    def c(self) -> CProps:
        return CProps(self.num_tissue_types, 0, self.mua.ctypes.data, self.mus.ctypes.data,
                      self.g.ctypes.data, self.n.ctypes.data)


@dataclass
class Job:
    geom: int = 0
    props: int = 0
    photons: int = 1_000_000
    seed: int = 1
    beam: str = "uniform"
    streams: int = 0
    stream_first: int = 0
    stream_count: int = 0

    def c(self) -> CJob:
        return CJob(self.geom, self.props, BEAMS[self.beam], 0, int(self.photons),
                    int(self.streams), int(self.seed), int(self.stream_first),
                    int(self.stream_count))

    def num_streams(self) -> int:
        return self.streams or max(1, min(int(self.photons), DEFAULT_STREAMS))


@dataclass
class Result:
    drs: np.ndarray       # uint64 [ny, nx], sum Q(W) of reflected photons
    drs_sq: np.ndarray    # uint64 [ny, nx], sum Q(W^2)
    trans: np.ndarray     # uint64 [ny, nx]
    totals: dict
    photon_log: np.ndarray | None = None
    absorption: np.ndarray | None = None  # uint64 [nz, ny, nx], sum Q(dW) per voxel

    @property
    def photons(self) -> int:
        return int(self.totals["photons"])

    def reflectance(self) -> np.ndarray:
        """per-bin diffuse reflectance R / N (what outname_drs.bin holds)"""
        return self.drs.astype(np.float64) / WEIGHT_SCALE / max(1, self.photons)

    def reflectance_sigma(self) -> np.ndarray:
        """per-bin standard error of reflectance() from sum W and sum W^2"""
        n = max(1, self.photons)
        m1 = self.drs.astype(np.float64) / WEIGHT_SCALE / n
        m2 = self.drs_sq.astype(np.float64) / WEIGHT_SCALE / n
        return np.sqrt(np.maximum(m2 - m1 * m1, 0.0) / n)

    def conservation_residual(self) -> int:
        t = self.totals
        return int(t["w_launched"]) - (int(t["r_in"]) + int(t["r_out"]) + int(t["t_in"]) +
                                       int(t["t_out"]) + int(t["absorbed"]) +
                                       int(t["rr_killed"]) - int(t["rr_created"]) +
                                       int(t["lost"]))


def _options(device=0, math="fast", block=0, blocks_per_sm=0, max_steps=0, log=None,
             cancel=None, absorption_map=False, use_graph=False, steps="merged") -> COptions:
    o = COptions()
    lib().mc3d_default_options(C.byref(o))
    o.device, o.math, o.block, o.blocks_per_sm, o.max_steps = (
        device, MATH[math], block, blocks_per_sm, max_steps)
    o.steps = STEPS[steps]
    o.absorption_map = int(bool(absorption_map))
    o.use_graph = int(bool(use_graph))
    o.photon_log = _ptr(log)
    o.cancel = _ptr(cancel)
    return o


def _arrays(geoms, props, jobs):
    g = (CGeom * len(geoms))(*[x.c() for x in geoms])
    p = (CProps * len(props))(*[x.c() for x in props])
    j = (CJob * len(jobs))(*[x.c() for x in jobs])
    return g, p, j


def _outs(geoms, jobs, absorption_map=False):
    res, outs = [], (COut * len(jobs))()
    for k, job in enumerate(jobs):
        if not 0 <= job.geom < len(geoms):
            raise Mc3dError(-1, f"job {k}: geometry index {job.geom} out of range")
        nx, ny, nz = geoms[job.geom].shape
        r = Result(np.zeros((ny, nx), np.uint64), np.zeros((ny, nx), np.uint64),
                   np.zeros((ny, nx), np.uint64), {})
        outs[k].drs, outs[k].drs_sq, outs[k].trans = (r.drs.ctypes.data, r.drs_sq.ctypes.data,
                                                      r.trans.ctypes.data)
        if absorption_map:
            r.absorption = np.zeros((nz, ny, nx), np.uint64)
            outs[k].absorption = r.absorption.ctypes.data
        res.append(r)
    return res, outs


def _finish(res, outs, jobs, log):
    base = 0
    for k, r in enumerate(res):
        r.totals = {n: int(getattr(outs[k].totals, n)) for n in TOTAL_FIELDS}
        if log is not None:
            r.photon_log = log[base: base + int(jobs[k].photons)]
        base += int(jobs[k].photons)
    return res


def run(geoms: Sequence[Geometry], props: Sequence[OpticalProps], jobs: Sequence[Job],
        table: np.ndarray | None = None, math: str = "fast", device: int = 0, block: int = 0,
        blocks_per_sm: int = 0, max_steps: int = 0, photon_log: bool = False,
        absorption_map: bool = False, cancel: np.ndarray | None = None,
        steps: str = "merged") -> list[Result]:
    """Run every job in one persistent launch (mc3d_run).  `cancel`, an int32 array
    of one element, is read by the kernel whenever a thread takes a new stream: set
    it non-zero (from another thread) to stop; the call then raises
    MC3D_ERR_CANCELLED and the partial results are in the exception's .results.
    `steps` (fast and FP64 math): "merged" joins the face crossings of a flight
    through uniform tissue into one step, "voxel" steps at every voxel face like
    the reference; exact math always steps per face."""
    table = default_table() if table is None else np.ascontiguousarray(table, dtype=np.uint32)
    g, p, j = _arrays(geoms, props, jobs)
    res, outs = _outs(geoms, jobs, absorption_map)
    log = (np.zeros(sum(int(x.photons) for x in jobs), PHOTON_RECORD_DTYPE)
           if photon_log else None)
    if cancel is not None:
        cancel = np.ascontiguousarray(cancel, np.int32)
    opt = _options(device, math, block, blocks_per_sm, max_steps, log,
                   absorption_map=absorption_map, cancel=cancel, steps=steps)
    st = lib().mc3d_run(g, len(geoms), p, len(props), j, len(jobs), table.ctypes.data,
                        len(table), C.byref(opt), outs)
    if st == -12:
        err = Mc3dError(st, lib().mc3d_last_error().decode(errors="replace"))
        err.results = _finish(res, outs, jobs, log)
        raise err
    _check(st)
    return _finish(res, outs, jobs, log)


class Plan:
    """Inputs resident on the device; execute() any number of times (mc3d_plan_*)."""

    def __init__(self, geoms, props, jobs, table=None, math="fast", device=0, block=0,
                 blocks_per_sm=0, max_steps=0, use_graph=False, steps="merged"):
        self.geoms, self.props, self.jobs = list(geoms), list(props), list(jobs)
        self.table = default_table() if table is None else np.ascontiguousarray(table, np.uint32)
        g, p, j = _arrays(self.geoms, self.props, self.jobs)
        opt = _options(device, math, block, blocks_per_sm, max_steps, use_graph=use_graph,
                       steps=steps)
        self._h = C.c_void_p()
        _check(lib().mc3d_plan_create(C.byref(self._h), g, len(self.geoms), p, len(self.props),
                                      j, len(self.jobs), self.table.ctypes.data, len(self.table),
                                      C.byref(opt)))

    def execute(self, stream: int | None = None) -> None:
        """launch on `stream` (a cudaStream_t handle); None or 0 = the plan's own stream"""
        _check(lib().mc3d_plan_execute(self._h, stream))

    def read(self) -> list[Result]:
        res, outs = _outs(self.geoms, self.jobs)
        _check(lib().mc3d_plan_read(self._h, outs))
        return _finish(res, outs, self.jobs, None)

    def shape(self) -> tuple[int, int, int]:
        b, gr, s = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().mc3d_plan_shape(self._h, C.byref(b), C.byref(gr), C.byref(s)))
        return b.value, gr.value, s.value

    def device_totals_ptr(self) -> int:
        p = C.c_void_p()
        _check(lib().mc3d_plan_device_totals(self._h, C.byref(p)))
        return p.value

    def close(self) -> None:
        if self._h:
            lib().mc3d_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stream_seeds(job: Job, first: int, count: int, table=None, device: int = 0):
    table = default_table() if table is None else np.ascontiguousarray(table, np.uint32)
    x = np.zeros(count, np.uint64)
    a = np.zeros(count, np.uint32)
    cj = job.c()
    _check(lib().mc3d_stream_seeds(C.byref(cj), table.ctypes.data, len(table), first, count,
                                   x.ctypes.data, a.ctypes.data, device))
    return x, a


def mwc_draws(x: np.ndarray, a: np.ndarray, n: int, device: int = 0) -> np.ndarray:
    x = np.ascontiguousarray(x, np.uint64)
    a = np.ascontiguousarray(a, np.uint32)
    out = np.zeros((len(x), n), np.float32)
    _check(lib().mc3d_mwc_draws(x.ctypes.data, a.ctypes.data, len(x), n, out.ctypes.data,
                                device))
    return out


SAFE_CAP = 63


def safe_distance(tissue: np.ndarray, device: int = 0) -> np.ndarray:
    """The safe-distance map of MC3D_STEPS_MERGED for a [nz, ny, nx] uint8 grid,
    [nz + 63, ny, nx]: per voxel the largest r <= 63 whose Chebyshev cube holds
    only the voxel's tissue and stays below the top face and inside the lateral
    faces; the medium continues below the grid with its last slice (computed on
    the GPU)."""
    t = np.ascontiguousarray(tissue, np.uint8)
    nz, ny, nx = t.shape
    out = np.zeros((nz + SAFE_CAP, ny, nx), np.uint8)
    _check(lib().mc3d_safe_distance(t.ctypes.data, nx, ny, nz, out.ctypes.data, device))
    return out


# ----------------------------------------------------------------- safe primes
def safeprime_table(n: int, below: int = 0, threads: int = 0) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    _check(lib().mc3d_safeprime_table(out.ctypes.data, n, below, threads))
    return out


DEFAULT_TABLE_LINES = 1 + (1 << 20)
_TABLE_FILE = HERE / "_data" / f"safeprimes_{DEFAULT_TABLE_LINES}.u32"
_table_cache = None


def default_table() -> np.ndarray:
    """The engine's safe-prime table (generated once, cached next to the library)."""
    global _table_cache
    if _table_cache is None:
        if _TABLE_FILE.exists() and _TABLE_FILE.stat().st_size == 4 * DEFAULT_TABLE_LINES:
            _table_cache = np.fromfile(_TABLE_FILE, np.uint32)
        else:
            t = safeprime_table(DEFAULT_TABLE_LINES)
            _TABLE_FILE.parent.mkdir(exist_ok=True)
            tmp = _TABLE_FILE.with_suffix(f".tmp{os.getpid()}")
            t.tofile(tmp)
            os.replace(tmp, _TABLE_FILE)
            _table_cache = t
    return _table_cache


def write_safeprimes(path: str | os.PathLike, table: np.ndarray) -> None:
    table = np.ascontiguousarray(table, np.uint32)
    _check(lib().mc3d_safeprimes_write(str(path).encode(), table.ctypes.data, len(table)))


def read_safeprimes(path: str | os.PathLike, cap: int = DEFAULT_TABLE_LINES) -> np.ndarray:
    out = np.zeros(cap, np.uint32)
    n = C.c_int64()
    _check(lib().mc3d_safeprimes_read(str(path).encode(), out.ctypes.data, cap, C.byref(n)))
    return out[: n.value].copy()


# ----------------------------------------------------------------- files
def geometry_read_from_file(path: str | os.PathLike) -> Geometry:
    nx, ny, nz = C.c_int32(), C.c_int32(), C.c_int32()
    dx, dy, dz = C.c_double(), C.c_double(), C.c_double()
    bp = str(path).encode()
    _check(lib().mc3d_read_geometry_header(bp, C.byref(nx), C.byref(ny), C.byref(nz),
                                           C.byref(dx), C.byref(dy), C.byref(dz)))
    t = np.zeros((nz.value, ny.value, nx.value), np.uint8)
    _check(lib().mc3d_read_geometry(bp, t.ctypes.data, t.size))
    return Geometry(t, dx.value, dy.value, dz.value)


def opticalprops_read_from_file(path: str | os.PathLike) -> OpticalProps:
    nt = C.c_int32()
    bp = str(path).encode()
    _check(lib().mc3d_read_optprops(bp, C.byref(nt), None, None, None, None, 0))
    arrs = [np.zeros(nt.value, np.float32) for _ in range(4)]
    _check(lib().mc3d_read_optprops(bp, C.byref(nt), *[a.ctypes.data for a in arrs], nt.value))
    return OpticalProps(*arrs)


def save_diff_refl(outname: str, geom: Geometry, R: np.ndarray, num_photons: int) -> None:
    nx, ny, _ = geom.shape
    R = np.ascontiguousarray(R, np.float64)
    _check(lib().mc3d_save_diff_refl(str(outname).encode(), nx, ny, float(np.float32(geom.dx)),
                                     float(np.float32(geom.dy)), R.ctypes.data, num_photons))


def run_3dmc_gpu(geometry: Geometry, optProps: OpticalProps, num_photons: int,
                 R: np.ndarray, T: np.ndarray, seed: int | None = None,
                 table: np.ndarray | None = None, math: str = "fast") -> int:
    """run_3dmc_gpu (src/mc3d_gpu.cu:388): accumulate un-normalised reflected and
    transmitted weight per bin into R and T ([ny, nx] float64), return the
    number of finished photons.  Seed defaults to time(NULL) like the reference."""
    seed = int(time.time()) if seed is None else seed
    res = run([geometry], [optProps], [Job(0, 0, num_photons, seed)], table=table, math=math)[0]
    R += res.drs.astype(np.float64) / WEIGHT_SCALE
    T += res.trans.astype(np.float64) / WEIGHT_SCALE
    return res.photons
