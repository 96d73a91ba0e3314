"""Seeded synthetic workloads and writers for the reference's input formats.

The reference ships no data set; its MATLAB example (matlab/geometry/*.m) builds a
layered skin model with a vessel and writes it with write_geometry_file.m /
write_optical_props_file.m.  The generators below build the five workloads the
engine is measured on, from numpy's PCG64 with fixed seeds:

  layered_vessel   256x256x128 voxels of 0.02 mm: 0.1 mm top layer, 2 mm middle
                   layer, the rest below; a vessel of radius 0.3 mm along x with
                   its axis 0.5 mm deep; uniform beam
  homogeneous      64^3 voxels of 0.1 mm, one tissue, pencil beam
  sweep            the homogeneous geometry under 128 seeded optical tables
  uneven           64 geometries from 64^3 to 320x320x160 with 1-20 ellipsoids
  deep_grid        1024x1024x256 voxels of 0.01 mm, 4 tissue types in blobs
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import Geometry, Job, OpticalProps


# ------------------------------------------------------------------ formats
def write_geometry_file(path: str | os.PathLike, tissue: np.ndarray, dx: float, dy: float,
                        dz: float) -> None:
    """Reference geometry file from engine tissue indices [nz, ny, nx] (0 = air).

    The file holds int32 3, nx, ny, nz, double dx, dy, dz and int32 values x fastest;
    the reader adds 1 and maps 256 to air (src/mc3d_io.cu:107-169), so engine
    index t is stored as t - 1 and air as 255."""
    t = np.asarray(tissue)
    nz, ny, nx = t.shape
    vals = t.astype(np.int32) - 1
    vals[t == 0] = 255
    with open(path, "wb") as f:
        np.array([3, nx, ny, nz], "<i4").tofile(f)
        np.array([dx, dy, dz], "<f8").tofile(f)
        vals.astype("<i4").tofile(f)


def write_optprops_file(path: str | os.PathLike, rows) -> None:
    """Reference optical-property file: int32 T, then T records of double mua,
    mus, g, n (src/mc3d_io.cu:16-66).  `rows` excludes air."""
    rows = np.asarray(rows, "<f8").reshape(-1, 4)
    with open(path, "wb") as f:
        np.array([len(rows)], "<i4").tofile(f)
        rows.tofile(f)


def read_property_file(path: str | os.PathLike):
    """Any save_property file (src/mc3d_io.cu:175-216): outname_drs.bin,
    _trans.bin (2 dims) or _abs.bin / _flu.bin (3 dims).  Returns (data, dx, dy,
    dz) with data [ny, nx] or [nz, ny, nx] (x fastest on disk) -- what
    matlab/read/read_general_mcfile.m returns, in C order; dz is 0 for 2 dims."""
    raw = open(path, "rb").read()
    dims = int(np.frombuffer(raw, "<i4", 1)[0])
    if dims not in (2, 3):
        raise ValueError(f"{path}: {dims} dimensions")
    n = [int(v) for v in np.frombuffer(raw, "<i4", dims, offset=4)]
    off = 4 + 4 * dims
    d = [float(v) for v in np.frombuffer(raw, "<f8", dims, offset=off)]
    off += 8 * dims
    count = int(np.prod(n))
    if len(raw) < off + 8 * count:
        raise ValueError(f"{path}: truncated")
    data = np.frombuffer(raw, "<f8", count, offset=off).reshape(n[::-1]).copy()
    return data, d[0], d[1], (d[2] if dims == 3 else 0.0)


def read_drs_file(path: str | os.PathLike) -> tuple[np.ndarray, float, float]:
    """outname_drs.bin (save_property with 2 dims, src/mc3d_io.cu:175-216)."""
    data, dx, dy, dz = read_property_file(path)
    if data.ndim != 2:
        raise ValueError(f"{path}: not a 2-D file")
    return data, dx, dy


# ------------------------------------------------------------------ skin model
SKIN_EPIDERMIS, SKIN_PAPILLARY, SKIN_RETICULAR, SKIN_SUBCUTIS, SKIN_MOLE, SKIN_VESSEL = 1, 2, 3, 4, 5, 6


def skin_geometry(dx: float = 0.02, length_xy: float = 1.0, length_z: float = 1.7,
                  epi: float = 0.1, dermis: float = 1.5, papillary_frac: float = 0.1,
                  vessel_radius: float = 0.06, vessel_depth: float = 0.25) -> Geometry:
    """The example model of matlab/geometry/prepare_geometry.m:2-55: epidermis,
    papillary and reticular dermis, subcutis, and a blood vessel along y at half
    the width.  The script writes file values 0 (epidermis) .. 5 (vessel, 4 being
    an unused mole); the reader adds one (src/mc3d_io.cu:155-163), so the grid
    holds SKIN_EPIDERMIS .. SKIN_VESSEL = 1 .. 6.  As in the script, voxel n
    (1-based) is tested for the vessel at n * dx."""
    nx = ny = int(round(length_xy / dx))
    nz = int(round(length_z / dx))
    epi_vox = int(np.floor(epi / dx))
    pap_vox = epi_vox + int(np.floor(papillary_frac * dermis / dx))
    ret_vox = pap_vox + int(np.floor((1 - papillary_frac) * dermis / dx))
    k = np.arange(nz)
    layer = np.where(k < epi_vox, SKIN_EPIDERMIS,
                     np.where(k < pap_vox, SKIN_PAPILLARY,
                              np.where(k < ret_vox, SKIN_RETICULAR, SKIN_SUBCUTIS)))
    t = np.broadcast_to(layer.astype(np.uint8)[:, None, None], (nz, ny, nx)).copy()
    xi = (np.arange(nx) + 1) * dx
    zk = (np.arange(nz) + 1) * dx
    vessel = ((xi[None, :] - length_xy / 2) ** 2 + (zk[:, None] - vessel_depth) ** 2
              <= vessel_radius ** 2)
    t[np.broadcast_to(vessel[:, None, :], t.shape)] = SKIN_VESSEL
    return Geometry(t, dx, dx, dx)


def skin_optprops_rows(lam: float, mua_blood) -> list[tuple[float, float, float, float]]:
    """The three (mua, mus, g, n) rows of prepare_optprops.m:29-51 at wavelength
    `lam` (nm), in 1/mm: epidermis, papillary dermis, reticular dermis.
    mua_blood(oxygenation, lam) is the whole-blood absorption in 1/m; the script
    interpolates it from muab.mat, which the reference does not distribute, so the
    caller supplies it."""
    melanin = (lam / 694.0) ** -3.46
    musr = 100 * (18.780 * (lam / 500.0) ** -0.22 + 17.6 * (lam / 500.0) ** -4)
    g = 0.62 + lam * 29e-5
    mus = musr / (1 - g) * 0.01
    return [((227 * melanin + 0.002 * mua_blood(0.5, lam) + (1 - 0.01 - 0.002) * 25) * 0.01,
             mus, g, 1.4),
            ((0.01 * mua_blood(0.5, lam) + (1 - 0.01) * 25) * 0.01, mus, g, 1.4),
            ((0.01 * mua_blood(0.8, lam) + (1 - 0.01) * 25) * 0.01, mus, g, 1.4)]


def skin_optprops(lam: float, mua_blood) -> OpticalProps:
    """An optical set for every tissue of skin_geometry.  Rows 1-3 are the
    script's (skin_optprops_rows).  The script stops there ("a very simple
    example"), though its geometry also holds subcutis, mole and vessel voxels;
    rows 4-6 are this module's stand-ins so that the model runs: subcutis and
    mole as reticular dermis, the vessel as whole blood at oxygenation 0.8
    (mua_blood(0.8) in 1/mm) with the dermis scattering and g 0.98."""
    rows = skin_optprops_rows(lam, mua_blood)
    ret = rows[2]
    rows += [ret, ret, (mua_blood(0.8, lam) * 0.01, ret[1], 0.98, 1.4)]
    return OpticalProps.from_tissues(rows)


# ------------------------------------------------------------------ workloads
@dataclass
class Workload:
    name: str
    geoms: list
    props: list
    jobs: list

    @property
    def photons(self) -> int:
        return sum(int(j.photons) for j in self.jobs)


LAYER_ROWS = [(0.5, 20.0, 0.8, 1.44), (0.05, 15.0, 0.85, 1.37), (0.01, 12.0, 0.9, 1.44),
              (2.0, 20.0, 0.98, 1.4)]


def layered_vessel_geometry(nx=256, ny=256, nz=128, d=0.02, top=0.1, middle=2.0,
                            radius=0.3, depth=0.5) -> Geometry:
    z = (np.arange(nz) + 0.5) * d
    y = (np.arange(ny) + 0.5) * d
    t = np.empty((nz, ny, nx), np.uint8)
    layer = np.where(z < top, 1, np.where(z < top + middle, 2, 3)).astype(np.uint8)
    t[:] = layer[:, None, None]
    yc = ny * d / 2
    vessel = ((y[None, :] - yc) ** 2 + (z[:, None] - depth) ** 2) <= radius ** 2
    t[np.broadcast_to(vessel[:, :, None], t.shape)] = 4
    return Geometry(t, d, d, d)


def layered_vessel(photons: int = 100_000_000, seed: int = 1796308352, scale: int = 1) -> Workload:
    """256x256x128 (optionally /scale per axis) layered tissue with a vessel."""
    g = layered_vessel_geometry(256 // scale, 256 // scale, 128 // scale, 0.02 * scale)
    p = OpticalProps.from_tissues(LAYER_ROWS)
    return Workload("layered_vessel_256x256x128" if scale == 1 else f"layered_vessel_s{scale}",
                    [g], [p], [Job(0, 0, photons, seed, "uniform")])


HOMOGENEOUS_ROW = (0.01, 10.0, 0.9, 1.4)


def homogeneous(photons: int = 1_000_000, seed: int = 1796308352, n: int = 64, d: float = 0.1,
                beam: str = "pencil") -> Workload:
    g = Geometry(np.ones((n, n, n), np.uint8), d, d, d)
    p = OpticalProps.from_tissues([HOMOGENEOUS_ROW])
    return Workload(f"homogeneous_{n}^3", [g], [p], [Job(0, 0, photons, seed, beam)])


def sweep(njobs: int = 128, photons_lo: float = 1e6, photons_hi: float = 1e8,
          rng_seed: int = 2024, seed_base: int = 1796308352, photon_scale: float = 1.0,
          beam: str = "pencil") -> Workload:
    """Hyperspectral sweep: homogeneous 64^3 geometry, one optical table per
    wavelength (mua log-uniform 1e-3..1, reduced mus 0.5..5, g 0.7..0.95, n 1.4)."""
    rng = np.random.Generator(np.random.PCG64(rng_seed))
    g = Geometry(np.ones((64, 64, 64), np.uint8), 0.1, 0.1, 0.1)
    props, jobs = [], []
    for k in range(njobs):
        gg = rng.uniform(0.7, 0.95)
        mua = 10 ** rng.uniform(-3, 0)
        musr = rng.uniform(0.5, 5.0)
        props.append(OpticalProps.from_tissues([(mua, musr / (1 - gg), gg, 1.4)]))
        ph = 10 ** rng.uniform(np.log10(photons_lo), np.log10(photons_hi))
        jobs.append(Job(0, k, max(1, int(ph * photon_scale)), seed_base + 7919 * k, beam))
    return Workload("sweep_128x64^3", [g], props, jobs)


def uneven(ngeoms: int = 64, photons: int = 10_000_000, rng_seed: int = 7, d: float = 0.02,
           seed_base: int = 1796308352, max_dim: int = 320) -> Workload:
    """Geometries from 64^3 to max_dim^2 x max_dim/2 with 1..20 ellipsoids and up to
    8 tissue types (n 1.33..1.50, mua/mus/g in the layered-model ranges)."""
    rng = np.random.Generator(np.random.PCG64(rng_seed))
    geoms, props, jobs = [], [], []
    for k in range(ngeoms):
        nx = int(rng.integers(64, max_dim + 1))
        ny = int(rng.integers(64, max_dim + 1))
        nz = int(rng.integers(64, max(65, max_dim // 2 + 1)))
        ntis = int(rng.integers(2, 9))
        t = np.ones((nz, ny, nx), np.uint8)
        zc = (np.arange(nz) + 0.5) * d
        yc = (np.arange(ny) + 0.5) * d
        xc = (np.arange(nx) + 0.5) * d
        for _ in range(int(rng.integers(1, 21))):
            c = rng.uniform([0, 0, 0], [nx * d, ny * d, nz * d])
            ax = rng.uniform(0.1, 1.0, 3)
            tt = int(rng.integers(2, ntis + 1))
            inside = (((xc[None, None, :] - c[0]) / ax[0]) ** 2 +
                      ((yc[None, :, None] - c[1]) / ax[1]) ** 2 +
                      ((zc[:, None, None] - c[2]) / ax[2]) ** 2) <= 1.0
            t[inside] = tt
        rows = [(10 ** rng.uniform(-2, 0.3), rng.uniform(10, 20), rng.uniform(0.8, 0.98),
                 rng.uniform(1.33, 1.50)) for _ in range(ntis)]
        geoms.append(Geometry(t, d, d, d))
        props.append(OpticalProps.from_tissues(rows))
        jobs.append(Job(k, k, photons, seed_base + 104729 * k, "uniform"))
    return Workload("uneven_64", geoms, props, jobs)


def deep_grid(photons: int = 1_000_000_000, rng_seed: int = 11, nx: int = 1024, ny: int = 1024,
              nz: int = 256, d: float = 0.01, seed: int = 1796308352) -> Workload:
    """1024x1024x256 at 0.01 mm (256 MB of voxels) with 4 tissue types in blobs of
    high-albedo tissue (mua ~0.001/mm, mus ~20/mm, g 0.9, n 1.4)."""
    rng = np.random.Generator(np.random.PCG64(rng_seed))
    coarse = rng.integers(1, 5, size=(max(1, nz // 16), max(1, ny // 16), max(1, nx // 16)),
                          dtype=np.uint8)
    t = np.repeat(np.repeat(np.repeat(coarse, 16, 0), 16, 1), 16, 2)[:nz, :ny, :nx]
    t = np.ascontiguousarray(t)
    rows = [(0.001 * f, 20.0 * f2, 0.9, 1.4) for f, f2 in
            zip(rng.uniform(0.8, 1.2, 4), rng.uniform(0.9, 1.1, 4))]
    return Workload(f"deep_grid_{nx}x{ny}x{nz}", [Geometry(t, d, d, d)],
                    [OpticalProps.from_tissues(rows)], [Job(0, 0, photons, seed, "uniform")])
