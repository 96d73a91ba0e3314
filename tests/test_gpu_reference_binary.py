"""The engine against the reference's own run_3dmc_gpu, compiled from its sources
(oracle/_ref/gpu-mc-ref) and run on the same GPU: per-bin diffuse reflectance
agrees within 3 sigma in the chi-square sense (the reference is uniform-beam only;
its pencil branch is compiled out)."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest
from scipy import stats

import ymc3d_b200 as m
from conftest import ROOT
from helpers import superbin
from ymc3d_b200.workloads import (LAYER_ROWS, layered_vessel_geometry, read_drs_file,
                                  write_geometry_file, write_optprops_file)

pytestmark = pytest.mark.gpu

REF_BIN = ROOT / "oracle" / "_ref" / "gpu-mc-ref"


def run_reference(tmp_path, geom, rows, photons, seed):
    assert REF_BIN.exists(), "oracle/_ref/gpu-mc-ref missing: run oracle/build_ref.py"
    gp, pp = tmp_path / "geom.bin", tmp_path / "props.bid"
    write_geometry_file(gp, geom.tissue, geom.dx, geom.dy, geom.dz)
    write_optprops_file(pp, rows)
    out = tmp_path / "ref"
    subprocess.run([str(REF_BIN), str(gp), str(pp), str(photons), str(seed), str(out),
                    str(REF_BIN.parent)], check=True, capture_output=True, timeout=900)
    raw = (tmp_path / "ref_ref.bin").read_bytes()
    fin = int(np.frombuffer(raw, "<i8", 1)[0])
    nx, ny = np.frombuffer(raw, "<i4", 2, offset=16)
    R = np.frombuffer(raw, "<f8", int(nx * ny), offset=24).reshape(int(ny), int(nx))
    drs, _, _ = read_drs_file(tmp_path / "ref_drs.bin")
    assert np.allclose(drs, R / fin)
    return R, fin


def compare(engine_res, R_ref, n_ref, f):
    """chi-square of superbinned R/N; the reference keeps no sum W^2, so its
    per-bin variance is the engine's scaled to the reference's photon count"""
    s = superbin(engine_res.drs.astype(np.float64), f) / m.WEIGHT_SCALE
    q = superbin(engine_res.drs_sq.astype(np.float64), f) / m.WEIGHT_SCALE
    n = engine_res.photons
    ra, rb = s / n, superbin(R_ref, f) / n_ref
    var_per_photon = np.maximum(q / n - ra ** 2, 0)
    var = var_per_photon / n + var_per_photon / n_ref
    ok = (ra > 1e-6) & (var > 0)
    chi2 = float(np.sum((ra[ok] - rb[ok]) ** 2 / var[ok]))
    dof = int(ok.sum())
    return chi2, dof, float(stats.chi2.sf(chi2, dof))


def test_layered_vessel_vs_reference(tmp_path, table):
    g = layered_vessel_geometry(64, 64, 32, 0.08)
    R, fin = run_reference(tmp_path, g, LAYER_ROWS, 1_000_000, 1796308352)
    assert fin >= 1_000_000
    r = m.run([g], [m.OpticalProps.from_tissues(LAYER_ROWS)],
              [m.Job(0, 0, 4_000_000, 12345, "uniform")], table=table)[0]
    chi2, dof, pv = compare(r, R, fin, 8)
    assert dof >= 32 and pv > 1e-4, (chi2, dof, pv)
    total_ref = R.sum() / fin
    total = r.drs.sum() / m.WEIGHT_SCALE / r.photons
    sigma = np.sqrt(total * (1 - total) * (1 / fin + 1 / r.photons))
    assert abs(total - total_ref) < 4 * sigma, (total, total_ref, sigma)


def test_homogeneous_vs_reference(tmp_path, table):
    g = m.Geometry(np.ones((32, 32, 32), np.uint8), 0.1, 0.1, 0.1)
    rows = [(0.05, 10.0, 0.9, 1.4)]
    R, fin = run_reference(tmp_path, g, rows, 500_000, 20240601)
    r = m.run([g], [m.OpticalProps.from_tissues(rows)],
              [m.Job(0, 0, 2_000_000, 777, "uniform")], table=table)[0]
    chi2, dof, pv = compare(r, R, fin, 4)
    assert dof >= 32 and pv > 1e-4, (chi2, dof, pv)


def test_headline_geometry_vs_reference(tmp_path, table):
    """the benchmark's own geometry (256x256x128 at 0.02 mm, layers and vessel):
    the reference at 4e6 photons against the engine's default fast path"""
    g = layered_vessel_geometry(256, 256, 128, 0.02)
    R, fin = run_reference(tmp_path, g, LAYER_ROWS, 4_000_000, 1796308352)
    r = m.run([g], [m.OpticalProps.from_tissues(LAYER_ROWS)],
              [m.Job(0, 0, 20_000_000, 4242, "uniform")], table=table)[0]
    chi2, dof, pv = compare(r, R, fin, 16)
    assert dof >= 200 and pv > 1e-4, (chi2, dof, pv)
    total_ref = R.sum() / fin
    total = r.drs.sum() / m.WEIGHT_SCALE / r.photons
    sigma = np.sqrt(total * (1 - total) * (1 / fin + 1 / r.photons))
    assert abs(total - total_ref) < 4 * sigma, (total, total_ref, sigma)


def test_long_path_medium_vs_reference(tmp_path, table):
    """A high-albedo medium at 0.01 mm voxels (mua 0.001, mus 20, g 0.9, n 1.4), where
    the reference's end-of-chunk quickfix (src/mc3d_gpu.cu:343-353) removes a few
    1e-3 of the launched weight: total reflectance and per-bin DRS of the engine's
    merged default and of its per-face steps against one reference run of 230,400
    photons (its minimum, one per slot; about 70 s on a B200)."""
    g = m.Geometry(np.ones((64, 512, 512), np.uint8), 0.01, 0.01, 0.01)
    rows = [(0.001, 20.0, 0.9, 1.4)]
    R, fin = run_reference(tmp_path, g, rows, 230_400, 20251204)
    for steps, seed in (("merged", 97), ("voxel", 98)):
        r = m.run([g], [m.OpticalProps.from_tissues(rows)],
                  [m.Job(0, 0, 4_000_000, seed, "uniform")], table=table, steps=steps)[0]
        chi2, dof, pv = compare(r, R, fin, 32)
        assert dof >= 200 and pv > 1e-4, (steps, chi2, dof, pv)
        total_ref = R.sum() / fin
        total = r.drs.sum() / m.WEIGHT_SCALE / r.photons
        # per-photon variance of the reflected weight from the engine's sum W^2
        var = r.drs_sq.sum() / m.WEIGHT_SCALE / r.photons - total ** 2
        sigma = np.sqrt(var * (1 / fin + 1 / r.photons))
        assert abs(total - total_ref) < 4 * sigma, (steps, total, total_ref, sigma)


def test_ellipsoid_inclusions_vs_reference(tmp_path, table):
    """A geometry of the uneven batch (ellipsoid inclusions of up to 8 tissues with
    refractive indices 1.33-1.50): curved interfaces, where the merged boxes
    shrink and Fresnel events happen at every angle."""
    from ymc3d_b200.workloads import uneven
    w = uneven(ngeoms=1, photons=1, max_dim=96, rng_seed=4)
    g, p = w.geoms[0], w.props[0]
    rows = np.stack([p.mua, p.mus, p.g, p.n], 1)[1:]
    R, fin = run_reference(tmp_path, g, rows, 1_000_000, 424243)
    r = m.run([g], [p], [m.Job(0, 0, 4_000_000, 8080, "uniform")], table=table)[0]
    chi2, dof, pv = compare(r, R, fin, 8)
    assert dof >= 32 and pv > 1e-4, (chi2, dof, pv)
    total_ref = R.sum() / fin
    total = r.drs.sum() / m.WEIGHT_SCALE / r.photons
    var = r.drs_sq.sum() / m.WEIGHT_SCALE / r.photons - total ** 2
    sigma = np.sqrt(var * (1 / fin + 1 / r.photons))
    assert abs(total - total_ref) < 4 * sigma, (total, total_ref, sigma)
    assert r.totals["fresnel"] > r.photons  # interfaces are crossed


@pytest.mark.parametrize("which", ["least_absorbing", "most_absorbing"])
def test_sweep_extremes_vs_reference(tmp_path, table, which):
    """The metric's own workload: the hyperspectral sweep's least and most
    absorbing optical sets (mua 0.001 and 0.92 /mm) on its 64^3 geometry at
    0.1 mm, the engine's merged steps against run_3dmc_gpu.  The least absorbing
    set has the longest paths, where the reference runs slowest."""
    from ymc3d_b200.workloads import sweep
    w = sweep(photon_scale=1.0, beam="uniform")
    mua = np.array([float(w.props[j.props].mua[1]) for j in w.jobs])
    k = int(mua.argmin() if which == "least_absorbing" else mua.argmax())
    p = w.props[w.jobs[k].props]
    rows = [(float(p.mua[1]), float(p.mus[1]), float(p.g[1]), float(p.n[1]))]
    g = w.geoms[0]
    R, fin = run_reference(tmp_path, g, rows,
                           200_000 if which == "least_absorbing" else 1_000_000, 90210 + k)
    r = m.run([g], [m.OpticalProps.from_tissues(rows)],
              [m.Job(0, 0, 4_000_000, 31415 + k, "uniform")], table=table)[0]
    chi2, dof, pv = compare(r, R, fin, 4)
    assert dof >= 32 and pv > 1e-4, (chi2, dof, pv)
    total_ref = R.sum() / fin
    total = r.drs.sum() / m.WEIGHT_SCALE / r.photons
    var = r.drs_sq.sum() / m.WEIGHT_SCALE / r.photons - total ** 2
    sigma = np.sqrt(var * (1 / fin + 1 / r.photons))
    assert abs(total - total_ref) < 4 * sigma, (total, total_ref, sigma)
