"""The gpu-mc command: the reference's argument handling, messages and output files
(src/mc3d_main.cu:15-98)."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT
from ymc3d_b200.workloads import read_drs_file, write_geometry_file, write_optprops_file

CLI = ROOT / "ymc3d_b200" / "gpu-mc"


def run(args, cwd):
    return subprocess.run([str(CLI)] + [str(a) for a in args], cwd=cwd, capture_output=True,
                          text=True, timeout=600)


def inputs(tmp_path, n=16, rows=((0.1, 10.0, 0.9, 1.4),)):
    write_geometry_file(tmp_path / "geom.bin", np.ones((n, n, n), np.uint8), 0.1, 0.1, 0.1)
    write_optprops_file(tmp_path / "props.bid", rows)
    return tmp_path / "geom.bin", tmp_path / "props.bid"


def test_usage(engine, tmp_path):
    r = run(["a", "b"], tmp_path)
    assert r.returncode == 1 and "Usage:" in r.stderr


def test_missing_inputs(engine, tmp_path):
    g, p = inputs(tmp_path)
    r = run([tmp_path / "nope.bin", p, "dummy", "out"], tmp_path)
    assert r.returncode == 1 and "was not opened" in r.stderr


def test_missing_table_exits_like_reference(engine, tmp_path):
    g, p = inputs(tmp_path)
    r = run([g, p, "dummy", "out"], tmp_path)
    assert r.returncode == 1 and "Couldn't find safeprimes_base32.txt." in r.stderr
    assert "#mua (mm-1), mus (mm-1), g, n." in r.stdout  # printed before the run


@pytest.mark.gpu
def test_cli_run_matches_library(engine, tmp_path, table):
    g, p = inputs(tmp_path)
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", table[:230401])
    (tmp_path / "params.txt").write_text("photons = 20000\nseed = 4242\nbeam = pencil\n")
    r = run([g, p, "params.txt", "out"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "seed: 4242" in r.stderr and "Total diffuse reflectance is" in r.stderr
    assert (tmp_path / "out_simparam.dat").read_text() == "20000 #num_photons\n"
    drs, dx, dy = read_drs_file(tmp_path / "out_drs.bin")
    res = engine.run([engine.geometry_read_from_file(g)], [engine.opticalprops_read_from_file(p)],
                     [engine.Job(0, 0, 20000, 4242, "pencil")], table=table[:230401])[0]
    assert np.array_equal(drs, res.drs.astype(np.float64) / engine.WEIGHT_SCALE / 20000)


@pytest.mark.gpu
def test_reference_command_line_on_the_library(engine, tmp_path, table):
    """The drop-in as a maintainer builds it: the reference's own main and file I/O
    (src/mc3d_main.cu, src/mc3d_io.cu) linked with the bridge that forwards
    run_3dmc_gpu to libmc3d.so.  Its 30,000,000 photons (src/mc3d_main.cu:57) under
    MC3D_SEED write _drs.bin and _simparam.dat byte for byte as gpu-mc does for the
    same inputs, photons and seed."""
    bridge = ROOT / "oracle" / "_ref" / "gpu-mc-bridge"
    if not bridge.exists():
        pytest.skip("the bridge is built only where the reference's sources were present")
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    g = layered_vessel_geometry(40, 36, 20, 0.1)
    write_geometry_file(tmp_path / "geom.bin", g.tissue, g.dx, g.dy, g.dz)
    write_optprops_file(tmp_path / "props.bid", LAYER_ROWS)
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", table[:230401])
    seed = 271828182
    import os
    ref = subprocess.run([str(bridge), "geom.bin", "props.bid", "dummy", "ref"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, MC3D_SEED=str(seed)))
    assert ref.returncode == 0, ref.stderr
    assert "Total diffuse reflectance is" in ref.stderr
    (tmp_path / "p.txt").write_text(f"photons = 30000000\nseed = {seed}\n")
    ours = run(["geom.bin", "props.bid", "p.txt", "ours"], tmp_path)
    assert ours.returncode == 0, ours.stderr
    for suffix in ("_drs.bin", "_simparam.dat"):
        assert (tmp_path / ("ref" + suffix)).read_bytes() == (tmp_path / ("ours" + suffix)).read_bytes()
    assert (tmp_path / "ref_simparam.dat").read_text() == "30000000 #num_photons\n"


@pytest.mark.gpu
def test_cli_absorption_and_transmission_maps(engine, tmp_path, table):
    write_geometry_file(tmp_path / "geom.bin", np.ones((12, 16, 20), np.uint8), 0.1, 0.1, 0.1)
    write_optprops_file(tmp_path / "props.bid", [(0.3, 10.0, 0.9, 1.4)])
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", table[:230401])
    (tmp_path / "p.txt").write_text("photons=5000\nseed=99\nabs_map=1\nsave_trans=1\n")
    r = run(["geom.bin", "props.bid", "p.txt", "out"], tmp_path)
    assert r.returncode == 0, r.stderr
    raw = (tmp_path / "out_abs.bin").read_bytes()
    dims, nx, ny, nz = np.frombuffer(raw, "<i4", 4)
    assert (dims, nx, ny, nz) == (3, 20, 16, 12)
    A = np.frombuffer(raw, "<f8", offset=16 + 24)
    F = np.frombuffer((tmp_path / "out_flu.bin").read_bytes(), "<f8", offset=40)
    assert A.size == 20 * 16 * 12 and np.allclose(F, A / np.float32(0.3))
    import json
    rep = json.loads((tmp_path / "out_report.json").read_text())
    assert abs(A.sum() - rep["absorbed"] / 2 ** 32 / 5000) < 1e-9
    assert (tmp_path / "out_trans.bin").exists()


@pytest.mark.gpu
@pytest.mark.parametrize("math,steps", [("exact", "merged"), ("fast", "voxel"), ("f64", "merged")])
def test_cli_math_and_step_modes(engine, tmp_path, table, math, steps):
    """math= and steps= reach the engine: the CLI's tallies equal the library's"""
    g, p = inputs(tmp_path)
    engine.write_safeprimes(tmp_path / "safeprimes_base32.txt", table[:230401])
    (tmp_path / "params.txt").write_text(f"photons=5000\nseed=77\nmath={math}\nsteps={steps}\n")
    r = run([g, p, "params.txt", "out"], tmp_path)
    assert r.returncode == 0, r.stderr
    drs, _, _ = read_drs_file(tmp_path / "out_drs.bin")
    res = engine.run([engine.geometry_read_from_file(g)], [engine.opticalprops_read_from_file(p)],
                     [engine.Job(0, 0, 5000, 77, "uniform")], table=table[:230401], math=math,
                     steps=steps)[0]
    assert np.array_equal(drs, res.drs.astype(np.float64) / engine.WEIGHT_SCALE / 5000)
