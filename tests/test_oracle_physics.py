"""The oracle's restated helpers against the reference formulas, and properties of
whole runs (exact conservation, thread-count independence)."""
from __future__ import annotations

import math

import numpy as np

import ymc3d_b200 as m
from helpers import oracle_job, residual


def grid_coord_py(x, ux, d):
    """src/mc3d_gpu.cu:53-63 in numpy float32"""
    x, d = np.float32(x), np.float32(d)
    i = int(np.floor(np.float32(x / d)))
    i += int(x == np.float32(np.float32(i + 1) * d))
    bmin = np.float32(np.float32(i) * d)
    return i if (x > bmin or (x == bmin and ux >= 0)) else i - 1


def test_grid_coord_faces(orc):
    L = orc.lib()
    d = np.float32(0.1)
    for k in range(-3, 70):
        face = np.float32(np.float32(k) * d)
        for ux in (1.0, 0.0, -1.0):
            got = L.orc_grid_coord_x(float(face), ux, float(d))
            assert got == grid_coord_py(face, ux, d)
        # a face is owned by the cell the direction points into
        assert L.orc_grid_coord_x(float(face), 1.0, float(d)) == \
            L.orc_grid_coord_x(float(face), -1.0, float(d)) + 1
    rng = np.random.default_rng(0)
    for x in np.float32(rng.uniform(-1, 7, 3000)):
        assert L.orc_grid_coord_x(float(x), 0.5, float(d)) == grid_coord_py(x, 0.5, d)


def fresnel_reference(ni, nt, cos_ai):
    """src/mc3d_gpu.cu:227-245 (with the sin_at*sin_at denominator)"""
    ai = math.acos(min(abs(cos_ai), 1.0))
    sin_ai = math.sin(ai)
    sin_at = ni / nt * sin_ai
    if sin_at > 1:
        return 1.0
    cos_at = math.sqrt(1 - sin_at * sin_at)
    den1 = sin_ai * cos_at + cos_ai * sin_at
    if den1 == 0:
        return float("nan")  # normal incidence: 0/0, epsilon < NaN is false -> transmit
    R1 = (sin_ai * cos_at - cos_ai * sin_at) / den1
    R2 = (cos_ai * cos_at - sin_ai * sin_at) / (cos_ai * cos_at + sin_at * sin_at)
    return 0.5 * R1 * R1 * (1 + R2 * R2)


def test_fresnel_quirks():
    assert math.isnan(fresnel_reference(1.4, 1.0, 1.0))          # always transmits
    assert fresnel_reference(1.4, 1.0, math.cos(math.radians(60))) == 1.0  # total reflection
    r = fresnel_reference(1.0, 1.4, math.cos(math.radians(30)))
    assert 0 < r < 0.1


def test_conservation_and_threads(orc, table):
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    g = layered_vessel_geometry(32, 32, 24, 0.1)
    g.tissue[10:12, 5:9, 5:9] = 0
    p = m.OpticalProps.from_tissues(LAYER_ROWS)
    job = m.Job(0, 0, 3000, 8642, "uniform", 301)
    a = oracle_job(g, p, job, table, threads=1)
    b = oracle_job(g, p, job, table, threads=8)
    assert a["totals"] == b["totals"] and np.array_equal(a["drs"], b["drs"])
    t = a["totals"]
    assert residual(t) == 0
    assert int(a["drs"].sum()) == t["r_in"] and int(a["trans"].sum()) == t["t_in"]
    assert t["photons"] == 3000 and t["fresnel"] > 0


def test_stream_subsets_add_up(orc, table):
    g = m.Geometry(np.ones((16, 16, 16), np.uint8), 0.1, 0.1, 0.1)
    p = m.OpticalProps.from_tissues([(0.2, 8.0, 0.85, 1.33)])
    job = m.Job(0, 0, 2000, 1357, "pencil", 150)
    whole = oracle_job(g, p, job, table)
    parts = [oracle_job(g, p, job, table, first=f, count=c)
             for f, c in ((0, 40), (40, 77), (117, 33))]
    for k in ("drs", "drs_sq", "trans"):
        assert np.array_equal(sum(q[k] for q in parts), whole[k])
    for k in whole["totals"]:
        assert sum(q["totals"][k] for q in parts) == whole["totals"][k]


def test_oracle_regression_fixture(orc):
    """the FP32 oracle still produces the pinned tallies and photon logs"""
    import json
    from pathlib import Path

    import sys
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    import make_oracle_regression as mk
    want = json.loads((Path(__file__).parent / "golden" / "oracle_regression.json").read_text())
    table = m.safeprime_table(mk.TABLE_LINES)
    for name, g, p, job in mk.cases():
        assert mk.run_case(g, p, job, table) == want[name], name
