"""The seeded workload generators and the reference-format writers."""
from __future__ import annotations

import numpy as np

from ymc3d_b200 import workloads as W


def test_layered_vessel_geometry():
    g = W.layered_vessel_geometry()
    nx, ny, nz = g.shape
    assert (nx, ny, nz) == (256, 256, 128) and g.dx == 0.02
    col = g.tissue[:, 0, 0]
    assert np.all(col[:5] == 1) and np.all(col[5:105] == 2) and np.all(col[105:] == 3)
    zc, yc = (np.arange(nz) + 0.5) * 0.02, (np.arange(ny) + 0.5) * 0.02
    in_vessel = ((yc[None, :] - 2.56) ** 2 + (zc[:, None] - 0.5) ** 2) <= 0.09
    assert np.array_equal(g.tissue[:, :, 7] == 4, in_vessel)
    assert np.all(g.tissue[:, :, 0] == g.tissue[:, :, -1])  # a cylinder along x


def test_sweep_and_uneven_ranges():
    s = W.sweep()
    assert len(s.jobs) == 128 and len(s.props) == 128
    ph = np.array([j.photons for j in s.jobs])
    assert ph.min() >= 1e6 and ph.max() <= 1e8
    for p in s.props:
        g = p.g[1]
        assert 0.7 <= g <= 0.95 and 1e-3 <= p.mua[1] <= 1 and p.n[1] == np.float32(1.4)
        assert 0.5 <= p.mus[1] * (1 - g) <= 5.0001
    u = W.uneven(ngeoms=6, max_dim=96)
    for g, p in zip(u.geoms, u.props):
        assert g.tissue.max() < p.num_tissue_types <= 9


def test_writers_round_trip(engine, tmp_path):
    g = W.layered_vessel_geometry(40, 30, 20, 0.05)
    g.tissue[3, 4, 5] = 0
    W.write_geometry_file(tmp_path / "g.bin", g.tissue, g.dx, g.dy, g.dz)
    back = engine.geometry_read_from_file(tmp_path / "g.bin")
    assert np.array_equal(back.tissue, g.tissue) and back.dx == g.dx
    W.write_optprops_file(tmp_path / "p.bid", W.LAYER_ROWS)
    p = engine.opticalprops_read_from_file(tmp_path / "p.bid")
    assert np.allclose(p.mua[1:], [r[0] for r in W.LAYER_ROWS])
    assert p.n[0] == 1.0 and p.mua[0] == 0


def test_read_property_file_2d_and_3d(engine, tmp_path):
    rng = np.random.default_rng(9)
    a2 = rng.uniform(size=(5, 7))
    engine.lib().mc3d_save_property(str(tmp_path / "a.bin").encode(), 2, 7, 5, 1, 0.1, 0.2, 0.0,
                                    a2.ctypes.data)
    d, dx, dy, dz = W.read_property_file(tmp_path / "a.bin")
    assert np.array_equal(d, a2) and (dx, dy, dz) == (0.1, 0.2, 0.0)
    a3 = np.ascontiguousarray(rng.uniform(size=(3, 5, 7)))
    engine.lib().mc3d_save_property(str(tmp_path / "b.bin").encode(), 3, 7, 5, 3, 0.1, 0.2, 0.3,
                                    a3.ctypes.data)
    d, dx, dy, dz = W.read_property_file(tmp_path / "b.bin")
    assert np.array_equal(d, a3) and dz == 0.3
    (tmp_path / "c.bin").write_bytes((tmp_path / "b.bin").read_bytes()[:-9])
    import pytest
    with pytest.raises(ValueError):
        W.read_property_file(tmp_path / "c.bin")


def test_skin_model_matches_the_matlab_recipe():
    g = W.skin_geometry()
    nx, ny, nz = g.shape
    assert (nx, ny, nz) == (50, 50, 85)
    col = g.tissue[:, 0, 0]
    # epidermis 0.1 mm = 5 voxels, papillary 10 % of 1.5 mm = 7, reticular 67
    assert np.all(col[:5] == W.SKIN_EPIDERMIS) and np.all(col[5:12] == W.SKIN_PAPILLARY)
    assert np.all(col[12:79] == W.SKIN_RETICULAR) and np.all(col[79:] == W.SKIN_SUBCUTIS)
    vessel = g.tissue == W.SKIN_VESSEL
    assert vessel.sum() > 0 and np.all(g.tissue[:, 0, :] == g.tissue[:, -1, :])
    # voxel (i, k) 1-based is in the vessel when (i dx - 0.5)^2 + (k dx - 0.25)^2 <= 0.06^2
    k, i = np.nonzero(vessel[:, 0, :])
    assert np.all(((i + 1) * 0.02 - 0.5) ** 2 + ((k + 1) * 0.02 - 0.25) ** 2 <= 0.06 ** 2 + 1e-12)
    blood = lambda oxy, lam: 1e4 * (1 + oxy)  # noqa: E731
    rows = W.skin_optprops_rows(600.0, blood)
    assert len(rows) == 3
    mel = (600 / 694) ** -3.46
    assert abs(rows[0][0] - (227 * mel + 0.002 * 1.5e4 + 0.988 * 25) * 0.01) < 1e-9
    assert abs(rows[1][0] - (0.01 * 1.5e4 + 0.99 * 25) * 0.01) < 1e-9
    assert abs(rows[2][0] - (0.01 * 1.8e4 + 0.99 * 25) * 0.01) < 1e-9
    p = W.skin_optprops(600.0, blood)
    assert p.num_tissue_types == 7  # air + six tissues, the grid's largest index is 6
    assert abs(p.g[1] - (0.62 + 600 * 29e-5)) < 1e-6
    assert p.mua[6] > p.mua[3] > 0 and np.all(p.n[1:] == np.float32(1.4))
