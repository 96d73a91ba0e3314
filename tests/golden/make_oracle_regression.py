"""Regenerate oracle_regression.json: tallies of the FP32 oracle on three small
seeded workloads.  The file pins the oracle against accidental change when its
source is refactored (the GPU exact-math kernel is pinned to the oracle bit for
bit, so any drift here would surface there too).

    python tests/golden/make_oracle_regression.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
import ymc3d_b200 as m  # noqa: E402
from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry  # noqa: E402

TABLE_LINES = 4097


def cases():
    g1 = m.Geometry(np.ones((20, 20, 20), np.uint8), 0.1, 0.1, 0.1)
    p1 = m.OpticalProps.from_tissues([(0.05, 10.0, 0.9, 1.4)])
    g2 = layered_vessel_geometry(40, 36, 24, 0.1)
    g2.tissue[12:14, 5:9, 5:9] = 0
    p2 = m.OpticalProps.from_tissues(LAYER_ROWS)
    g3 = m.Geometry(np.ones((12, 12, 12), np.uint8), 0.1, 0.1, 0.1)
    p3 = m.OpticalProps.from_tissues([(0.1, 5.0, 0.0, 1.4)])
    return [("homogeneous_pencil", g1, p1, m.Job(0, 0, 1500, 1796308352, "pencil", 300)),
            ("layered_air_uniform", g2, p2, m.Job(0, 0, 1500, 424242, "uniform")),
            ("g_zero_quickfix", g3, p3, m.Job(0, 0, 300, 777, "uniform"))]


def run_case(g, p, job, table):
    o = oracle.run(g.tissue, g.dx, g.dy, g.dz, p.mua, p.mus, p.g, p.n, job.photons,
                   job.num_streams(), job.seed, table, beam=m.BEAMS[job.beam], threads=4,
                   photon_log=True)
    digest = hashlib.sha256(o["drs"].tobytes() + o["drs_sq"].tobytes() + o["trans"].tobytes()
                            + o["photon_log"].tobytes()).hexdigest()
    return {"totals": o["totals"], "sha256": digest}


def main():
    table = m.safeprime_table(TABLE_LINES)
    out = {name: run_case(g, p, job, table) for name, g, p, job in cases()}
    (Path(__file__).parent / "oracle_regression.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
