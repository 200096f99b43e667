"""Writes the golden fixtures of tests/golden/, all produced by the oracle (the CPU FP64
restatement of the reference) on small seeded inputs:

  step_fp64.json      one FP64 step of 64 electrons (synthetic gas 0, equal-sharing
                      ionization, energy grid of 20001 points, E = 1.25e7 V/m), plus the
                      Philox KAT vectors;
  swarm_resample.json Swarm.resample! of 600 electrons to n0 = 1040 (clones), then to
                      n0 = 360 (roulette), then repack!;
  resample_cells.json the cell sort and resample!(ntarget = 10, nmax = 15) of 1200
                      electrons on an 8 x 8 x 16 mesh (h = 4 um);
  deposit_cic.json    density! of 700 electrons as int64 CIC (2^-32 e) on an 8 x 8 x 8 mesh.

Run from the repository root:
    python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from mcstreamer_b200 import constants as co  # noqa: E402
from mcstreamer_b200 import lxcat  # noqa: E402
from oracle import pyoracle as po  # noqa: E402
from tests.helpers import broad, oracle_arrays, oracle_pop  # noqa: E402
from tests.test_oracle import KAT  # noqa: E402


def main():
    neps, seed, ez, dt = 20001, 17, 1.25e7, 5e-13
    t = lxcat.load_lxcat_records(lxcat.synthetic_records(0, uniform_sharing=False), {"SYN": 2.5e25},
                                 lxcat.EnergyGrid(0.0, 1000 * co.eV, neps))
    tab = po.OracleTable.from_lxcat(t)
    p = broad(64, seed)
    op = oracle_pop(p, 256, seed)
    assert po.advance(op, tab, po.field_uniform(0, 0, ez), dt, threads=1) == 0
    o = oracle_arrays(op)
    doc = {
        "neps": neps, "seed": seed, "ez": ez, "dt": dt,
        "input": {"x": p.x.tolist(), "v": p.v.tolist(), "w": p.w.tolist(), "s": p.s.tolist(),
                  "active": p.active.tolist()},
        "output": {"x": o.x.tolist(), "v": o.v.tolist(), "w": o.w.tolist(), "s": o.s.tolist(),
                   "active": o.active.tolist()},
        "philox_kat": [[c, k, out] for c, k, out in KAT],
    }
    (ROOT / "tests" / "golden" / "step_fp64.json").write_text(json.dumps(doc))
    print("wrote step_fp64.json with", o.n, "particles")
    write_swarm_resample()
    write_resample_cells()
    write_deposit()


def _arrays(p):
    return {"x": p.x.tolist(), "v": p.v.tolist(), "w": p.w.tolist(), "s": p.s.tolist(),
            "active": p.active.tolist()}


def write_swarm_resample():
    from tests.helpers import maxwellian
    p = maxwellian(600, 31, mean_ev=3.0)
    op = oracle_pop(p, 2400, 31, step=4)
    assert po.swarm_resample(op, 1040, 0.1) == 0
    after_clone = oracle_arrays(op)
    assert po.swarm_resample(op, 360, 0.1) == 0
    after_drop = oracle_arrays(op)
    assert po.repack(op) == 0
    doc = {"seed": 31, "step": 4, "cap": 2400, "n0": [1040, 360], "input": _arrays(p), "after_clone": _arrays(after_clone),
           "after_drop": _arrays(after_drop), "after_repack": _arrays(oracle_arrays(op))}
    (ROOT / "tests" / "golden" / "swarm_resample.json").write_text(json.dumps(doc))
    print("wrote swarm_resample.json")


RS_MESH = (8, 8, 16, 4e-6)


def resample_cloud():
    nx, ny, nz, h = RS_MESH
    p = broad(1200, 41, emax_ev=10.0, x0=(nx * h / 2, ny * h / 2, nz * h / 2), spread=4e-6)
    rng = np.random.default_rng(42)
    p.w[:] = np.rint(10 ** rng.uniform(0, 3, p.n))
    p.active[rng.random(p.n) < 0.05] = 0
    return p


def write_resample_cells():
    nx, ny, nz, h = RS_MESH
    p = resample_cloud()
    op = oracle_pop(p, 4800, 41)
    f = po.field_cart3d(nx, ny, nz, h, (0.0, 0.0, 0.0), np.zeros(3 * (nx + 1) * (ny + 1) * (nz + 1)))
    assert po.sort_cells(op, f) == 0
    assert po.resample_cells(op, f, 10, 15, 0) == 0
    doc = {"seed": 41, "cap": 4800, "mesh": list(RS_MESH), "ntarget": 10, "nmax": 15, "input": _arrays(p),
           "output": _arrays(oracle_arrays(op))}
    (ROOT / "tests" / "golden" / "resample_cells.json").write_text(json.dumps(doc))
    print("wrote resample_cells.json with", op.n, "particles")


DEP_MESH = (8, 8, 8, 4e-6)


def write_deposit():
    nx, ny, nz, h = DEP_MESH
    rng = np.random.default_rng(51)
    x = (nx * h / 2) + rng.normal(0.0, 6e-6, (700, 3))
    w = np.rint(10 ** rng.uniform(0, 3, 700))
    from mcstreamer_b200.jumc import ParticleArrays
    p = ParticleArrays(x, np.zeros((700, 3)), w, np.ones(700), np.ones(700, np.uint8))
    trk = po.tracker_cart3d(nx, ny, nz, h, (0.0, 0.0, 0.0))
    po.deposit(oracle_pop(p, 700, 0), trk, -1.0)
    q = trk._q.copy()
    nz_idx = np.nonzero(q)[0]
    doc = {"mesh": list(DEP_MESH), "val": -1.0, "x": x.tolist(), "w": w.tolist(),
           "nodes": nz_idx.tolist(), "q": q[nz_idx].tolist(), "n_nodes": int(q.size)}
    (ROOT / "tests" / "golden" / "deposit_cic.json").write_text(json.dumps(doc))
    print("wrote deposit_cic.json with", len(nz_idx), "charged nodes")


if __name__ == "__main__":
    main()
