"""Writes tests/golden/step_fp64.json: one FP64 step of 64 electrons (synthetic gas 0,
equal-sharing ionization, energy grid of 20001 points, E = 1.25e7 V/m) run through the
oracle, plus the Philox KAT vectors.  Run from the repository root:
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


if __name__ == "__main__":
    main()
