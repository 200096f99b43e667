"""load_lxcat (JuMC/src/lxcat.jl:17-134) against an independent loop restatement."""
import json

import numpy as np
import pytest

from mcstreamer_b200 import constants as co
from mcstreamer_b200 import lxcat
from oracle import lxcat_ref


def test_load_lxcat_matches_loop_restatement():
    recs = lxcat.synthetic_records(0, uniform_sharing=False)
    e = lxcat.EnergyGrid(0.0, 200 * co.eV, 301)
    t = lxcat.load_lxcat_records(recs, {"SYN": 2.5e25}, e)
    kinds, rows, maxrate = lxcat_ref.load_lxcat(recs, {"SYN": 2.5e25}, 0.0, 200 * co.eV, 301)
    assert [lxcat.KIND_NAMES[p.kind] for p in t.proc] == kinds
    np.testing.assert_allclose(t.rate, np.array(rows), rtol=1e-13, atol=1e-3)
    assert t.maxrate == pytest.approx(maxrate, rel=1e-14)


def test_synthetic_gas_maxrate_and_order():
    t = lxcat.synthetic_table(0)
    # nu_max = N v(1000 eV) (sigma_el + sigma_ion + 3 sigma_exc) at the top of the grid
    v = np.sqrt(2 * 1000 * co.eV / co.electron_mass)
    expect = 2.5e25 * v * (6e-20 + 2.5e-20 + 3e-21)
    assert t.maxrate == pytest.approx(expect, rel=1e-6)
    assert t.maxrate == pytest.approx(4.126e13, rel=1e-3)
    names = [lxcat.KIND_NAMES[p.kind] for p in t.proc]
    assert names[0] == "ELASTIC" and "NULL" in names
    integ = t.rate.sum(axis=1)
    assert np.all(np.diff(integ) <= 0)
    # the rows (null included) sum to maxrate at every energy
    np.testing.assert_allclose(t.rate.sum(axis=0), t.maxrate, rtol=1e-12)
    # origperm inverts the sort
    assert np.array_equal(t.perm[t.origperm], np.arange(len(t.proc)))


def test_effective_becomes_elastic(tmp_path):
    recs = [
        {"kind": "EFFECTIVE", "target": "A", "mass_ratio": 1e-4, "comment": "",
         "data": [[0.0, 1e-19], [100.0, 1e-19]]},
        {"kind": "EXCITATION", "target": "A", "threshold": 5.0, "comment": "",
         "data": [[5.0, 0.0], [100.0, 2e-20]]},
    ]
    p = tmp_path / "a.json"
    p.write_text(json.dumps(recs))
    e = lxcat.EnergyGrid(0.0, 50 * co.eV, 51)
    t = lxcat.load_lxcat([p], {"A": 1e25}, e)
    el = [i for i, q in enumerate(t.proc) if q.kind == lxcat.ELASTIC][0]
    ex = [i for i, q in enumerate(t.proc) if q.kind == lxcat.EXCITATION][0]
    v = np.sqrt(2 * e.values() / co.electron_mass)
    np.testing.assert_allclose(t.rate[el] + t.rate[ex], 1e25 * v * 1e-19, rtol=1e-12)
    assert t.proc[ex].param == pytest.approx(5.0 * co.eV)


def test_photoemission_records_need_their_absorber():
    """PhotoEmission takes nu_min, nu_max = c * dens[absorber] * chi (lxcat.jl:86-93): a record
    without an absorber, or with one of no density, fails as the reference's lookup does."""
    rec = {"kind": "PHOTOEMISSION", "target": "A", "comment": "", "data": [[0, 1e-20], [10, 1e-20]],
           "chi_min": 1e-23, "chi_max": 1e-21}
    grid = lxcat.EnergyGrid(0.0, 1e-18, 11)
    with pytest.raises(KeyError):
        lxcat.load_lxcat_records([rec], {"A": 1.0}, grid)
    with pytest.raises(KeyError):
        lxcat.load_lxcat_records([dict(rec, absorber="B")], {"A": 1.0}, grid)
    t = lxcat.load_lxcat_records([dict(rec, absorber="A")], {"A": 2.0}, grid, photon_multiplier=10.0)
    assert t.has_photoemission and t.photon_multiplier == 10.0


def test_flat_linear_interpolation_matches_numpy_interp():
    """Interpolations.jl Gridded(Linear()) with Flat() extrapolation (lxcat.jl:63-64) is
    piecewise-linear between knots and constant beyond the ends: the semantics of
    numpy.interp, used here as an independent implementation."""
    import numpy as np

    from mcstreamer_b200.lxcat import _interp_flat
    rng = np.random.default_rng(5)
    x0 = np.sort(rng.uniform(0.0, 100.0, 300))
    y0 = rng.normal(size=300)
    x = np.concatenate([rng.uniform(-20.0, 120.0, 5000), x0, [x0[0], x0[-1], -1e9, 1e9]])
    np.testing.assert_allclose(_interp_flat(x0, y0, x), np.interp(x, x0, y0), rtol=1e-13, atol=1e-13)
