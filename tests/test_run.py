"""The TOML front end's host parts (MCStreamer/src/main.jl): geteb's units and sampseg's
seed distribution, without a GPU."""
import math

import numpy as np
import pytest

from mcstreamer_b200 import constants as co
from mcstreamer_b200.run import geteb, sampseg


def test_geteb_units():
    """geteb (main.jl:349-360): -eb times the unit's scale; Td scales with nair."""
    assert geteb({"eb": 15.0, "field_units": "kV/cm"}) == -1.5e6
    assert geteb({"eb": 2.0, "field_units": "MV/m"}) == -2e6
    assert geteb({"eb": 7.0, "field_units": "V/m"}) == -7.0
    assert geteb({"eb": 100.0}) == -100.0 * (co.Td * co.nair)
    assert geteb({"eb": 100.0, "nair": 2.5e25}) == -100.0 * (co.Td * 2.5e25)
    with pytest.raises(KeyError):
        geteb({"eb": 1.0, "field_units": "furlong"})


def test_sampseg_distribution():
    """sampseg(z0, z1, w) (main.jl:320-341): with probability l / (l + sqrt(2 pi) w) a point
    of the segment blurred in x, y; else a 3-D Gaussian around the nearer end."""
    z0, z1, w, n = 1e-3, 1.4e-3, 5e-5, 40_000
    x = sampseg(z0, z1, w, n, np.random.default_rng(1))
    p = (z1 - z0) / (z1 - z0 + math.sqrt(2 * math.pi) * w)
    inside = (x[:, 2] >= z0) & (x[:, 2] <= z1)
    # points on the segment, plus the end caps' half-Gaussians that fall back onto it: none
    # (the cap draws put z beyond the end they belong to)
    assert abs(inside.mean() - p) < 5 * math.sqrt(p * (1 - p) / n)
    assert abs(x[:, 0].std() - w) < 0.02 * w and abs(x[:, 1].std() - w) < 0.02 * w
    below = x[:, 2] < z0
    assert abs(below.mean() - (1 - p) / 2) < 5 * math.sqrt(0.25 / n)
    with pytest.raises(ValueError):
        sampseg(1.0, 0.5, w, 1, np.random.default_rng(0))


def test_read_input_resolves_like_main(tmp_path):
    """Paths relative to the input's folder, fld(tmax, dt) steps, the default Poisson levels
    and nair, the init-file settings with their defaults, the output path."""
    from mcstreamer_b200.run import read_input

    d = tmp_path / "case"
    d.mkdir()
    (d / "input.toml").write_text("""
eb = 100.0
dt = 1e-12
tmax = 1.05e-10
rng_seed = 7
cross_sections = ["../cs/a.json", "b.json"]
[init_files]
ne_file = "afivo/ne.hdf"
q_file = "afivo/q.hdf"
format = "afivo"
""")
    c = read_input(str(d / "input.toml"))
    assert c["cross_sections"] == [str(d / "../cs/a.json"), str(d / "b.json")]
    assert c["steps"] == 105 and c["seed"] == 7 and c["poisson_levels"] == 9
    assert c["eb"] == -100.0 * (co.Td * co.nair)
    init = c["init_files"]
    assert init["ne_file"] == str(d / "afivo/ne.hdf") and init["method"] == "noiseless"
    assert init["format"] == "afivo" and math.isinf(init["fluid_threshold"])
    assert c["outpath"] == str(d / "input")
    assert read_input(str(d / "input.toml"), tmax=3e-12)["steps"] == 3


def test_sampseg_point_seed():
    """z1 = z0 (the default when [seed] has no z1): a 3-D Gaussian of width w at z0."""
    x = sampseg(1e-3, 1e-3, 2e-5, 20_000, np.random.default_rng(2))
    assert abs(x[:, 2].mean() - 1e-3) < 5 * 2e-5 / math.sqrt(20_000)
    np.testing.assert_allclose(x.std(axis=0), 2e-5, rtol=0.03)


def test_cross_sections_take_the_air_densities(tmp_path):
    """main.jl:46-47: N2 at 0.79 and O2 at 0.21 of nair; a record's rate scales with its
    target's density (load_lxcat, lxcat.jl:17-134)."""
    import json

    from mcstreamer_b200 import lxcat
    recs = lxcat.synthetic_records(0, target="N2")
    f = tmp_path / "cs.json"
    f.write_text(json.dumps(recs))
    nair = 2.5e25
    a = lxcat.load_lxcat([f], {"N2": nair * 0.79, "O2": nair * 0.21})
    recs_o2 = lxcat.synthetic_records(0, target="O2")
    f2 = tmp_path / "cs2.json"
    f2.write_text(json.dumps(recs_o2))
    b = lxcat.load_lxcat([f2], {"N2": nair * 0.79, "O2": nair * 0.21})
    assert a.maxrate / b.maxrate == pytest.approx(0.79 / 0.21, rel=1e-12)
