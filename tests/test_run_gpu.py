"""MCStreamer.main(finput) on the device (run.main): a small input in the reference's TOML
schema, once with seed electrons (sampseg, a needle fluid, photo-ionization) and once from
init files (AfivoLoader, PoissonInitSampling, fluid_threshold), each run through nsteps with
its output files."""
import json
import math

import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import fieldsio, h5, lxcat
from mcstreamer_b200.run import main

R, LEN, M, N = 1e-3, 2e-3, 32, 64


def _inputs(tmp_path, extra):
    recs = lxcat.synthetic_records(0, target="N2") + lxcat.synthetic_photo_records(target="N2", absorber="O2")
    (tmp_path / "cs.json").write_text(json.dumps(recs))
    text = f"""
eb = 15.0
field_units = "kV/cm"
n = 4000
maxp = 400000
ntarget = 10
nmax = 15
dt = 1e-12
tmax = 4e-12
cross_sections = ["cs.json"]
rng_seed = 3
initial_weight = 20.0
poisson_levels = 3

[domain]
R = {R}
L = {LEN}
M = {M}
N = {N}

[photoionization]
photon_weight = 1.0
photon_multiplier = 1000.0

[seed]
z0 = 0.8e-3
z1 = 1.1e-3
w = 4e-5

[interval]
poisson = 1e-12
output = 2e-12
resample = 2e-12
""" + extra
    (tmp_path / "input.toml").write_text(text)
    return str(tmp_path / "input.toml")


@pytest.mark.gpu
def test_main_with_seed_electrons_and_needle(ctx, tmp_path):
    finput = _inputs(tmp_path, """
[needle]
sigma_z = 2e-4
sigma_r = 5e-5
position_z = 1.5e-3
position_r = 0.0
ne0 = 1e19
""")
    # set-up only: the seed's ions are in qfixed, +w for each of the 4000 electrons (all
    # inside the grid), and nothing has moved
    r = main(finput, ctx=ctx, run=False, photon_capacity=2_000_000)
    try:
        assert r.diagnostics == [] and r.streamer.electrons.nparticles() == 4000
        assert r.streamer.grid.read_fixed(L.Q_FIXED).sum() == 4000 * round(20.0 * 2 ** 32)
    finally:
        r.close()
    r = main(finput, ctx=ctx, photon_capacity=2_000_000)
    try:
        assert r.steps == 4 and len(r.diagnostics) == 4
        assert r.eb == -1.5e6
        s = r.streamer
        assert s.photons is not None and s.fluid is not None
        assert all(d["active_superelectrons"] > 0 for d in r.diagnostics)
        assert s.fluid.download()[0].max() > 0
        out = sorted((tmp_path / "input").glob("*.h5"))
        assert [p.name for p in out] == ["0000.h5", "0001.h5"]
        f = fieldsio.load_fields(str(out[0]))
        assert f["grid"]["N"] == N and f["ez"].shape == (M, N + 1)
    finally:
        r.close()


@pytest.mark.gpu
def test_main_from_init_files(ctx, tmp_path):
    rc = (np.arange(M) + 0.5) * (R / M)
    zc = (np.arange(N) + 0.5) * (LEN / N)
    ne = np.asfortranarray(3e19 * np.exp(-rc[:, None] ** 2 / (2 * (1e-4) ** 2))
                           * ((zc > 5e-4) & (zc < 1.5e-3))[None, :])
    for name in ("ne.h5", "q.h5"):
        with h5.Writer(str(tmp_path / name)) as w:
            w.write("e", ne)
            w.write("M_plus", np.asfortranarray(1.01 * ne))
            w.write("M_min", np.zeros_like(ne))
            w.write("r", rc)
            w.write("z", zc)
    finput = _inputs(tmp_path, """
[init_files]
ne_file = "ne.h5"
q_file = "q.h5"
method = "poisson"
format = "afivo"
fluid_threshold = 2e19
""")
    r0 = main(finput, ctx=ctx, tmax=2e-12, run=False, photon_capacity=2_000_000)
    try:
        ne_fluid0 = r0.streamer.fluid.download()[0]
    finally:
        r0.close()
    r = main(finput, ctx=ctx, tmax=2e-12, photon_capacity=2_000_000)
    try:
        assert r.steps == 2
        s = r.streamer
        assert s.fluid is not None and (s.fluid.download()[0] > 0).sum() > 0
        # no [needle]: the reference's hasfluid is false (main.jl:173-180), so the init-file
        # fluid keeps the density initfromfiles! gave it
        assert not s.hasfluid
        np.testing.assert_array_equal(s.fluid.download()[0], ne_fluid0)
        assert s.electrons.nparticles() > 1000
        assert math.isfinite(r.diagnostics[-1]["mean_energy"])
    finally:
        r.close()
