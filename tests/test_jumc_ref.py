"""oracle.cpp pinned against a second, independent restatement of the Julia code.

oracle/jumc_ref.py restates advance!, do_one_collision!, collide, apply!, collisions!,
repack!, Swarm.resample!, resample!, density!, FieldInterp and the tracker in plain Python
from the Julia source (JuMC/src/mixed_population.jl:24-77, collisions.jl:26-39,96-123,159-192,
electron.jl:27,38-62,108-139, util.jl:4-30, population.jl:88-106,191-215,
Swarm/src/Swarm.jl:193-223, MCStreamer/src/grid.jl:33-90, gridfields.jl:94-224,
poisson.jl:65-84, resample.jl:7-84), with its own Philox4x32-10 and Julia's LinRange
arithmetic.  None of the expected values here come from oracle.cpp: both are fed the same
uniforms and must agree bit for bit."""
import numpy as np
import pytest

from mcstreamer_b200 import constants as co
from mcstreamer_b200 import lxcat, streamer
from oracle import jumc_ref as R
from oracle import pyoracle as po
from tests.helpers import attaching_table, broad, oracle_arrays, oracle_pop, serial_run

# Philox4x32-10 known-answer vectors (Random123 kat_vectors)
KAT = [
    ([0, 0, 0, 0], [0, 0], (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_restatement_philox_known_answers(ctr, key, out):
    assert R.philox4x32_10(ctr, key) == out


def assert_same(rp: R.Population, op, what: str):
    x, v, w, s, a = rp.arrays()
    o = oracle_arrays(op)
    assert rp.n == o.n, f"{what}: {rp.n} particles, oracle {o.n}"
    for name, mine, theirs in (("x", x, o.x), ("v", v, o.v), ("w", w, o.w), ("s", s, o.s), ("active", a, o.active)):
        np.testing.assert_array_equal(mine, theirs[:o.n], err_msg=f"{what}: {name}")


@pytest.mark.parametrize("variant,uniform_sharing,emax", [(0, True, 120.0), (2, False, 120.0), ("att", False, 30.0),
                                                          ("att", True, 30.0)])
def test_advance_fixed_field_bit_for_bit(variant, uniform_sharing, emax):
    """advance! in a FixedField over 4 steps: every process fires (broad energies), both
    ionization kinds, attachment and the dead-particle sub-stepping."""
    if variant == "att":
        t = attaching_table(uniform_sharing)
    else:
        t = lxcat.synthetic_table(variant, uniform_sharing=uniform_sharing)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    n, seed, dt, ez = 300, 11, 4e-13, 5 * 100 * co.Td * 2.5e25
    p = broad(n, seed, emax_ev=emax)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 8 * n)
    op = oracle_pop(p, 8 * n, seed)
    for step in range(4):
        R.advance(rp, rt, R.FixedField([0.0, 0.0, ez]), dt, draws=R.philox_draws(seed, step))
        assert po.advance(op, ot, po.field_uniform(0, 0, ez), dt, threads=3) == 0
        assert_same(rp, op, f"step {step}")
    assert rp.n > n
    if variant == "att":
        assert sum(not q.active for q in rp.p) > 5


def _cyl_setup(Rr, Ln, M, N, n, seed):
    i = np.arange(M + 3)[:, None] / M
    j = np.arange(N + 3)[None, :] / N
    er = 2e6 * i * (1 - 0.3 * j) + 1e5 * np.sin(7 * j)
    ez = -1.5e7 + 3e6 * np.cos(3 * i) * j
    p = broad(n, seed, emax_ev=80.0)
    rng = np.random.default_rng(seed)
    r = Rr * np.sqrt(rng.random(n)) * 0.98
    th = 2 * np.pi * rng.random(n)
    p.x[:, 0], p.x[:, 1] = r * np.cos(th), r * np.sin(th)
    p.x[:, 2] = Ln * (0.02 + 0.96 * rng.random(n))
    return er, ez, p


# (R, L, M, N): the first grid has dr(grid) == R / M; on the second, step(grid.rc) and
# step(grid.zc) differ from R / M and L / N in the last bit, as on many grids
CYL_GRIDS = [(1e-4, 2e-4, 24, 48), (3e-4, 7e-4, 24, 100)]


def test_second_grid_has_centre_steps_off_by_an_ulp():
    g = R.GridCyl(*CYL_GRIDS[1])
    assert g.dr() != g.R / g.M or g.dz() != g.L / g.N


@pytest.mark.parametrize("grid", CYL_GRIDS)
def test_advance_field_interp_tracker_and_density_bit_for_bit(grid):
    """advance! in the staggered FieldInterp with the CollisionTracker, then density!."""
    Rr, Ln, M, N = grid
    t = lxcat.synthetic_table(0)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    er, ez, p = _cyl_setup(Rr, Ln, M, N, 250, 31)
    g = R.GridCyl(Rr, Ln, M, N)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 4 * len(p.w))
    op = oracle_pop(p, 4 * len(p.w), 31)
    rf, rtk = R.FieldInterp(g, er, ez), R.TrackerCyl(g)
    of, otk = po.field_cyl(Rr, Ln, M, N, er.T.ravel(), ez.T.ravel()), po.tracker_cyl(Rr, Ln, M, N)
    for step in range(3):
        R.advance(rp, rt, rf, 3e-13, tracker=rtk, draws=R.philox_draws(31, step))
        assert po.advance(op, ot, of, 3e-13, tracker=otk, threads=2) == 0
        assert_same(rp, op, f"step {step}")
    assert np.abs(rtk.q).sum() > 0
    np.testing.assert_array_equal(rtk.q, otk._q)
    dens = R.density_cyl(g, rp, -1.0)
    otk2 = po.tracker_cyl(Rr, Ln, M, N)
    po.deposit(op, otk2, -1.0)
    np.testing.assert_array_equal(dens, otk2._q)


def test_collisions_bit_for_bit():
    """collisions! (fixed-step sampling without a push) over three calls."""
    t = lxcat.synthetic_table(0)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    p = broad(500, 5)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 2000)
    op = oracle_pop(p, 2000, 5)
    for step in range(3):
        R.collisions(rp, rt, 2e-14, draws=lambda i, st=step: R.PhiloxEventDraws(5, i, st, R.TAG_COLLISIONS))
        assert po.collisions(op, ot, 2e-14, threads=2) == 0
        assert_same(rp, op, f"call {step}")


NX, NY, NZ, H = 16, 16, 32, 4e-6
CENTRE = (NX * H / 2, NY * H / 2, NZ * H / 2)


def _mesh_field():
    fn = streamer.gaussian_charge_field(CENTRE, 10e-6, 2e21, e_bg=(0.0, 0.0, -15e6))
    xs, ys, zs = H * np.arange(NX + 1), H * np.arange(NY + 1), H * np.arange(NZ + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.asarray(fn(X.ravel(), Y.ravel(), Z.ravel())).reshape(-1, 3)


def test_mesh_step_tracker_repack_sort_and_resample_bit_for_bit():
    """The 3-D node mesh of the streamer configurations: advance! with the trilinear field
    and the int64 CIC tracker, then repack!, the stable cell sort and resample!."""
    t = lxcat.synthetic_table(0)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    E = _mesh_field()
    p = broad(300, 21, emax_ev=120.0, x0=CENTRE, spread=14e-6)
    p.w[:] = 1e3
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 2000)
    op = oracle_pop(p, 2000, 21)
    rf, rtk = R.NodeField3D(NX, NY, NZ, H, (0, 0, 0), E), R.TrackerNodes3D(NX, NY, NZ, H, (0, 0, 0))
    of = po.field_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0), E.reshape(-1))
    otk = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    for step in range(3):
        R.advance(rp, rt, rf, 2e-13, tracker=rtk, draws=R.philox_draws(21, step))
        assert po.advance(op, ot, of, 2e-13, tracker=otk, threads=2) == 0
        assert_same(rp, op, f"step {step}")
    np.testing.assert_array_equal(rtk.q, otk._q)
    R.repack(rp)
    po.repack(op)
    assert_same(rp, op, "repack!")
    key = R.cell_key_3d(NX, NY, NZ, H, (0, 0, 0))
    R.sort_by_cell(rp, key)
    po.sort_cells(op, of)
    assert_same(rp, op, "cell sort")
    n0 = rp.n
    R.resample(rp, key, 3, 4, 21, 0)
    po.resample_cells(op, of, 3, 4, 0)
    assert_same(rp, op, "resample!")
    assert rp.n > n0 and sum(not q.active for q in rp.p) > 0   # both splits and merges happened


def test_cyl_cell_resample_bit_for_bit():
    """resample! on the reference's own cylindrical cells (cellindex over (0:M+1, 0:N+1))."""
    Rr, Ln, M, N = CYL_GRIDS[1]
    _, _, p = _cyl_setup(Rr, Ln, M, N, 600, 8)
    p.x[:, 2] = Ln * (0.4 + 0.2 * (p.x[:, 2] / Ln))       # crowd the cells so merges happen
    p.x[:, :2] *= 0.2
    p.w[:] = np.random.default_rng(8).uniform(1.0, 50.0, len(p.w))
    g = R.GridCyl(Rr, Ln, M, N)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 4000)
    op = oracle_pop(p, 4000, 8)
    of = po.field_cyl(Rr, Ln, M, N, np.zeros((M + 3) * (N + 3)), np.zeros((M + 3) * (N + 3)))
    key = R.cell_key_cyl(g)
    R.sort_by_cell(rp, key)
    po.sort_cells(op, of)
    assert_same(rp, op, "cell sort")
    R.resample(rp, key, 4, 6, 8, 3)
    po.resample_cells(op, of, 4, 6, 3)
    assert_same(rp, op, "resample!")


@pytest.mark.parametrize("n0", [200, 2000])
def test_swarm_resample_bit_for_bit(n0):
    """Swarm.resample!: roulette (n0 below the count) and Poisson clones (above)."""
    p = broad(600, 9)
    rp = R.Population(p.x, p.v, p.w, p.s, p.active, 8000)
    op = oracle_pop(p, 8000, 9, step=4)
    R.swarm_resample(rp, n0, 0.1, 9, 4)
    po.swarm_resample(op, n0, 0.1)
    assert_same(rp, op, "Swarm.resample!")


def test_serial_draws_replay_reproduces_a_run():
    """The injected-uniform input: per-particle values recorded from one serial run replay
    the same run through SerialDraws (the form the device's injected mode consumes)."""
    t = lxcat.synthetic_table(0)
    rt = R.Table.from_lxcat(t)
    p = broad(120, 4)
    gen = np.random.default_rng(4)
    recs = {}

    def draws(i):
        recs[i] = R.CountingSource(lambda: 1.0 - gen.random())
        return recs[i]
    a = R.Population(p.x, p.v, p.w, p.s, p.active, 1000)
    R.advance(a, rt, R.FixedField([0.0, 0.0, 1e7]), 4e-13, draws=draws)
    b = R.Population(p.x, p.v, p.w, p.s, p.active, 1000)
    R.advance(b, rt, R.FixedField([0.0, 0.0, 1e7]), 4e-13, draws=lambda i: R.SerialDraws(recs[i].values))
    for x, y in zip(a.arrays(), b.arrays()):
        np.testing.assert_array_equal(x, y)
    assert sum(len(r.values) for r in recs.values()) > 4 * 120


@pytest.mark.parametrize("uniform_sharing", [True, False])
def test_oracle_injected_uniforms_replay_the_serial_run(uniform_sharing):
    """orc_advance_injected fed each particle's draws of a serial run reproduces that run
    bit for bit over three steps (secondaries draw in the steps after they appear)."""
    t = attaching_table(uniform_sharing)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    p = broad(250, 3, emax_ev=60.0)
    ez = 5 * 100 * co.Td * 2.5e25
    rp, per_step = serial_run(rt, p, R.FixedField([0.0, 0.0, ez]), 4e-13, 7, steps=3)
    op = oracle_pop(p, 16 * len(p.w), 3)
    for k, per in enumerate(per_step):
        assert po.advance_injected(op, ot, po.field_uniform(0, 0, ez), 4e-13, per, threads=3) == 0
    assert_same(rp, op, "injected")
    assert sum(len(a) for a in per_step[-1]) > 1000


def test_oracle_injected_uniforms_running_out_is_reported():
    t = lxcat.synthetic_table(0)
    rt, ot = R.Table.from_lxcat(t), po.OracleTable.from_lxcat(t)
    p = broad(50, 2)
    _, per_step = serial_run(rt, p, R.FixedField([0.0, 0.0, 1e7]), 4e-13, 2)
    short = [a[:-1] for a in per_step[0]]
    op = oracle_pop(p, 1000, 2)
    assert po.advance_injected(op, ot, po.field_uniform(0, 0, 1e7), 4e-13, short) == 11
