"""Streamer step on the 3-D mesh (cell + offset layout) against the CPU oracle:
trilinear node-field gather, Yoshida push, collisions, collision tracker (int64 CIC into
qfixed) and the fused particle deposit (int64 CIC into qpart)."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import jumc, lxcat, streamer
from oracle import pyoracle as po
from tests.helpers import broad, oracle_arrays, oracle_pop, particle_mismatch, vec_relerr

NX, NY, NZ, H = 16, 16, 32, 4e-6
CENTRE = (NX * H / 2, NY * H / 2, NZ * H / 2)


def _field_nodes(grid):
    fn = streamer.gaussian_charge_field(CENTRE, 10e-6, 2e21, e_bg=(0.0, 0.0, -15e6))
    x, y, z = grid.node_coords(0, grid.nz + 1)
    return fn(x, y, z)


def _setup(ctx, n, precision, seed=21, spread=14e-6, emax_ev=120.0, weight=1e3, capf=3):
    t = lxcat.synthetic_table(0, uniform_sharing=True)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.Grid3D(NX, NY, NZ, H, precision=precision, ctx=ctx)
    e = _field_nodes(grid)
    grid.set_efield(e)
    e_or = e.astype(np.float32).astype(np.float64) if precision == "fp32" else e
    p0 = broad(n, seed, emax_ev=emax_ev, x0=CENTRE, spread=spread)
    p0.w[:] = weight
    pop = jumc.Population(capf * n, p0, tab, precision=precision, seed=seed, mesh=grid)
    otab = po.OracleTable.from_lxcat(t)
    ofield = po.field_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0), e_or.reshape(-1))
    return t, tab, grid, p0, pop, otab, ofield


def _close(*objs):
    for o in objs:
        o.close()


@pytest.mark.gpu
def test_mesh_step_fp64_matches_oracle_with_tracker_and_deposit(ctx):
    n = 32768
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp64")
    # positions as the device holds them (cell + offset round trip)
    p_dev = pop.download()
    opop = oracle_pop(p_dev, 3 * n, 21)
    trk = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    fld = streamer.FieldInterp(grid)
    grid.zero(L.Q_FIXED)
    grid.zero(L.Q_PART)
    dt = 2e-13
    streamer.advance_deposit(pop, fld, dt, streamer.CollisionTracker(grid), grid, -1.0)
    assert po.advance(opop, otab, ofield, dt, tracker=trk) == 0
    g, o = pop.download(), oracle_arrays(opop)
    assert g.n == o.n and g.n > n
    bad = particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30)
    assert bad.sum() == 0, f"{bad.sum()} slots differ, worst {vec_relerr(g.x, o.x).max():.3g}"
    qf = grid.read_fixed(L.Q_FIXED)
    assert qf.sum() == trk._q.sum()
    # per node: a few units of 2^-32 e from per-corner rounding of several deposits
    assert np.abs(qf - trk._q).max() <= 8
    # fused deposit == oracle density! of the oracle's post-step population
    qp = grid.read_fixed(L.Q_PART)
    dep = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    po.deposit(opop, dep, -1.0)
    assert qp.sum() == dep._q.sum()
    assert np.abs(qp - dep._q).max() <= 8
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
def test_mesh_step_fp32_within_tolerance(ctx):
    n = 32768
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp32")
    p_dev = pop.download()
    opop = oracle_pop(p_dev, 3 * n, 21)
    fld = streamer.FieldInterp(grid)
    dt = 2e-13
    jumc.advance(pop, fld, dt)
    assert po.advance(opop, otab, ofield, dt) == 0
    g, o = pop.download(), oracle_arrays(opop)
    bad = particle_mismatch(g, o, 1e-5, xatol=1e-13, vatol=1e-2, satol=1e-5, n=n)
    assert bad.sum() / n < 2e-3, f"{bad.sum()} of {n} parents differ"
    assert abs(g.n - o.n) <= max(8, 0.01 * (o.n - n))
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
def test_mesh_deposit_is_bit_exact(ctx):
    n = 50000
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp32", spread=20e-6)
    rng = np.random.default_rng(3)
    p0.w[:] = 10 ** rng.uniform(2, 4, n)
    p0.active[::11] = 0
    pop.upload(p0)
    grid.zero(L.Q_PART)
    streamer.density(grid, pop, -1.0)
    q = grid.read_fixed(L.Q_PART)
    dep = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    po.deposit(oracle_pop(p0, n, 0), dep, -1.0, quantize_f32=True)
    np.testing.assert_array_equal(q, dep._q)
    # total charge == sum of llrint(w * 2^32) over active in-mesh particles
    inside = (grid.cell_key(p0.x) < np.iinfo(np.int64).max) & (p0.active == 1)
    w32 = p0.w.astype(np.float32).astype(np.float64)
    assert q.sum() == -np.sum(np.rint(w32[inside] * 2.0 ** 32).astype(np.int64))
    _close(pop, grid, tab)


@pytest.mark.gpu
def test_mesh_particles_leaving_and_reentering(ctx):
    """Fast particles near the faces leave the mesh (zero field outside, gridfields.jl:116)."""
    n = 8192
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp64", spread=30e-6, emax_ev=400.0, capf=40)
    p_dev = pop.download()
    opop = oracle_pop(p_dev, 40 * n, 21)
    fld = streamer.FieldInterp(grid)
    for _ in range(6):
        jumc.advance(pop, fld, 4e-13)
        assert po.advance(opop, otab, ofield, 4e-13) == 0
    g, o = pop.download(), oracle_arrays(opop)
    outside = (grid.cell_key(o.x) == np.iinfo(np.int64).max).sum()
    assert outside > 0
    assert g.n == o.n
    bad = particle_mismatch(g, o, 1e-11, xatol=1e-30, vatol=1e-30)
    assert bad.sum() <= 2, f"{bad.sum()} slots differ"
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
@pytest.mark.parametrize("chunks,weights", [(1, "exact"), (3, "exact"), (7, "exact"), (3, "rounded")])
def test_host_resident_step_equals_device_step(ctx, chunks, weights):
    """mcs_advance_deposit_host (chunked, pipelined transfers) against upload + fused step +
    download of the same population: the same particles in the same slots, the same
    secondaries in the same order, the same int64 charges.  With FP32-exact weights the
    stepped particles' weights stay on the host (57 bytes down per particle); weights that
    the FP32 upload rounds come back rounded, as a download gives them (65 bytes)."""
    n = 40000
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp32", emax_ev=200.0)
    host_in = pop.download()                     # the cloud as the device layout holds it
    fld = streamer.FieldInterp(grid)
    trk = streamer.CollisionTracker(grid)
    dt = 2e-13
    grid.zero(L.Q_FIXED); grid.zero(L.Q_PART)
    streamer.advance_deposit(pop, fld, dt, trk, grid, -1.0)
    ref = pop.download()
    q_ref = (grid.read_fixed(L.Q_FIXED), grid.read_fixed(L.Q_PART))
    assert ref.n > n                            # the step made secondaries
    cap = 2 * n
    host = jumc.ParticleArrays.empty(cap)
    host.x[:n], host.v[:n], host.w[:n], host.s[:n], host.active[:n] = (host_in.x, host_in.v, host_in.w, host_in.s,
                                                                       host_in.active)
    if weights == "rounded":
        host.w[:n] *= 1.0 + 2.0 ** -40          # off the FP32 grid; rounds back to the same float
        assert not np.array_equal(host.w[:n], host_in.w)
    work = jumc.Population((n + chunks - 1) // chunks + n // 2, None, tab, precision="fp32", seed=21, mesh=grid)
    grid.zero(L.Q_FIXED); grid.zero(L.Q_PART)
    m = streamer.advance_deposit_host(work, fld, dt, trk, grid, host, n, -1.0, chunks=chunks)
    assert m == ref.n
    chunk = (n + chunks - 1) // chunks
    nch = (n + chunk - 1) // chunk
    up, down = streamer.host_step_bytes(work)
    assert up == 65 * n
    assert down == 65 * (m - n) + (65 if weights == "rounded" else 57) * n + 12 * nch
    np.testing.assert_array_equal(host.x[:m], ref.x)
    np.testing.assert_array_equal(host.v[:m], ref.v)
    np.testing.assert_array_equal(host.w[:m], ref.w)
    np.testing.assert_array_equal(host.s[:m], ref.s)
    np.testing.assert_array_equal(host.active[:m], ref.active)
    np.testing.assert_array_equal(grid.read_fixed(L.Q_FIXED), q_ref[0])
    np.testing.assert_array_equal(grid.read_fixed(L.Q_PART), q_ref[1])
    _close(work, pop, grid, tab)


@pytest.mark.gpu
def test_every_mesh_kernel_shape_gives_the_same_step(ctx):
    """MCS_OPT_MESH_SHAPE changes block size, tile length and register budget of the FP32 mesh
    step, never its result: particles, secondaries and charges are bit-identical."""
    n = 30000
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp32", emax_ev=200.0)
    snap = jumc.Population(3 * n, None, tab, precision="fp32", seed=21, mesh=grid)
    ctx.check(ctx.lib.mcs_pop_copy(snap.h, pop.h))
    fld = streamer.FieldInterp(grid)
    trk = streamer.CollisionTracker(grid)
    ref = None
    try:
        for shape in range(L.MESH_SHAPES):
            ctx.check(ctx.lib.mcs_ctx_set_option(ctx.h, L.OPT_MESH_SHAPE, shape))
            ctx.check(ctx.lib.mcs_pop_copy(pop.h, snap.h))
            ctx.check(ctx.lib.mcs_pop_set_seed(pop.h, 21, 0))
            grid.zero(L.Q_FIXED); grid.zero(L.Q_PART)
            streamer.advance_deposit(pop, fld, 2e-13, trk, grid, -1.0)
            g = pop.download()
            got = (g.x.tobytes(), g.v.tobytes(), g.w.tobytes(), g.s.tobytes(), g.active.tobytes(),
                   grid.read_fixed(L.Q_FIXED).tobytes(), grid.read_fixed(L.Q_PART).tobytes())
            if ref is None:
                ref = got
                assert g.n > n
            assert got == ref, f"shape {shape} differs"
    finally:
        ctx.check(ctx.lib.mcs_ctx_set_option(ctx.h, L.OPT_MESH_SHAPE, 0))
    _close(snap, pop, grid, tab)


@pytest.mark.gpu
def test_mesh_fp64_three_steps_ragged_tiles_with_attachment(ctx):
    """Three fused steps (push, collide, track, deposit) of a population that spans several
    tiles with a ragged last one, with frequent attachment (removed electrons keep
    sub-stepping, mixed_population.jl:32) and ionization: particles and secondaries slot for
    slot, charges node for node, against the oracle after every step."""
    from tests.helpers import attaching_table
    n = 3 * 2048 + 777
    t = attaching_table(uniform_sharing=True)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.Grid3D(NX, NY, NZ, H, precision="fp64", ctx=ctx)
    e = _field_nodes(grid)
    grid.set_efield(e)
    p0 = broad(n, 5, emax_ev=60.0, x0=CENTRE, spread=14e-6)
    p0.w[:] = 1e3
    pop = jumc.Population(8 * n, p0, tab, precision="fp64", seed=5, mesh=grid)
    otab = po.OracleTable.from_lxcat(t)
    ofield = po.field_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0), e.reshape(-1))
    opop = oracle_pop(pop.download(), 8 * n, 5)
    trk = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    fld = streamer.FieldInterp(grid)
    grid.zero(L.Q_FIXED)
    dt = 2e-13
    removed = 0
    for _ in range(3):
        grid.zero(L.Q_PART)
        streamer.advance_deposit(pop, fld, dt, streamer.CollisionTracker(grid), grid, -1.0)
        assert po.advance(opop, otab, ofield, dt, tracker=trk) == 0
        g, o = pop.download(), oracle_arrays(opop)
        assert g.n == o.n
        bad = particle_mismatch(g, o, 1e-12, xatol=1e-30, vatol=1e-30)
        assert bad.sum() == 0, f"{bad.sum()} slots differ"
        removed = int((g.active[:n] == 0).sum())
        qf = grid.read_fixed(L.Q_FIXED)
        assert qf.sum() == trk._q.sum() and np.abs(qf - trk._q).max() <= 8
        dep = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
        po.deposit(opop, dep, -1.0)
        qp = grid.read_fixed(L.Q_PART)
        assert qp.sum() == dep._q.sum() and np.abs(qp - dep._q).max() <= 8
    assert g.n > n and removed > 0          # both ionization and attachment happened
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
def test_mesh_step_of_an_empty_population(ctx):
    """No particles: the step (and its append) leaves the population empty and deposits
    nothing."""
    t, tab, grid, p0, pop0, otab, ofield = _setup(ctx, 64, "fp32")
    pop0.close()
    pop = jumc.Population(1024, jumc.ParticleArrays.empty(0), tab, precision="fp32", seed=1, mesh=grid)
    fld = streamer.FieldInterp(grid)
    grid.zero(L.Q_FIXED)
    grid.zero(L.Q_PART)
    for _ in range(2):
        streamer.advance_deposit(pop, fld, 2e-13, streamer.CollisionTracker(grid), grid, -1.0)
    ctx.sync()
    assert pop.nparticles() == 0
    assert not grid.read_fixed(L.Q_PART).any() and not grid.read_fixed(L.Q_FIXED).any()
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
def test_mesh_step_beyond_capacity_is_reported(ctx):
    """Secondaries beyond the population's capacity: MCS_ERR_CAPACITY (population.jl:90's
    error), and the population stops at its capacity."""
    n = 20000
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, n, "fp32", emax_ev=200.0, capf=1)
    fld = streamer.FieldInterp(grid)
    with pytest.raises(L.MCSError) as err:
        for _ in range(4):
            streamer.advance_deposit(pop, fld, 2e-13, streamer.CollisionTracker(grid), grid, -1.0)
        ctx.sync()
    assert err.value.code == L.ERR_CAPACITY
    assert pop.nparticles() == n
    _close(fld, pop, grid, tab)


@pytest.mark.gpu
def test_charge_read_by_occupied_planes(ctx):
    """read_fixed_planes moves only the z-slab that holds charge and leaves the host array equal
    to the full read, also after the cloud moved and left planes empty."""
    t, tab, grid, p0, pop, otab, ofield = _setup(ctx, 6000, "fp32", spread=5e-6)
    plane = (NX + 1) * (NY + 1)
    host = np.zeros((NX + 1) * (NY + 1) * (NZ + 1), dtype=np.int64)
    grid.zero(L.Q_PART)
    streamer.density(grid, pop, -1.0)
    filled = grid.read_fixed_planes(L.Q_PART, host)
    full = grid.read_fixed(L.Q_PART)
    np.testing.assert_array_equal(host, full)
    nz = np.nonzero(full.reshape(NZ + 1, plane).any(axis=1))[0]
    assert filled == (nz[0], nz[-1] + 1) and filled[1] - filled[0] < NZ + 1
    # a smaller cloud near the bottom: the earlier slab's planes above it become zero
    p1 = broad(2000, 7, emax_ev=10.0, x0=(CENTRE[0], CENTRE[1], 6 * H), spread=3e-6)
    pop2 = jumc.Population(4000, p1, tab, precision="fp32", seed=7, mesh=grid)
    grid.zero(L.Q_PART)
    streamer.density(grid, pop2, -1.0)
    filled2 = grid.read_fixed_planes(L.Q_PART, host, filled)
    np.testing.assert_array_equal(host, grid.read_fixed(L.Q_PART))
    assert filled2[1] <= filled[1]
    # nothing deposited: the slab is empty and the host array all zero
    grid.zero(L.Q_PART)
    assert grid.read_fixed_planes(L.Q_PART, host, filled2) == (0, 0)
    assert not host.any()
    _close(pop2, pop, grid, tab)
