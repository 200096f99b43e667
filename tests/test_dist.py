"""Multi-process host logic of the sharded streamer step, on CPU with the gloo backend
(world size 2): sharded deposits summed by an int64 all-reduce equal the single-process
deposit bit for bit; instance balancing; a rank that leaves early becomes an error on its
peer instead of a hang."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from mcstreamer_b200 import dist as mdist


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


NX, NY, NZ, H = 8, 8, 8, 4e-6


def _cloud(n):
    rng = np.random.default_rng(3)
    x = (NX * H / 2) + rng.normal(0.0, 6e-6, (n, 3))
    w = 10 ** rng.uniform(2, 4, n)
    return x, w


def _deposit(x, w):
    from oracle import pyoracle as po
    from tests.helpers import oracle_pop
    from mcstreamer_b200.jumc import ParticleArrays
    n = len(w)
    p = ParticleArrays(x, np.zeros((n, 3)), w, np.ones(n), np.ones(n, np.uint8))
    trk = po.tracker_cart3d(NX, NY, NZ, H, (0.0, 0.0, 0.0))
    po.deposit(oracle_pop(p, n, 0), trk, -1.0)
    return trk._q.copy()


def _rank_deposit(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    x, w = _cloud(n)
    lo, hi = mdist.shard_bounds(n, rank, world)
    q = torch.from_numpy(_deposit(x[lo:hi], w[lo:hi]))
    mdist.allreduce_int64_(q)
    if rank == 0:
        out.put(q.numpy().tobytes())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_deposit_allreduce_is_exact():
    n, world = 20000, 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_deposit, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = np.frombuffer(out.get(timeout=120), dtype=np.int64)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    x, w = _cloud(n)
    np.testing.assert_array_equal(got, _deposit(x, w))


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 100, 4194304):
        for world in (1, 2, 3, 8):
            spans = [mdist.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1


def test_balance_instances_is_deterministic_and_balanced():
    rng = np.random.default_rng(3)
    work = 10 ** rng.uniform(np.log10(4096), np.log10(1048576), 256)   # electrons per instance
    a = mdist.balance_instances(work, 8)
    assert a == mdist.balance_instances(work, 8)
    assert sorted(i for lst in a for i in lst) == list(range(256))
    loads = [sum(work[i] for i in lst) for lst in a]
    assert max(loads) / np.mean(loads) < 1.05


def _rank_leaves(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        return  # leaves between steps, without joining the next collective
    try:
        mdist.allreduce_int64_(torch.zeros(16, dtype=torch.int64))
        out.put("no error")
    except Exception as e:  # the peer is gone: the collective fails instead of hanging
        out.put(type(e).__name__)


def test_lost_rank_surfaces_as_error():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_leaves, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = out.get(timeout=120)
    for p in procs:
        p.join(60)
    assert res != "no error"


# ---- swarm instances dealt to ranks (no data-path collective), results gathered ----
INST = [(0, 120.0, 96, 5), (1, 300.0, 400, 6), (2, 800.0, 160, 7), (0, 50.0, 320, 8), (1, 600.0, 64, 9),
        (2, 200.0, 250, 10), (0, 1000.0, 128, 11)]   # (gas, E/N in Td, electrons, seed)


def _instance_result(k):
    """One tiny swarm instance stepped by the oracle: 15 steps of advance! + Swarm.resample!
    + repack!; the result is the final population's moments."""
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200 import lxcat, swarm
    from oracle import pyoracle as po
    gas, en, n, seed = INST[k]
    t = po.OracleTable.from_lxcat(lxcat.synthetic_table(gas))
    p = swarm.initial_particles(n, "maxwellian", seed)
    op = po.OraclePop(p.x, p.v, p.w, p.s, p.active, cap=8 * n, seed=seed)
    _, fin = po.swarm_run(op, t, po.field_uniform(0, 0, en * co.Td * 2.5e25), 1e-13, 15, n, 0.1, 1, threads=1)
    return fin.tolist()


def _rank_instances(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    work = [n * 15 for _, _, n, _ in INST]
    mine = mdist.my_instances(work, rank, world)
    local = {k: _instance_result(k) for k in mine}
    res = mdist.gather_by_index(local, len(INST))
    out.put((rank, mine, res))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_instances_gather_to_the_single_process_results():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_instances, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = [out.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    mines = sorted(i for _, mine, _ in got for i in mine)
    assert mines == list(range(len(INST)))            # every instance on exactly one rank
    assert all(len(mine) > 0 for _, mine, _ in got)
    ref = [_instance_result(k) for k in range(len(INST))]
    for _, _, res in got:                              # every rank holds every result
        assert res == ref


def test_shard_requests_is_a_balanced_partition():
    from mcstreamer_b200.serve import poisson_requests
    reqs = poisson_requests(200.0, 5.0, seed=4)
    parts = [mdist.shard_requests(reqs, r, 4) for r in range(4)]
    ids = sorted(q.rid for p in parts for q in p)
    assert ids == sorted(q.rid for q in reqs)
    loads = [sum(q.n for q in p) for p in parts]
    assert max(loads) / np.mean(loads) < 1.1
    assert mdist.shard_requests(reqs, 0, 1) == list(reqs)


def _rank_slab(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    plane, planes = 50, 40
    rng = np.random.default_rng(rank)
    q = np.zeros((planes, plane), dtype=np.int64)
    z0 = 5 + 12 * rank                                  # the ranks' charge in different planes
    q[z0:z0 + 9] = rng.integers(-2**40, 2**40, (9, plane))
    full = torch.from_numpy(q.copy()).reshape(-1)
    slab = torch.from_numpy(q.copy()).reshape(-1)
    mdist.allreduce_int64_(full)
    lo, hi = mdist.allreduce_slab_int64_(slab, plane)
    out.put((rank, lo, hi, bool(torch.equal(full, slab))))
    dist.barrier()
    dist.destroy_process_group()


def test_slab_allreduce_equals_full_allreduce():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_slab, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for _, lo, hi, same in got:
        assert same and (lo, hi) == (5, 26)
