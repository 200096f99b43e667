#!/usr/bin/env python
"""Throughput of the electron step (electron steps/s) on the streamer workload.

A step is one launch of the fused streamer step over the whole population: Yoshida push
in the trilinear node field, null-collision Monte Carlo (elastic, excitation, ionization,
attachment), collision tracker (int64 CIC into qfixed) and the particle deposit (int64 CIC
into qpart), preceded by zeroing qpart.  Default workload "cfg1": 128x128x256 mesh, h=4 um,
4,194,304 particles (weight 1e3, Gaussian cloud sigma 50 um, 1 eV isotropic), synthetic
gas 0, dt=2e-13 s, seed 1, FP32 push/sampling with FP64 time and int64 charge.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

N > 1 (torchrun, one rank per GPU): each rank steps its own shard of the cloud (same
number of particles per rank: weak scaling) and the int64 particle-deposit grids are
summed with an NCCL all-reduce every step, which is exact and order independent.
--impl reference times the CPU restatement of the reference's algorithm (the oracle,
all host threads) on a bounded sample of the same workload; only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path
from typing import Optional

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "electron steps/s"
UNIT = "electron-steps/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--particles", type=int, default=None, help="override the particle count (per rank)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-chunks", type=int, default=8, help="chunks of the pipelined host-resident step")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-cfg1", action="store_true", help="cfg2: skip the cfg1 kernel sub-record")
    ap.add_argument("--mesh-shape", type=int, default=None, help="cfg1/cfg2: MCS_OPT_MESH_SHAPE of the step kernel")
    ap.add_argument("--pre-steps", type=int, default=0, help="cfg1: evolve the input cloud this many steps first")
    ap.add_argument("--cap-factor", type=float, default=6.0, help="cfg2: population capacity / initial electrons")
    ap.add_argument("--replicas", type=int, default=16, help="cfg0: device replicas per precision")
    ap.add_argument("--oracle-replicas", type=int, default=4, help="cfg0: oracle replicas")
    ap.add_argument("--cfg0-steps", type=int, default=2000, help="cfg0: steps per run")
    ap.add_argument("--plain-stride", type=int, default=4, help="cfg3: plain drop-in measured on every n-th instance")
    ap.add_argument("--cfg3-profile", action="store_true",
                    help="cfg3: only W + K batched steps of one kernel variant (a short run to profile)")
    ap.add_argument("--variant", type=int, default=None, help="cfg3 --cfg3-profile: the k_bstep variant")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="cfg4: arrival window (s)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="cfg4: arrival rate (requests/s)")
    ap.add_argument("--serve-limit", type=float, default=420.0, help="cfg4: wall-clock limit of a serving run (s)")
    ap.add_argument("--serve-sample", type=int, default=24, help="cfg4: requests re-run alone (plain drop-in)")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 5 + k and r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def alg_bytes_per_launch(n_active: float, n_sec: float, nodes: int) -> float:
    """Algorithmic HBM bytes of one fused step launch: each active particle read once
    (cell 4 + offset 12 + velocity 12 + w 4 + s 4 + active 1 = 37 B) and written once
    (33 B, w unchanged), each secondary written once (37 B), the node field read once
    (12 B per node) and the particle-charge grid read-modified-written once (16 B per node)."""
    return n_active * 70.0 + n_sec * 37.0 + nodes * 12.0 + nodes * 16.0


# ---------------------------------------------------------------------------------------
class CpuSample:
    """The oracle (FP64 CPU restatement) on a bounded sample of the workload: one step of
    advance! with the tracker, then density! of the result, on the first M particles of
    the same cloud (M sized so one step takes about `seconds`)."""

    def __init__(self, spec, seconds: float, threads: int):
        from mcstreamer_b200 import lxcat, workloads
        from oracle import pyoracle as po
        self.po, self.spec, self.threads = po, spec, threads
        self.tab = po.OracleTable.from_lxcat(lxcat.synthetic_table(0))
        plane = (spec.nx + 1) * (spec.ny + 1)
        fn = workloads.streamer_field_fn(spec)
        xs = spec.h * np.arange(spec.nx + 1)
        ys = spec.h * np.arange(spec.ny + 1)
        e = np.empty((spec.nodes, 3))
        for k0 in range(0, spec.nz + 1, 32):
            k1 = min(spec.nz + 1, k0 + 32)
            Z, Y, X = np.meshgrid(spec.h * np.arange(k0, k1), ys, xs, indexing="ij")
            e[k0 * plane:k1 * plane] = fn(X.ravel(), Y.ravel(), Z.ravel())
        e = e.astype(np.float32).astype(np.float64)
        self.field = po.field_cart3d(spec.nx, spec.ny, spec.nz, spec.h, (0.0, 0.0, 0.0), e.reshape(-1))
        probe = min(spec.n, 65536)
        self.parts = workloads.streamer_particles(workloads.streamer_spec(spec.name, n=probe))
        dt = self.run()
        m = int(min(spec.n, max(probe, probe * seconds / max(dt, 1e-3))))
        m = max(probe, (m // 65536) * 65536) if m >= 65536 else m
        if m != probe:
            self.parts = workloads.streamer_particles(workloads.streamer_spec(spec.name, n=m))

    def run(self) -> float:
        po, spec, p = self.po, self.spec, self.parts
        m = p.n
        op = po.OraclePop(p.x, p.v, p.w, p.s, p.active, cap=2 * m, seed=spec.seed)
        trk = po.tracker_cart3d(spec.nx, spec.ny, spec.nz, spec.h, (0.0, 0.0, 0.0))
        dep = po.tracker_cart3d(spec.nx, spec.ny, spec.nz, spec.h, (0.0, 0.0, 0.0))
        t0 = time.perf_counter()
        po.advance(op, self.tab, self.field, spec.dt, tracker=trk, threads=self.threads)
        po.deposit(op, dep, -1.0)
        return time.perf_counter() - t0

    def measure(self, reps: int = 1) -> dict:
        dts = [self.run() for _ in range(reps)]
        dt = min(dts)
        m = self.parts.n
        return {"value": m / dt, "unit": UNIT, "cores": self.threads, "kind": "port",
                "sample": f"1 step (advance! + tracker + density!) of the first {m} particles of the same "
                          f"cloud, FP64 oracle, {self.threads} threads, {dt:.2f} s per step"}


def cpu_sample(spec, seconds: float, threads: int) -> dict:
    return CpuSample(spec, seconds / 2, threads).measure(reps=2)


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    # the cfg2 mesh (270M nodes) does not fit the oracle's host field arrays in a bounded
    # run: its per-electron work is timed on the cfg1 cloud (same gas, field, cloud)
    spec = workloads.streamer_spec("cfg1" if args.workload == "cfg2" else args.workload)
    threads = os.cpu_count() or 1
    os.environ["ORACLE_THREADS"] = str(threads)
    per_step = min(2.0, max(0.5, 60.0 / max(1, args.steps + args.warmup)))
    cs = CpuSample(spec, per_step, threads)
    for _ in range(args.warmup):
        cs.run()
    vals = [cs.measure() for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * spec.n / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"streamer step {args.workload}", "particles": spec.n,
                   "mesh": [spec.nx, spec.ny, spec.nz], "h": spec.h, "dt": spec.dt},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": vals[-1]["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
def run_mine(args):
    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import dist as mdist
    from mcstreamer_b200 import jumc, lxcat, streamer, workloads

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    spec = workloads.streamer_spec(args.workload, n=args.particles)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    if args.mesh_shape is not None:
        ctx.check(ctx.lib.mcs_ctx_set_option(ctx.h, L.OPT_MESH_SHAPE, args.mesh_shape))
    table = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.Grid3D(spec.nx, spec.ny, spec.nz, spec.h, precision="fp32", ctx=ctx)
    grid.set_efield_fn(workloads.streamer_field_fn(spec), planes_per_chunk=16)
    parts = workloads.streamer_particles(spec, rank=rank)
    seed = spec.seed + 1000 * rank
    # the input batch: a snapshot restored (device to device) before every step, so each
    # timed step is one push+collide+track+deposit launch over the same 4.2M-particle cloud
    fld = streamer.FieldInterp(grid)
    trk = streamer.CollisionTracker(grid)
    if args.pre_steps > 0:
        # an evolved cloud: the input advanced pre_steps steps (repacked, sorted by cell), so
        # the timed steps see relaxed energies and their real collisions and ionizations
        evo = jumc.Population(4 * spec.n, parts, table, precision="fp32", seed=seed, mesh=grid)
        for _ in range(args.pre_steps):
            streamer.advance_deposit(evo, fld, spec.dt, trk, grid, -1.0)
            ctx.check(ctx.lib.mcs_repack(evo.h))
        ctx.check(ctx.lib.mcs_sort_cells(evo.h, grid.h_))
        ctx.check(ctx.lib.mcs_repack(evo.h))
        parts = evo.download()
        evo.close()
        spec.n = parts.n
    snap = jumc.Population(spec.n, parts, table, precision="fp32", seed=seed, mesh=grid)
    pop = jumc.Population(2 * spec.n, None, table, precision="fp32", seed=seed, mesh=grid)
    qpart = torch.as_tensor(grid.charge_array(L.Q_PART), device=f"cuda:{local}") if ws > 1 else None
    n_active = float(parts.active.sum())

    def restore():
        ctx.check(ctx.lib.mcs_pop_copy(pop.h, snap.h))

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        grid.zero(L.Q_PART)
        if ev is not None:
            ev[1].record(stream)
        streamer.advance_deposit(pop, fld, spec.dt, trk, grid, -1.0)
        if ev is not None:
            ev[2].record(stream)
        if qpart is not None:
            mdist.allreduce_int64_(qpart)
        if ev is not None:
            ev[3].record(stream)

    grid.zero(L.Q_FIXED)
    ctx.check(ctx.lib.mcs_pop_step_log(pop.h, 1))
    for _ in range(args.warmup):
        restore()
        step()
    torch.cuda.synchronize()
    ctx.sync()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        for k in range(args.steps):
            restore()
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.sync()
    bracket_ms = t0.elapsed_time(t1)
    step_ms = float(sum(e[0].elapsed_time(e[3]) for e in evs))
    kms = [e[1].elapsed_time(e[2]) for e in evs]
    log = np.zeros((1, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_pop_read_step_log(pop.h, L.dptr(log), 1))
    n_post = float(log[0, L.S_COUNT])
    sec_per_step = max(0.0, n_post - n_active)
    clocks = clk.summary()
    active_timed = n_active * args.steps

    if dist is not None:
        t = torch.tensor([step_ms, active_timed, bracket_ms], device=f"cuda:{local}", dtype=torch.float64)
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = t.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms_max, active_all, bracket_max = float(mx[0]), float(sm[1]), float(mx[2])
    else:
        ms_max, active_all, bracket_max = step_ms, active_timed, bracket_ms
    value = active_all / (ms_max * 1e-3)
    kmean = float(np.mean(kms))
    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    alg = alg_bytes_per_launch(n_active, sec_per_step, spec.nodes)
    achieved = alg / (kmean * 1e-3) / 1e9
    rec_tag = "cfg1e" if args.pre_steps > 0 else "cfg1"   # the evolved cloud has its own capture
    tr = profile_record(f"traffic_k_step_mesh_{rec_tag}")
    traffic = tr.get("bytes_per_launch") if tr and not tr.get("stale") else None

    e2e = None
    if args.e2e_steps > 0:
        e2e = run_e2e(args, spec, parts, pop, grid, fld, trk, ctx, stream, torch, L, ws, dist, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_sample(spec, args.cpu_seconds, os.cpu_count() or 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": f"streamer step {args.workload}: {spec.nx}x{spec.ny}x{spec.nz} mesh h={spec.h:g} m, "
                            f"{spec.n} particles per GPU (w={spec.weight[0]:g}..{spec.weight[1]:g}), Gaussian cloud "
                            f"sigma=50um, 1 eV isotropic, synthetic gas 0, dt={spec.dt:g} s, one push+collide+track+"
                            f"CIC-deposit launch per step over the same input cloud",
                "particles_per_gpu": spec.n, "active_per_step": n_active, "secondaries_per_step": sec_per_step,
                "input_evolved_steps": args.pre_steps,
                "step_timing": "CUDA events around zero(qpart)+step kernel(+all-reduce) of each step, summed; the "
                               "device-to-device restore of the input cloud between steps is outside the windows",
                "ms_per_step_incl_restore": bracket_max / args.steps,
                "l2": "inputs larger than L2 (particle arrays 37 B x 4.2M = 155 MB per GPU)",
                "parallelism": f"dp{ws} (particle shards, int64 all-reduce of the deposit grid)" if ws > 1 else "1 GPU",
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "kernel": mesh_kernel_name(ctx), "kernel_ms": kmean,
                         "alg_bytes_per_launch": alg, "peak_source": f"{pk_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "issue": issue_roofline_from(profile_record(f"issue_k_step_mesh_{rec_tag}"),
                                                      n_active, kmean, clocks)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "gpu_launches": args.steps * 3,   # k_step_mesh, k_pool_scan, k_pool_copy
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_e2e(args, spec, parts, pop, grid, fld, trk, ctx, stream, torch, L, ws, dist, local):
    """The same step through the C ABI with a host-resident population (the plain drop-in for
    a Julia population in host memory): the particles live in pinned host arrays in the Julia
    layout and mcs_advance_deposit_host steps them in place, with uploads, fused steps and
    downloads pipelined over chunks; the deposit grid is read back every step.  The byte
    counts are the library's own (mcs_pop_host_step_bytes)."""
    import ctypes as C

    from mcstreamer_b200 import dist as mdist
    from mcstreamer_b200 import jumc, streamer

    chunks = max(1, args.e2e_chunks)
    n = parts.n
    cap = 2 * n
    nodes = spec.nodes
    # device workspace: one chunk and its secondaries
    work = jumc.Population(2 * ((n + chunks - 1) // chunks), None, pop.collisions, precision="fp32",
                           seed=spec.seed + 1000 * int(os.environ.get("RANK", "0")), mesh=grid)

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    ix, iv = pinned((n, 3), torch.float64), pinned((n, 3), torch.float64)
    iw, i_s, ia = pinned((n,), torch.float64), pinned((n,), torch.float64), pinned((n,), torch.uint8)
    ix[:], iv[:], iw[:], i_s[:], ia[:] = parts.x, parts.v, parts.w, parts.s, parts.active
    ox, ov = pinned((cap, 3), torch.float64), pinned((cap, 3), torch.float64)
    ow, os_, oa = pinned((cap,), torch.float64), pinned((cap,), torch.float64), pinned((cap,), torch.uint8)
    hq = pinned((nodes,), torch.int64)
    lib = ctx.lib
    nn = C.c_int64()
    h2d = d2h = 0
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    active = 0.0
    n_active = float(parts.active.sum())
    ms = 0.0
    for k in range(args.e2e_steps + 1):
        # the input cloud restored into the host arrays outside the timed window
        ox[:n], ov[:n], ow[:n], os_[:n], oa[:n] = ix, iv, iw, i_s, ia
        nn.value = n
        torch.cuda.synchronize()
        t0.record(stream)
        grid.zero(L.Q_PART)
        ctx.check(lib.mcs_advance_deposit_host(work.h, pop.collisions.h, fld.h, spec.dt, trk.h, grid.h_, -1.0,
                                               L.dptr(ox), L.dptr(ov), L.dptr(ow), L.dptr(os_), L.u8ptr(oa),
                                               C.byref(nn), cap, chunks))
        up, down = streamer.host_step_bytes(work)   # what the call copied (host counters, no device work)
        if ws > 1:
            mdist.allreduce_charge(grid, L.Q_PART)
        ctx.check(lib.mcs_grid_read_fixed(grid.h_, L.Q_PART, L.i64ptr(hq)))
        t1.record(stream)
        torch.cuda.synchronize()
        if k == 0:
            continue   # warm-up: the workspace's staging buffers are allocated here
        ms += t0.elapsed_time(t1)
        active += n_active
        h2d += up
        d2h += down + nodes * 8
    work.close()
    if ws > 1:
        t = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
        a = torch.tensor([active], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(a)
        active = float(a[0])
    return {"value": active / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d // args.e2e_steps,
            "d2h_bytes_per_step": d2h // args.e2e_steps, "steps": args.e2e_steps,
            "path": f"mcs_advance_deposit_host on pinned host arrays in the Julia layout ({chunks} chunks: uploads, "
                    "fused steps and downloads pipelined on three streams) + mcs_grid_read_fixed; CUDA events "
                    "around each step, the restore of the input cloud outside them"}


# ---------------------------------------------------------------------------------------
# The headline workload ("cfg2", the default): the large streamer run.  67,108,864
# electrons (log-uniform weights 1e2..1e4, Gaussian cloud sigma 50 um, 1 eV) on a
# 512x512x1024 mesh (h = 2 um) in the Gaussian-charge field plus -15 MV/m, dt = 2e-13 s,
# seed 2.  The population evolves from step to step -- ionization grows it by a few per cent
# a step, the secondaries are staged and appended in parent order, the tracker deposits
# their ions -- and every 10th step (steps 9, 19, ...) ends with resample!(ntarget = 64,
# nmax = 96), which sorts by cell first; every step ends with repack! (main.jl:313).  W warm-up steps are the first W steps of that run
# and the K timed steps the next K; a step is zero(qpart) + the fused push/collide/track/
# deposit launch (+ the resample on its step).
# ---------------------------------------------------------------------------------------
CFG2_PERIOD, CFG2_NTARGET, CFG2_NMAX = 10, 64, 96


def source_sha(files) -> str:
    import hashlib
    h = hashlib.sha256()
    for f in files:
        h.update((ROOT / f).read_bytes())
    return h.hexdigest()[:16]


def profile_record(name: str) -> Optional[dict]:
    """A committed per-kernel record (profiles/<name>.json) with the sha of the sources it was
    measured on; `stale` is set when those sources have changed since."""
    p = ROOT / "profiles" / f"{name}.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    files = d.get("sources")
    # a record without the sha of its kernel's sources cannot be shown current
    d["stale"] = (source_sha(files) != d.get("source_sha")) if files else True
    return d


class SubMeshOracle:
    """The oracle (FP64 restatement, all host threads) stepping a sample of the streamer
    workload on the box of the mesh within `half` cells of its centre: the node field of that
    box and two int64 deposit grids of its size (the full 270M-node cfg2 mesh does not fit
    the oracle's host arrays in a bounded run).  The cloud has sigma 25 cells; a particle
    beyond the box (over 5 sigma out) sees no field and deposits nothing."""

    def __init__(self, spec, threads: int, half: int = 128):
        from mcstreamer_b200 import lxcat, workloads
        from oracle import pyoracle as po
        self.po, self.spec, self.threads = po, spec, threads
        self.tab = po.OracleTable.from_lxcat(lxcat.synthetic_table(0))
        c = (spec.nx // 2, spec.ny // 2, spec.nz // 2)
        self.i0 = [max(0, ci - half) for ci in c]
        self.nc = [min(n, ci + half) - i0 for n, ci, i0 in zip((spec.nx, spec.ny, spec.nz), c, self.i0)]
        self.origin = tuple(spec.h * i for i in self.i0)
        nx, ny, nz = self.nc
        fn = workloads.streamer_field_fn(spec)
        xs = self.origin[0] + spec.h * np.arange(nx + 1)
        ys = self.origin[1] + spec.h * np.arange(ny + 1)
        plane = (nx + 1) * (ny + 1)
        e = np.empty(((nz + 1) * plane, 3))
        for k0 in range(0, nz + 1, 32):
            k1 = min(nz + 1, k0 + 32)
            Z, Y, X = np.meshgrid(self.origin[2] + spec.h * np.arange(k0, k1), ys, xs, indexing="ij")
            e[k0 * plane:k1 * plane] = fn(X.ravel(), Y.ravel(), Z.ravel())
        e = e.astype(np.float32).astype(np.float64)        # the device field is FP32
        self.field = po.field_cart3d(nx, ny, nz, spec.h, self.origin, e.reshape(-1))

    def step(self, op) -> float:
        po, spec = self.po, self.spec
        nx, ny, nz = self.nc
        trk = po.tracker_cart3d(nx, ny, nz, spec.h, self.origin)
        dep = po.tracker_cart3d(nx, ny, nz, spec.h, self.origin)
        t0 = time.perf_counter()
        po.advance(op, self.tab, self.field, spec.dt, tracker=trk, threads=self.threads, clamp=True)
        po.deposit(op, dep, -1.0)
        return time.perf_counter() - t0


def cfg2_sample(spec, m: int, seed: int):
    """m electrons of the cfg2 cloud distribution (the device draws the full cloud itself)."""
    from mcstreamer_b200 import workloads
    return workloads.streamer_particles(workloads.streamer_spec(spec.name, n=m))


def oracle_rate(sub: SubMeshOracle, parts, seconds: float, seed: int) -> dict:
    """Electron steps/s of the oracle on `parts`, sized down so one step takes about
    `seconds` (a strided subsample of the given particles)."""
    po = sub.po
    probe = min(parts.n, 32768)
    idx = np.linspace(0, parts.n - 1, probe).astype(np.int64)
    op = po.OraclePop(parts.x[idx], parts.v[idx], parts.w[idx], parts.s[idx], parts.active[idx], cap=4 * probe,
                      seed=seed)
    dt = sub.step(op)
    m = int(min(parts.n, max(probe, probe * seconds / max(dt, 1e-3))))
    idx = np.linspace(0, parts.n - 1, m).astype(np.int64)
    op = po.OraclePop(parts.x[idx], parts.v[idx], parts.w[idx], parts.s[idx], parts.active[idx], cap=4 * m,
                      seed=seed)
    active = float(parts.active[idx].sum())
    dt = sub.step(op)
    return {"value": active / dt, "unit": UNIT, "cores": sub.threads, "kind": "port", "m": m, "seconds": dt}


def host_link_gbs(torch, nbytes: int = 1 << 30, reps: int = 4) -> dict:
    """Pinned host <-> device copy bandwidth of this GPU (GB/s): each direction alone, and
    per direction with both running at once on two streams -- the bound of a pipelined
    host-resident step, whose uploads and downloads overlap."""
    h_up = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_dn = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_up = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_dn = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()

    def rate(up: bool, down: bool) -> float:
        cur = torch.cuda.current_stream()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        s_up.wait_event(e0)
        s_dn.wait_event(e0)
        for _ in range(reps):
            if up:
                with torch.cuda.stream(s_up):
                    d_up.copy_(h_up, non_blocking=True)
            if down:
                with torch.cuda.stream(s_dn):
                    h_dn.copy_(d_dn, non_blocking=True)
        cur.wait_stream(s_up)
        cur.wait_stream(s_dn)
        e1.record(cur)
        torch.cuda.synchronize()
        return reps * nbytes / (e0.elapsed_time(e1) * 1e-3) / 1e9

    rate(True, True)   # warm-up
    out = {"h2d_gbs": rate(True, False), "d2h_gbs": rate(False, True), "both_gbs_per_direction": rate(True, True)}
    del h_up, h_dn, d_up, d_dn
    torch.cuda.empty_cache()
    return out


def cfg2_e2e(args, spec, pop, grid, fld, trk, ctx, stream, torch, L):
    """The same steps through the C ABI with the population in HOST memory (the plain drop-in
    for a Julia Population): the population entering the first timed step is downloaded into
    pinned host arrays in the Julia layout (65 B per electron), and mcs_advance_deposit_host
    steps it in place -- uploads, fused steps and downloads pipelined over chunks; the weights,
    which a step leaves unchanged, stay on the host when the upload kept them exactly -- after
    which the deposit grid is brought to pinned host memory (the slab of z-planes that holds
    charge; the rest of the host array is kept zero), every step.  The byte counts are the
    library's own (mcs_pop_host_step_bytes).  No resample! is
    called (the library has no host-resident resample; it is one step in ten of the device
    run)."""
    import ctypes as C

    from mcstreamer_b200 import jumc, streamer
    n = pop.nparticles()
    cap = int(n * 1.25) + 1024
    chunks = max(1, args.e2e_chunks)

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    x, v = pinned((cap, 3), torch.float64), pinned((cap, 3), torch.float64)
    w, s, a = pinned((cap,), torch.float64), pinned((cap,), torch.float64), pinned((cap,), torch.uint8)
    hq = pinned((spec.nodes,), torch.int64)
    nn = C.c_int64()
    lib = ctx.lib
    ctx.check(lib.mcs_pop_download(pop.h, L.dptr(x), L.dptr(v), L.dptr(w), L.dptr(s), L.u8ptr(a), cap, C.byref(nn)))
    work = jumc.Population(int(1.5 * ((cap + chunks - 1) // chunks)) + 4096, None, pop.collisions, precision="fp32",
                           seed=spec.seed, mesh=grid)
    hq[:] = 0
    plane = (spec.nx + 1) * (spec.ny + 1)
    filled = (0, 0)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = active = 0.0
    h2d = d2h = 0
    for k in range(args.e2e_steps + 1):
        n_in = nn.value
        act_in = float(a[:n_in].sum())
        torch.cuda.synchronize()
        t0.record(stream)
        grid.zero(L.Q_PART)
        ctx.check(lib.mcs_advance_deposit_host(work.h, pop.collisions.h, fld.h, spec.dt, trk.h, grid.h_, -1.0,
                                               L.dptr(x), L.dptr(v), L.dptr(w), L.dptr(s), L.u8ptr(a), C.byref(nn),
                                               cap, chunks))
        up, down = streamer.host_step_bytes(work)   # what the call copied (host counters, no device work)
        # the whole deposit grid on the host, moving the z-slab that holds charge
        filled = grid.read_fixed_planes(L.Q_PART, hq, filled)
        t1.record(stream)
        torch.cuda.synchronize()
        if k == 0:
            continue   # warm-up: the workspace's staging buffers are allocated here
        ms += t0.elapsed_time(t1)
        active += act_in
        h2d += up
        d2h += down + (filled[1] - filled[0]) * plane * 8 + 16
    work.close()
    steps = args.e2e_steps
    m = nn.value
    host = jumc.ParticleArrays(x[:m], v[:m], w[:m], s[:m], a[:m])
    # the host link's own bound for these bytes: both directions at once, on this GPU, now
    link = host_link_gbs(torch)
    bound_ms = max(h2d, d2h) / steps / (link["both_gbs_per_direction"] * 1e9) * 1e3
    link.update({"bound_ms_per_step": bound_ms, "ms_per_step": ms / steps, "frac": bound_ms / (ms / steps),
                 "note": "pinned 1 GiB copies timed with CUDA events after the e2e steps; bound = the larger "
                         "direction's bytes per step at the both-directions rate; frac = bound / measured"})
    return host, {"value": active / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d // steps,
            "d2h_bytes_per_step": d2h // steps, "steps": steps, "electrons_at_start": n, "host_link": link,
            "path": f"mcs_advance_deposit_host on pinned host arrays in the Julia layout ({chunks} chunks: uploads, "
                    "fused steps and downloads pipelined on three streams; unchanged weights are not downloaded) + "
                    "the 2.15 GB deposit grid into a "
                    "pinned host array, every step, moving the z-planes that hold charge (mcs_grid_fixed_plane_range "
                    "+ mcs_grid_read_fixed_range; the host array equals the full grid); the population entering the "
                    "first timed step, evolving; CUDA events around each step; no resample! (no host-resident entry "
                    "point)", "deposit_planes": [int(filled[0]), int(filled[1])]}


def cfg1_kernel_record(ctx, table, stream, torch, L, steps: int = 20, warmup: int = 5) -> dict:
    """cfg1's kernel datum (4,194,304 electrons, 128x128x256 mesh, every step over the same
    1 eV input cloud restored device to device outside the windows)."""
    from mcstreamer_b200 import jumc, streamer, workloads
    spec = workloads.streamer_spec("cfg1")
    grid = streamer.Grid3D(spec.nx, spec.ny, spec.nz, spec.h, precision="fp32", ctx=ctx)
    grid.set_efield_gaussian(spec.centre, workloads.CHARGE_SIGMA, workloads.CHARGE_PEAK, workloads.E_BACKGROUND)
    snap = jumc.Population(spec.n, None, table, precision="fp32", seed=spec.seed, mesh=grid)
    snap.init_cloud(spec.n, spec.centre, workloads.CLOUD_SIGMA, workloads.CLOUD_ENERGY_EV, *spec.weight)
    ctx.check(ctx.lib.mcs_sort_cells(snap.h, grid.h_))
    pop = jumc.Population(2 * spec.n, None, table, precision="fp32", seed=spec.seed, mesh=grid)
    fld, trk = streamer.FieldInterp(grid), streamer.CollisionTracker(grid)
    grid.zero(L.Q_FIXED)
    kms = []
    for k in range(warmup + steps):
        ctx.check(ctx.lib.mcs_pop_copy(pop.h, snap.h))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        grid.zero(L.Q_PART)
        e0.record(stream)
        streamer.advance_deposit(pop, fld, spec.dt, trk, grid, -1.0)
        e1.record(stream)
        if k >= warmup:
            kms.append((e0, e1))
    torch.cuda.synchronize()
    ctx.sync()
    km = float(np.mean([a.elapsed_time(b) for a, b in kms]))
    alg = alg_bytes_per_launch(spec.n, 0.0, spec.nodes)
    fld.close()
    pop.close(); snap.close(); grid.close()
    return {"workload": "cfg1: 4,194,304 electrons (w 1e3) on 128x128x256 cells, h 4 um, 1 eV cloud restored before "
                        "each step", "kernel_ms": km, "electron_steps_per_s": spec.n / (km * 1e-3),
            "alg_bytes_per_launch": alg, "achieved_gbs": alg / (km * 1e-3) / 1e9}


def mesh_kernel_name(ctx) -> str:
    import ctypes as C
    v = C.c_int()
    ctx.check(ctx.lib.mcs_ctx_get_option(ctx.h, 1, C.byref(v)))
    b, p, m = C.c_int(), C.c_int(), C.c_int()
    ctx.check(ctx.lib.mcs_mesh_shape(v.value, C.byref(b), C.byref(p), C.byref(m)))
    return f"k_step_mesh<float,{b.value},{p.value},{m.value},8>"


def run_cfg2(args):
    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import dist as mdist
    from mcstreamer_b200 import jumc, lxcat, streamer, workloads

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    spec = workloads.streamer_spec("cfg2", n=args.particles)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    if args.mesh_shape is not None:
        ctx.check(ctx.lib.mcs_ctx_set_option(ctx.h, L.OPT_MESH_SHAPE, args.mesh_shape))
    table = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.Grid3D(spec.nx, spec.ny, spec.nz, spec.h, precision="fp32", ctx=ctx)
    t_setup = time.perf_counter()
    grid.set_efield_gaussian(spec.centre, workloads.CHARGE_SIGMA, workloads.CHARGE_PEAK, workloads.E_BACKGROUND)
    seed = spec.seed + 1000 * rank
    cap = int(args.cap_factor * spec.n)
    pop = jumc.Population(cap, None, table, precision="fp32", seed=seed, mesh=grid)
    pop.init_cloud(spec.n, spec.centre, workloads.CLOUD_SIGMA, workloads.CLOUD_ENERGY_EV, *spec.weight)
    ctx.check(ctx.lib.mcs_sort_cells(pop.h, grid.h_))
    streamer.reserve_resample(pop)   # the resample! scratch, allocated before the timed steps
    fld = streamer.FieldInterp(grid)
    trk = streamer.CollisionTracker(grid)
    qpart = torch.as_tensor(grid.charge_array(L.Q_PART), device=f"cuda:{local}") if ws > 1 else None
    grid.zero(L.Q_FIXED)
    total = args.warmup + args.steps
    ctx.check(ctx.lib.mcs_pop_step_log(pop.h, total))
    ctx.sync()
    t_setup = time.perf_counter() - t_setup

    act_in = [float(spec.n)]            # active electrons entering step k
    resampled = {}                      # step -> active electrons after its resample!

    def step(k, ev):
        ev[0].record(stream)
        grid.zero(L.Q_PART)
        ev[1].record(stream)
        streamer.advance_deposit(pop, fld, spec.dt, trk, grid, -1.0)
        ev[2].record(stream)
        if qpart is not None:               # the occupied z-slab of the deposit grid only
            mdist.allreduce_slab_int64_(qpart, (spec.nx + 1) * (spec.ny + 1))
        if (k + 1) % CFG2_PERIOD == 0:      # resample! sorts the population by cell first
            ctx.check(ctx.lib.mcs_resample_cells(pop.h, grid.h_, CFG2_NTARGET, CFG2_NMAX))
        ctx.check(ctx.lib.mcs_repack(pop.h))   # repack! every step, as nsteps does (main.jl:313)
        ev[3].record(stream)

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(total)]
    for k in range(args.warmup):
        step(k, evs[k])
        if (k + 1) % CFG2_PERIOD == 0:     # outside the step windows: the count entering step k+1
            resampled[k] = float(pop.moments()[L.M_COUNT])
    torch.cuda.synchronize()
    ctx.sync()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    n_first = pop.nparticles()
    with ClockSampler(local) as clk:
        for k in range(args.warmup, total):
            step(k, evs[k])
            if (k + 1) % CFG2_PERIOD == 0:
                resampled[k] = float(pop.moments()[L.M_COUNT])
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.sync()
    log = np.zeros((total, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_pop_read_step_log(pop.h, L.dptr(log), total))
    post = log[:, L.S_COUNT]
    for k in range(1, total):
        act_in.append(resampled.get(k - 1, post[k - 1]))
    timed = range(args.warmup, total)
    step_ms = float(sum(evs[k][0].elapsed_time(evs[k][3]) for k in timed))
    bracket_ms = evs[args.warmup][0].elapsed_time(evs[total - 1][3])
    kern = [evs[k][1].elapsed_time(evs[k][2]) for k in timed]
    res_ms = [evs[k][2].elapsed_time(evs[k][3]) for k in timed if (k + 1) % CFG2_PERIOD == 0]
    active_timed = float(sum(act_in[k] for k in timed))
    sec = [post[k] - act_in[k] for k in timed]
    clocks = clk.summary()

    if dist is not None:
        t = torch.tensor([step_ms, active_timed, bracket_ms], device=f"cuda:{local}", dtype=torch.float64)
        mx, sm = t.clone(), t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms_max, active_all, bracket_max = float(mx[0]), float(sm[1]), float(mx[2])
    else:
        ms_max, active_all, bracket_max = step_ms, active_timed, bracket_ms
    value = active_all / (ms_max * 1e-3)
    kmean = float(np.mean(kern))
    mean_in = float(np.mean([act_in[k] for k in timed]))
    mean_sec = float(np.mean(sec))
    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    alg = alg_bytes_per_launch(mean_in, max(0.0, mean_sec), spec.nodes)
    alg_particles = alg_bytes_per_launch(mean_in, max(0.0, mean_sec), 0)
    achieved = alg / (kmean * 1e-3) / 1e9
    # ncu records of the evolved cfg1 cloud (relaxed energies, like cfg2's timed steps): the
    # full cfg2 workload is too large for a multi-pass capture, so its DRAM traffic is that
    # capture's bytes per entering electron times cfg2's electrons
    tr = profile_record("traffic_k_step_mesh_cfg1e")
    issue = profile_record("issue_k_step_mesh_cfg1e")
    traffic = None
    if tr and not tr.get("stale") and tr.get("electrons"):
        traffic = tr["bytes_per_launch"] / tr["electrons"] * mean_in

    e2e = host = None
    if args.e2e_steps > 0 and ws == 1:
        host, e2e = cfg2_e2e(args, spec, pop, grid, fld, trk, ctx, stream, torch, L)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        # one oracle step of a strided sample of the evolved population (the host copy the
        # e2e leg stepped, else a download)
        parts = host if host is not None else pop.download()
        sub = SubMeshOracle(spec, os.cpu_count() or 1)
        r = oracle_rate(sub, parts, args.cpu_seconds, seed)
        cpu = {k: r[k] for k in ("value", "unit", "cores", "kind")}
        cpu["sample"] = (f"1 step (advance! + tracker + density!) of {r['m']} electrons taken evenly from the "
                         f"{parts.n} of the evolved cfg2 population, FP64 oracle on {r['cores']} threads, on the "
                         f"{sub.nc[0]}x{sub.nc[1]}x{sub.nc[2]}-cell box of the mesh around the cloud, "
                         f"{r['seconds']:.2f} s")
    cfg1 = None
    if rank == 0 and not args.no_cfg1:
        cfg1 = cfg1_kernel_record(ctx, table, stream, torch, L)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": f"streamer run cfg2: {spec.nx}x{spec.ny}x{spec.nz} mesh h={spec.h:g} m, {spec.n} electrons "
                            f"per GPU at the start (w log-uniform {spec.weight[0]:g}..{spec.weight[1]:g}, Gaussian "
                            f"cloud sigma=50um, 1 eV), Gaussian charge sigma=40um peak 1e20 e/m^3 + -15 MV/m, "
                            f"synthetic gas 0, dt={spec.dt:g} s, seed {spec.seed}; the population evolves; "
                            f"resample!(ntarget={CFG2_NTARGET}, nmax={CFG2_NMAX}) after every {CFG2_PERIOD}th step, repack! "
                            f"after every step (main.jl:313); "
                            f"warm-up = steps 0..{args.warmup - 1}, timed = steps {args.warmup}..{total - 1}",
                "electrons_entering_first_timed_step": act_in[args.warmup], "slots_at_first_timed_step": n_first,
                "mean_active_per_timed_step": mean_in, "secondaries_per_step": mean_sec,
                "secondaries_note": "post-step minus entering active electrons (ionizations minus attachments)",
                "active_per_step": [act_in[k] for k in range(total)],
                "step_kernel_ms": kmean, "resample_ms": res_ms,
                "capacity_slots": cap, "setup_s": t_setup,
                "l2": "inputs larger than L2 (>= 67M electrons x 37 B = 2.5 GB, mesh 4.3 GB field + 2.15 GB charges)",
                "step_timing": "CUDA events around each step (zero(qpart) + fused step kernel (+ int64 all-reduce) "
                               "+ resample! on its steps + repack!), summed over the K timed steps; the active-electron "
                               "count read after a resample! lies between two steps' windows",
                "ms_per_step_bracket": bracket_max / args.steps,
                "parallelism": f"dp{ws} (independent clouds, int64 all-reduce of the occupied z-slab of the deposit "
                               "grid)" if ws > 1
                               else "1 GPU",
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic,
                         "traffic_source": ("dram bytes per entering electron of one k_step_mesh launch on the "
                                            "evolved cfg1 cloud (profiles/traffic_k_step_mesh_cfg1e.json) times "
                                            "the mean entering electrons" if traffic is not None else None),
                         "kernel": mesh_kernel_name(ctx), "kernel_ms": kmean,
                         "alg_bytes_per_launch": alg, "alg_bytes_particles_only": alg_particles,
                         "frac_particles_only": alg_particles / (kmean * 1e-3) / 1e9 / hbm,
                         "alg_note": "70 B per entering electron + 37 B per secondary + 28 B per mesh node (field "
                                     "read, charge read-modify-write) per launch; the cloud covers about 1 % of "
                                     "the mesh, so the node term is an upper bound",
                         "peak_source": f"{pk_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "issue": issue_roofline_from(issue, mean_in, kmean, clocks)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "cfg1": cfg1,
            "clocks": clocks,
            # per step: k_step_mesh, k_pool_scan, k_pool_copy, and repack!'s k_scan,
            # k_repack_holes, k_repack_move; per resample!: 22 (keys, 4 radix passes of
            # histogram + scan + scatter, gather, segments, counts, merges, writes)
            "gpu_launches": args.steps * 6 + sum(1 for k in timed if (k + 1) % CFG2_PERIOD == 0) * 22,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def issue_roofline_from(rec: Optional[dict], n_active: float, kernel_ms: float, clocks) -> Optional[dict]:
    """Warp instructions per electron step from a committed ncu record (only when the kernel's
    sources are unchanged since the capture) against one instruction per cycle on each of the
    4 schedulers of every SM at the sampled clock."""
    if not rec or rec.get("stale") or not clocks or not clocks.get("sm_mhz") or not kernel_ms:
        return {"available": False, "why": "no ncu record for the current kernel sources"} if rec else None
    try:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    except Exception:
        return None
    per = rec["warp_inst_per_electron_step"]
    achieved = per * n_active / (kernel_ms * 1e-3)
    peak = sms * 4 * clocks["sm_mhz"] * 1e6
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp instructions/s",
            "frac": achieved / peak, "warp_inst_per_electron_step": per, "source": rec.get("note")}


def run_reference_cfg2(args):
    """The oracle on the cfg2 workload: a sample of the cfg2 cloud on the mesh box around it,
    evolved W untimed steps and then K timed steps (each a bounded sample), all host threads."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.streamer_spec("cfg2")
    threads = os.cpu_count() or 1
    sub = SubMeshOracle(spec, threads)
    per_step = min(2.0, max(0.5, 60.0 / max(1, args.steps + args.warmup)))
    parts = cfg2_sample(spec, 32768, spec.seed)
    probe = sub.po.OraclePop(parts.x, parts.v, parts.w, parts.s, parts.active, cap=4 * parts.n, seed=spec.seed)
    dt = sub.step(probe)
    m = int(max(32768, 32768 * per_step / max(dt, 1e-3)))
    parts = cfg2_sample(spec, m, spec.seed)
    cap = 8 * m
    op = sub.po.OraclePop(parts.x, parts.v, parts.w, parts.s, parts.active, cap=cap, seed=spec.seed)
    vals = []
    for k in range(args.warmup + args.steps):
        if op.n > cap // 2:
            break
        act = float(op.active[:op.n].sum())
        t = sub.step(op)
        sub.po.repack(op)
        if k >= args.warmup:
            vals.append(act / t)
    v = statistics.median(vals) if vals else None
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(vals),
        "warmup": args.warmup, "ms_per_step": 1e3 * spec.n / v if v else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "streamer run cfg2 (oracle on a sample of the cloud, evolving)", "sample_start": m,
                   "mesh_box": sub.nc, "h": spec.h, "dt": spec.dt},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{m} electrons of the cfg2 cloud distribution stepped by the FP64 oracle "
                                   f"(advance! + tracker + density!, repack!) on the {sub.nc[0]}x{sub.nc[1]}x"
                                   f"{sub.nc[2]}-cell box of the mesh around the cloud; median over the timed steps"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# The plain swarm ("cfg0"): Swarm.swarm at 100 Td -- 65,536 electrons of the synthetic gas
# 0 at N = 2.5e25 m^-3, 1 eV Maxwellian start, dt = 1e-13 s, 2000 steps, Swarm.resample!
# to 65,536 (tol 0.1, repack! every step), seeds 0..R-1 -- on the device in FP32 and FP64,
# and the same runs by the FP64 oracle on the host.  The line reports every coefficient of
# Swarm.jl:144-161 (W, D_L, D_T, <eps>, k_ion, nu, alpha, eta) with the replica 3 sigma and
# the FP32 relative error against the oracle.
# ---------------------------------------------------------------------------------------
CFG0 = dict(n0=65_536, en_td=100.0, density=2.5e25, dt=1e-13, nt=2000, tol=0.1)
CFG0_KEYS = ("drift", "diffusion_l", "diffusion_t", "mean_energy", "k_ion", "nu", "alpha", "eta")


def cfg0_row(r, table_proc, density):
    from mcstreamer_b200 import _lib as L
    ion = [j for j, p in enumerate(table_proc) if p.kind in (L.IONIZATION, L.IONIZATION_UNIFORM)]
    return {"drift": r.drift, "diffusion_l": r.diffusion_l, "diffusion_t": r.diffusion_t,
            "mean_energy": r.mean_energy, "k_ion": float(r.k[ion[0]]) / density, "nu": r.nu, "alpha": r.alpha,
            "eta": r.eta}


def cfg0_stats(rows):
    out = {}
    for k in CFG0_KEYS:
        a = np.array([r[k] for r in rows], dtype=np.float64)
        out[k] = (float(a.mean()), float(3.0 * a.std(ddof=1) / np.sqrt(len(a))) if len(a) > 1 else float("inf"))
    return out


def cfg0_oracle(seed: int, table, steps: int, n0: int, threads: int):
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200 import swarm
    from oracle import pyoracle as po
    ot = po.OracleTable.from_lxcat(table)
    eb = CFG0["en_td"] * co.Td * CFG0["density"]
    p = swarm.initial_particles(n0, "maxwellian", seed)
    op = po.OraclePop(p.x, p.v, p.w, p.s, p.active, cap=4 * n0, seed=seed)
    mom, fin = po.swarm_run(op, ot, po.field_uniform(0, 0, eb), CFG0["dt"], steps, n0, CFG0["tol"], 1, threads)
    return swarm.coefficients(CFG0["en_td"], eb, CFG0["dt"], mom, fin, table.proc)


def run_cfg0(args):
    import torch

    from mcstreamer_b200 import jumc, lxcat, swarm
    torch.cuda.set_device(0)
    lt = lxcat.synthetic_table(0)
    ctx = jumc.Context(0)
    tab = jumc.CollisionTable(lt, ctx)
    n0, nt = CFG0["n0"], args.cfg0_steps
    reps, oreps = args.replicas, args.oracle_replicas
    rows = {"fp32": [], "fp64": []}
    res = {"fp32": [], "fp64": []}
    secs = {}
    for prec in ("fp32", "fp64"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(reps):
            r = swarm.swarm_one(tab, CFG0["en_td"], CFG0["density"], n0, CFG0["dt"], nt, maxp=4 * n0,
                                precision=prec, seed=s, init="maxwellian", tol=CFG0["tol"])
            res[prec].append(r)
            rows[prec].append(cfg0_row(r, tab.proc, CFG0["density"]))
        secs[prec] = time.perf_counter() - t0
    threads = os.cpu_count() or 1
    os.environ["ORACLE_THREADS"] = str(threads)
    t0 = time.perf_counter()
    orows, ores = [], []
    for s in range(oreps):
        r = cfg0_oracle(s, lt, nt, n0, threads)
        ores.append(r)
        orows.append(cfg0_row(r, tab.proc, CFG0["density"]))
    osec = time.perf_counter() - t0
    # the FP64 device runs follow the oracle's trajectories: same seeds, same coefficients
    same = {k: max(abs(rows["fp64"][s][k] - orows[s][k]) / max(abs(orows[s][k]), 1e-300) for s in range(oreps))
            for k in CFG0_KEYS}
    st32, st64, sto = cfg0_stats(rows["fp32"]), cfg0_stats(rows["fp64"]), cfg0_stats(orows)
    coeff = {}
    for k in CFG0_KEYS:
        m32, e32 = st32[k]
        mo, eo = sto[k]
        both = float(np.hypot(e32, eo))
        coeff[k] = {"fp32": m32, "fp32_3sigma": e32, "fp64_device": st64[k][0], "fp64_device_3sigma": st64[k][1],
                    "oracle_fp64": mo, "oracle_3sigma": eo,
                    "fp32_rel_err_vs_oracle": (m32 - mo) / mo if mo else None,
                    "within_3sigma": bool(abs(m32 - mo) <= both),
                    "fp64_device_vs_oracle_same_seeds_max_rel": same[k]}
    half = nt // 2
    tavg = {}
    for key in ("drift", "mean_energy"):
        a32 = np.array([swarm.time_averages(r, half)[key] for r in res["fp32"]])
        ao = np.array([swarm.time_averages(r, half)[key] for r in ores])
        m32, e32 = float(a32.mean()), float(3 * a32.std(ddof=1) / np.sqrt(len(a32)))
        mo, eo = float(ao.mean()), (float(3 * ao.std(ddof=1) / np.sqrt(len(ao))) if len(ao) > 1 else float("inf"))
        tavg[key] = {"fp32": m32, "fp32_3sigma": e32, "oracle_fp64": mo, "oracle_3sigma": eo,
                     "fp32_rel_err_vs_oracle": (m32 - mo) / mo, "within_3sigma": bool(abs(m32 - mo) <= np.hypot(e32, eo))}
    electron_steps = sum(float(r.counts.sum()) for r in res["fp32"])
    line = {
        "metric": METRIC, "value": electron_steps / secs["fp32"], "unit": UNIT, "n_gpus": 1, "steps": nt,
        "warmup": 0, "ms_per_step": 1e3 * secs["fp32"] / (reps * nt), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain swarm cfg0: {n0} electrons, {CFG0['en_td']:g} Td, N={CFG0['density']:g} m^-3, "
                               f"synthetic gas 0, 1 eV Maxwellian start, dt={CFG0['dt']:g} s, {nt} steps, "
                               f"Swarm.resample!({n0}, {CFG0['tol']}) + repack! every step, seeds 0..{reps - 1} "
                               f"(device) and 0..{oreps - 1} (oracle)",
                   "replicas": reps, "oracle_replicas": oreps, "device_fp32_s": secs["fp32"],
                   "device_fp64_s": secs["fp64"], "oracle_s": osec, "oracle_threads": threads,
                   "timing": "wall clock of the replicas' mcs_swarm_run calls (each synchronises)"},
        "coefficients": coeff,
        "time_averaged_second_half": tavg,
        "units": {"drift": "m/s", "diffusion_l": "m^2/s", "diffusion_t": "m^2/s", "mean_energy": "J",
                  "k_ion": "m^3/s", "nu": "1/s", "alpha": "1/m", "eta": "1/m"},
        "cpu_baseline": {"value": sum(float(r.counts.sum()) for r in ores) / osec, "unit": UNIT, "cores": threads,
                         "kind": "port", "sample": f"{oreps} full replicas of the same runs, FP64 oracle"},
        "e2e": None, "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    tab.close()
    ctx.close()
    return 0


# ---------------------------------------------------------------------------------------
# Batched swarms ("cfg3"): swarm solves/s of 256 uneven instances in one batch, against the
# same solves run one after another through the plain single-population entry point.
# ---------------------------------------------------------------------------------------
BATCH_METRIC = "batched swarm solves/s"
BATCH_UNIT = "solves/s"


def batch_alg_bytes(n_active: float, n_sec: float) -> float:
    """Algorithmic HBM bytes of one batched advance! launch: each active electron read once
    (x, v 24 B + w 4 + s 4 + active 1 = 33 B) and written once (x, v, s: 28 B), each
    secondary written once (37 B)."""
    return n_active * 61.0 + n_sec * 37.0


def batch_cpu_sample(spec, seconds: float, threads: int) -> dict:
    """The oracle (FP64, all host threads) on instances of the workload: advance! +
    Swarm.resample! per step, timed until `seconds` pass; electron steps/s scaled to solves/s."""
    from mcstreamer_b200 import lxcat, workloads
    from oracle import pyoracle as po
    os.environ["ORACLE_THREADS"] = str(threads)
    tabs = {}
    done_e, t_used, ks = 0.0, 0.0, []
    order = np.argsort(spec.n)[len(spec.n) // 2:]  # mid-to-large instances keep the threads busy
    for k in order[::max(1, len(order) // 8)]:
        g = int(spec.gas[k])
        if g not in tabs:
            tabs[g] = po.OracleTable.from_lxcat(lxcat.synthetic_table(g))
        p0 = workloads.swarm_instance_particles(spec, int(k))
        op = po.OraclePop(p0.x, p0.v, p0.w, p0.s, p0.active, cap=4 * len(p0.w), seed=int(spec.seeds[k]))
        f = po.field_uniform(0, 0, float(spec.en_td[k]) * spec.density * 1e-21)
        po.advance(op, tabs[g], f, spec.dt, clamp=True)
        po.swarm_resample(op, int(spec.n[k]), 0.1)
        t0 = time.perf_counter()
        steps = 0
        while time.perf_counter() - t0 < seconds / 4 and steps < 50:
            n_before = float(po.moments(op)[0])
            po.advance(op, tabs[g], f, spec.dt, clamp=True)
            po.swarm_resample(op, int(spec.n[k]), 0.1)
            done_e += n_before
            steps += 1
        t_used += time.perf_counter() - t0
        ks.append((int(k), steps))
        if t_used > seconds:
            break
    rate = done_e / t_used
    solves = spec.k / (spec.steps * float(spec.n.sum()) / rate)
    return {"value": solves, "unit": BATCH_UNIT, "cores": threads, "kind": "port",
            "electron_steps_per_s": rate,
            "sample": f"oracle FP64 advance!+Swarm.resample! on instances {ks} (instance, steps); "
                      f"{done_e:.3g} electron steps in {t_used:.1f} s, scaled to {spec.k} solves x {spec.steps} steps"}


def _variant_int(fn: str, v: int) -> int:
    import ctypes as C

    from mcstreamer_b200 import _lib as L
    out = C.c_int(0)
    L.check(getattr(L.lib(), fn)(int(v), C.byref(out)))
    return out.value


def run_batch(args):
    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200 import jumc, lxcat, workloads
    from mcstreamer_b200.batch import SwarmBatch

    from mcstreamer_b200 import dist as mdist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    spec = workloads.batched_swarms()
    # instances are independent: each rank steps its share (dealt by predicted work), no
    # collective on the data path
    mine = mdist.my_instances((spec.n * spec.steps).tolist(), rank, ws)
    ctx = jumc.Context(local, clamp_energy=True)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    tables = {g: jumc.CollisionTable(lxcat.synthetic_table(g), ctx) for g in sorted(set(spec.gas.tolist()))}
    caps = 2 * spec.n
    ez = spec.en_td * spec.density * co.Td

    def fill(b, host: bool = False):
        """Join every instance: electrons drawn on the device, or (host=True) generated on
        the host and uploaded in the Julia layout.  Returns the host->device bytes."""
        nbytes = 0
        for k in mine:
            if host:
                p0 = workloads.swarm_instance_particles(spec, k)
                b.add(tables[int(spec.gas[k])], float(ez[k]), int(spec.seeds[k]), int(spec.n[k]), int(caps[k]), p0)
                nbytes += p0.n * (8 * 8 + 1)
            else:
                b.add_maxwellian(tables[int(spec.gas[k])], float(ez[k]), int(spec.seeds[k]), int(spec.n[k]),
                                 int(caps[k]), int(spec.n[k]), spec.mean_ev)
        return nbytes

    my_caps = int(caps[mine].sum())
    if args.cfg3_profile:
        b = SwarmBatch(ctx, len(mine), my_caps)
        if args.variant is not None:
            b.set_variant(args.variant)
        fill(b)
        b.step(spec.dt, args.warmup, graph=False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(spec.dt, args.steps, graph=False)
        e1.record(stream)
        b.sync()
        print(json.dumps({"workload": "cfg3 profile run", "variant": args.variant, "warmup": args.warmup,
                          "steps": args.steps, "ms_per_step": e0.elapsed_time(e1) / max(args.steps, 1)}), flush=True)
        b.close()
        return 0
    # autotune on a batch a few steps into the run, then a fresh batch for the timed solve
    b = SwarmBatch(ctx, len(mine), my_caps)
    fill(b)
    b.step(spec.dt, args.warmup, graph=True)
    chosen, times = b.autotune(spec.dt, trial_steps=2)
    shape = SwarmBatch.variant_shape(chosen)
    kernel_ms, prof_step_ms = b.profile(spec.dt, 3)
    b.close()
    # the timed region: every instance's whole solve, spec.steps batched steps from the 1 eV
    # Maxwellian start, in CUDA-graph chunks of 100 steps
    b = SwarmBatch(ctx, len(mine), my_caps)
    b.set_variant(chosen)
    fill(b)
    b.sync()
    n_start = float(spec.n[mine].sum())
    if dist is not None:
        dist.barrier()
    chunk = 100
    e_steps_sum = 0.0
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        done = 0
        while done < spec.steps:
            m = min(chunk, spec.steps - done)
            b.step(spec.dt, m, graph=True)
            done += m
        t1.record(stream)
        torch.cuda.synchronize()
    b.sync()
    solve_ms = t0.elapsed_time(t1)
    cur = b.read_current()
    n_end = float(cur[:, L.S_COUNT].sum())
    clocks = clk.summary()
    b.close()
    e_local = 0.5 * (n_start + n_end) * spec.steps
    if dist is not None:
        t = torch.tensor([solve_ms, e_local], device=f"cuda:{local}", dtype=torch.float64)
        mx, sm = t.clone(), t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        solve_ms, e_local = float(mx[0]), float(sm[1])
    step_ms = solve_ms / spec.steps
    value = spec.k / (solve_ms * 1e-3)
    e_steps = e_local / (solve_ms * 1e-3)
    if ws > 1:
        if rank == 0:
            print(json.dumps({
                "metric": BATCH_METRIC, "value": value, "unit": BATCH_UNIT, "n_gpus": ws, "steps": spec.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"batched swarms cfg3: {spec.k} instances dealt to {ws} ranks by predicted "
                                       f"work, {spec.steps} steps per solve", "parallelism": f"instances over {ws} GPUs",
                           "electron_steps_per_s": e_steps, "solve_time_s": solve_ms * 1e-3},
                "roofline": None, "cpu_baseline": None, "e2e": None, "clocks": clocks,
                "gpu_launches": spec.steps * 9}), flush=True)
        dist.barrier()
        dist.destroy_process_group()
        return 0

    # plain drop-in: each solve alone, all spec.steps steps, on a size-stratified sample (the
    # instances sorted by electron count, every `stride`-th); the serial time of all K is the
    # sample's total times the stride
    mom = np.zeros(L.MOMENTS_BASE)

    def plain(precision: str, ks, steps: int, calls: bool = False) -> float:
        """Total ms of the solves ks, each alone: the fused loop entry point, or (calls=True)
        the per-step call sequence of Swarm.jl:124-142 through the C ABI: advance!, the
        step sums, resample!, repack!."""
        t_ms = 0.0

        def run(pop, tab, fld, k, nsteps):
            if not calls:
                ctx.check(ctx.lib.mcs_swarm_run(pop.h, tab.h, fld.h, spec.dt, nsteps, int(spec.n[k]), 0.1, 1, None))
                return
            for _ in range(nsteps):
                ctx.check(ctx.lib.mcs_advance(pop.h, tab.h, fld.h, spec.dt, None))
                ctx.check(ctx.lib.mcs_moments(pop.h, None, L.dptr(mom), L.MOMENTS_BASE))
                ctx.check(ctx.lib.mcs_swarm_resample(pop.h, int(spec.n[k]), 0.1))
                ctx.check(ctx.lib.mcs_repack(pop.h))

        for k in ks:
            tab = tables[int(spec.gas[k])]
            pop = jumc.Population(int(caps[k]), None, tab, precision=precision, seed=int(spec.seeds[k]))
            pop.init_maxwellian(int(spec.n[k]), spec.mean_ev)
            fld = jumc.FixedField(float(ez[k]), ctx)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(pop, tab, fld, k, steps)
            e1.record(stream)
            torch.cuda.synchronize()
            t_ms += e0.elapsed_time(e1)
            fld.close()
            pop.close()
        return t_ms

    by_size = np.argsort(spec.n, kind="stable")
    s32, s_calls, s64 = args.plain_stride, 4 * args.plain_stride, 4 * args.plain_stride
    k32 = by_size[s32 // 2::s32]
    kc = by_size[s_calls // 2::s_calls]
    k64 = by_size[s64 // 2::s64]
    t32 = plain("fp32", k32, spec.steps) * s32
    t32c = plain("fp32", kc, spec.steps, calls=True) * s_calls
    t64 = plain("fp64", k64, spec.steps) * s64
    plain32, plain32c, plain64 = (spec.k / (t * 1e-3) for t in (t32, t32c, t64))

    # end to end through the public API: host particles uploaded into a fresh batch, steps,
    # and every step the sums of all instances read back to the host
    e2e_steps = max(3, min(args.steps, 20))
    b2 = SwarmBatch(ctx, spec.k, int(caps.sum()))
    b2.set_variant(chosen)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    up_bytes = fill(b2, host=True)
    t_up = time.perf_counter() - t0
    b2.step(spec.dt, 1, graph=True)
    b2.read_current()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        b2.step(spec.dt, 1, graph=True)
        b2.read_current()
    t_steps = (time.perf_counter() - t1) / e2e_steps
    b2.close()
    e2e_solves = spec.k / (t_up + spec.steps * t_steps)

    # the batched FP32 form's error against FP64 runs of the same swarms (gas 0, three E/N)
    from mcstreamer_b200 import swarm as mswarm
    acc = {}
    for en, r in mswarm.fp32_batched_vs_fp64(ctx, tables[0], (100.0, 300.0, 1000.0), spec.density, 131072,
                                             spec.steps, 1000, spec.dt).items():
        acc[f"{en:g} Td"] = {
            key: {"fp32": a32, "fp64": a64, "rel_diff": (a32 - a64) / a64 if a64 else None,
                  "combined_3sigma_rel": float(np.hypot(e32, e64) / abs(a64)) if a64 else None}
            for key, (a32, e32, a64, e64) in r.items()}

    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    alg = batch_alg_bytes(0.5 * (n_start + n_end), 0.0)
    achieved = alg / (kernel_ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu:
        cpu = batch_cpu_sample(spec, args.cpu_seconds, os.cpu_count() or 1)
    # DRAM bytes of one launch from the committed ncu record of the autotuner's usual variant
    # (per entering electron, times this batch's), while the kernel's sources are unchanged
    brec = profile_record("traffic_k_bstep_cfg3")
    btraffic = btraffic_src = None
    if brec and not brec.get("stale") and brec.get("electrons") and chosen == 19:
        btraffic = brec["bytes_per_launch"] / brec["electrons"] * float(spec.n.sum())
        btraffic_src = "profiles/traffic_k_bstep_cfg3.json (one launch of variant 19, ncu --set full)"
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": BATCH_UNIT, "n_gpus": 1, "steps": spec.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": f"batched swarms cfg3: {spec.k} instances, E/N log-spaced 10-1000 Td, electrons "
                        f"log-uniform 4096-1048576 (total {int(spec.n.sum())}), synthetic gases 0/1/2, "
                        f"N={spec.density:g} m^-3, dt={spec.dt:g} s, {spec.steps} steps per solve, Swarm.resample! "
                        f"to the initial count every step, repack every step, one CUDA graph per batched step",
            "solve_time_s": solve_ms * 1e-3,
            "timing": f"CUDA events around the whole solve of all {spec.k} instances ({spec.steps} batched steps "
                      "from a fresh batch, CUDA graphs of 100 steps); autotuned on a separate batch",
            "electron_steps_per_s": e_steps,
            "autotune": {"variant": chosen, "block": shape[0], "particles_per_thread": shape[1],
                         "ctas_per_sm_bound": _variant_int("mcs_batch_variant_min_blocks", chosen),
                         "refill_idle_lanes": _variant_int("mcs_batch_variant_refill", chosen),
                         "trial_ms": [round(float(t), 4) for t in times]},
            "l2": "inputs larger than L2 (44.6M electrons x 33 B = 1.5 GB resident)",
            "fp32_vs_fp64": {"how": f"batched FP32 against independent FP64 runs (mcs_swarm_run), 131072 "
                                    f"electrons from a 1 eV Maxwellian, gas 0, steps 1000-{spec.steps}, batch-means "
                                    "errors; W = drift (m/s), E = mean energy (eV), k = ionization rate (m^3/s)",
                             "results": acc},
            "plain_drop_in": {
                "fp32_solves_per_s": plain32, "fp32_serial_s": t32 * 1e-3,
                "fp32_calls_solves_per_s": plain32c, "fp32_calls_serial_s": t32c * 1e-3,
                "speedup_fp32_calls": value / plain32c,
                "fp64_solves_per_s": plain64, "fp64_serial_s": t64 * 1e-3,
                "samples": {"fp32": len(k32), "fp32_calls": len(kc), "fp64": len(k64)},
                "how": f"each solve alone for all {spec.steps} steps from the same start: "
                       "mcs_swarm_run(FP32|FP64, repack_every=1), and (fp32_calls) the per-step ccall sequence "
                       "mcs_advance + mcs_moments + mcs_swarm_resample + mcs_repack; measured on the instances "
                       f"sorted by electron count, every {s32}th (fp32) / {s_calls}th (calls, fp64), and scaled "
                       "by that stride; CUDA events around each solve",
                "speedup_fp32": value / plain32, "speedup_fp64": value / plain64},
            "parallelism": "1 GPU",
        },
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": btraffic, "traffic_source": btraffic_src,
                     "kernel": f"k_bstep<{shape[0]},{shape[1]}>", "kernel_ms": kernel_ms,
                     "step_ms_no_graph": prof_step_ms, "alg_bytes_per_launch": alg,
                     "peak_source": f"{pk_kind} (MEASURED_PEAKS.json hbm_gbs)"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_solves, "unit": BATCH_UNIT,
                "h2d_bytes_per_step": up_bytes / spec.steps, "d2h_bytes_per_step": spec.k * L.BATCH_MOMENTS * 8,
                "path": "SwarmBatch.add from host arrays (Julia layout, uploaded once per solve; h2d bytes "
                        "amortised over the solve's steps) -> SwarmBatch.step -> read_current every step",
                "upload_s": t_up, "ms_per_step": t_steps * 1e3},
        "clocks": clocks,
        "gpu_launches": spec.steps * 9,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# Served swarm requests ("cfg4"): Poisson arrivals, continuous batching, memory admission.
# ---------------------------------------------------------------------------------------
SERVE_METRIC = "served swarm solves/s"


def run_serve(args):
    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import constants as co
    from mcstreamer_b200 import jumc, lxcat
    from mcstreamer_b200.serve import StopRule, SwarmServer, percentiles, poisson_requests
    from mcstreamer_b200.workloads import SWARM_DENSITY, SWARM_DT

    from mcstreamer_b200 import dist as mdist

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    ctx = jumc.Context(local, clamp_energy=True)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    tables = [jumc.CollisionTable(lxcat.synthetic_table(v), ctx) for v in (0, 1, 2, 3)]
    rule = StopRule()
    # warm the kernels, the graph and the allocator on a throw-away request
    warm = SwarmServer(ctx, tables, SWARM_DT, SWARM_DENSITY, budget_bytes=1e9, rule=rule)
    warm.run(poisson_requests(200.0, 0.02, seed=99, n_range=(1024, 4096)), realtime=False)
    warm.close()

    def serve(rate: float, seconds: float, seed: int, limit: float):
        reqs = poisson_requests(rate, seconds, seed=seed)
        # several GPUs: each serves its share of the arrivals (dealt online by predicted work)
        mine = mdist.shard_requests(reqs, rank, ws)
        srv = SwarmServer(ctx, tables, SWARM_DT, SWARM_DENSITY, budget_bytes=160e9, rule=rule)
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        got = srv.run(mine, deadline=limit)
        wall = time.perf_counter() - t0
        unfinished, gpu_steps, pool = srv.unfinished, srv.gpu_steps, srv.pool_slots
        srv.close()
        if dist is not None:
            parts = [None] * ws
            dist.all_gather_object(parts, (got, unfinished, wall, gpu_steps))
            got = sorted((r for p in parts for r in p[0]), key=lambda r: r.rid)
            unfinished = sum(p[1] for p in parts)
            wall = max(p[2] for p in parts)
            gpu_steps = max(p[3] for p in parts)
        info = {"rate": rate, "seconds": seconds, "requests": len(reqs), "completed": len(got),
                "unfinished_at_limit": unfinished, "wall_s": wall, "gpu_steps": gpu_steps,
                "pool_slots": pool}
        makespan = max(r.finished for r in got) if got else wall
        info["solves_per_s"] = len(got) / makespan if makespan > 0 else 0.0
        info["latency_s"] = percentiles([r.latency for r in got])
        info["electron_steps"] = float(sum(r.n * r.steps for r in got))
        info["settled"] = sum(1 for r in got if r.settled)
        # keeps up: every request answered and the last one no later than 10 % after the
        # arrival window closed
        info["keeps_up"] = bool(unfinished == 0 and makespan <= 1.1 * seconds)
        return reqs, got, info

    with ClockSampler(local) as clk:
        reqs, got, main = serve(args.serve_rate, args.serve_seconds, 4, args.serve_limit)
    clocks = clk.summary()
    sustained = None
    if not main["keeps_up"] and main["solves_per_s"] > 0:
        # the highest arrival rate it sustains: 80 % of the throughput measured under overload
        rate2 = 0.8 * main["solves_per_s"]
        _, _, sustained = serve(rate2, args.serve_seconds, 5, args.serve_limit)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    # the plain drop-in, one request at a time, on a seeded sample of the served requests:
    # per step mcs_advance + mcs_moments (with the table: the rate estimator) +
    # mcs_swarm_resample + mcs_repack for the request's own stopping step count (a request's
    # steps are the same alone and in the mix); its rate estimate is checked against the
    # served one
    rng = np.random.default_rng(17)
    pick = sorted(rng.choice(len(got), size=min(args.serve_sample, len(got)), replace=False).tolist())
    by_id = {r.rid: r for r in reqs}
    t_serial, n_match, rows = 0.0, 0, []
    for i in pick:
        g = got[i]
        q = by_id[g.rid]
        tab = tables[q.gas]
        ion = [j for j, p in enumerate(tab.proc) if p.kind in (L.IONIZATION, L.IONIZATION_UNIFORM)][0]
        mom = np.zeros(L.MOMENTS_BASE + len(tab))
        pop = jumc.Population(max(64, 2 * q.n), None, tab, precision="fp32", seed=q.seed)
        pop.init_maxwellian(q.n, q.mean_ev)
        fld = jumc.FixedField(q.en_td * SWARM_DENSITY * co.Td, ctx)
        nu = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(g.steps):
            ctx.check(ctx.lib.mcs_advance(pop.h, tab.h, fld.h, SWARM_DT, None))
            ctx.check(ctx.lib.mcs_moments(pop.h, tab.h, L.dptr(mom), len(mom)))
            nu.append(mom[L.MOMENTS_BASE + ion] / max(mom[L.M_COUNT], 1.0))
            ctx.check(ctx.lib.mcs_swarm_resample(pop.h, q.n, 0.1))
            ctx.check(ctx.lib.mcs_repack(pop.h))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        t_serial += dt
        k, err = rule.stats(np.asarray(nu))
        k /= SWARM_DENSITY
        same = abs(k - g.k_ion) <= 1e-9 * max(abs(g.k_ion), 1e-300)
        n_match += int(same)
        rows.append({"rid": g.rid, "n": q.n, "steps": g.steps, "serial_s": dt, "k_ion_served": g.k_ion,
                     "k_ion_alone": k})
        fld.close()
        pop.close()
    serial_rate = len(pick) / t_serial if t_serial > 0 else 0.0
    value = main["solves_per_s"]
    line = {
        "metric": SERVE_METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": main["gpu_steps"],
        "warmup": 1, "ms_per_step": 1e3 * main["wall_s"] / max(1, main["gpu_steps"]), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": f"served swarms cfg4: Poisson arrivals {args.serve_rate:g} req/s over {args.serve_seconds:g} s, "
                        f"gases 0-3, E/N log-uniform 10-1000 Td, electrons log-uniform 1024-2097152, stop at 3 sigma "
                        f"<= 1% of k_ion (batch means, blocks of {rule.block}, after {rule.min_steps} relaxation "
                        f"steps, at most {rule.max_steps} steps), 160 GB budget, seed 4",
            "at_configured_rate": main,
            "keeps_up_with_arrivals": main["keeps_up"],
            "sustained_rate_run": sustained,
            "plain_serial": {"solves_per_s": serial_rate, "speedup": value / serial_rate if serial_rate else None,
                             "sample": len(pick), "results_equal_alone_and_served": n_match,
                             "how": "a seeded sample of the served requests, each alone through the per-step "
                                    "C-ABI sequence (mcs_advance, mcs_moments with the table, mcs_swarm_resample, "
                                    "mcs_repack) for its stopping step count; solves/s = sample / total time. A "
                                    "serial server's queue at the configured rate grows without bound",
                             "requests": rows},
            "parallelism": f"requests dealt over {ws} GPUs" if ws > 1 else "1 GPU",
        },
        "roofline": None,
        "cpu_baseline": None,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "path": "SwarmServer.run: host requests -> SwarmBatch.add -> graph steps -> read_logs every "
                        "chunk -> responses; the value is end to end by construction"},
        "clocks": clocks,
        "gpu_launches": main["gpu_steps"] * 9,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


POISSON_METRIC = "poisson solves/s"


def poisson_alg_bytes_tile(M: int, N: int) -> float:
    """Algorithmic HBM bytes of one fused post-smoothing launch over M x N cells: the level's
    solution and right-hand side read once (8 + 8 B per cell), the next coarser solution
    read once (2 B per fine cell) and the smoothed solution written once (8 B per cell)."""
    return 26.0 * M * N


def poisson_alg_bytes_gs(M: int, N: int) -> float:
    """Algorithmic HBM bytes of one red-black pass over M x N cells: the potential read
    once (8 B per cell: every cell is a neighbour of the updated colour), the right-hand
    side and the write of the updated half (4 + 4 B per cell)."""
    return 16.0 * M * N


def poisson_oracle_call(spec, qf, qp, threads):
    """One poisson! of the CPU restatement from a zero potential; returns (seconds, iters)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import poisson_ref as P
    u = P.cells(spec.M, spec.N)
    er, ez = P.faces(spec.M, spec.N), P.faces(spec.M, spec.N)
    conf = P.default_conf(spec.R, spec.L, spec.M, spec.N, levels=spec.levels)
    t0 = time.perf_counter()
    _, it1, it2, _ = P.poisson(conf, qf, qp, u, er, ez, spec.eb, spec.R, spec.L)
    return time.perf_counter() - t0, (it1, it2)


def poisson_inputs(spec):
    from mcstreamer_b200 import workloads
    p = workloads.poisson_electrons(spec)
    qf = workloads.poisson_ion_charge(spec)
    qp = workloads.poisson_electron_charge(spec, p.x, p.w)
    return p, qf, qp


def poisson_config(spec, extra=None):
    c = {"workload": f"poisson! on the sample grid: R={spec.R:g} m, L={spec.L:g} m, {spec.M}x{spec.N} cells, "
                     f"{spec.levels} multigrid levels, tolerance 1e8 e, smoothing 2+2, free b.c. at r=R; "
                     f"{spec.n} channel electrons of weight {spec.weight:g} deposited each call (density!), "
                     f"analytic ion charge, eb={spec.eb:g} V/m, cold start (u = 0), seed {spec.seed}",
         "cells": spec.M * spec.N, "l2": "working set (u, q, 3 finest workspace levels: 630 MB) exceeds L2",
         "parallelism": "1 GPU"}
    if extra:
        c.update(extra)
    return c


def run_poisson(args):
    import ctypes as C

    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import jumc, lxcat, streamer, workloads
    from mcstreamer_b200.poisson import MGConfig, PoissonSolver

    ws, rank, local = dist_env()
    if ws > 1:
        # replicas only: the solve is not sharded
        import torch.distributed as dist
        dist.init_process_group("nccl")
    torch.cuda.set_device(local)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spec = workloads.poisson_spec()
    parts, qf, qp_host = poisson_inputs(spec)
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.GridCyl(spec.R, spec.L, spec.M, spec.N, ctx=ctx)
    pop = jumc.Population(spec.n, parts, tab, precision="fp64")
    solver = PoissonSolver(grid, MGConfig(levels=spec.levels))
    grid.write_fixed(L.Q_FIXED, qf)
    lib = ctx.lib

    def step():
        ctx.check(lib.mcs_grid_zero(grid.h_, L.Q_PART))
        ctx.check(lib.mcs_deposit(pop.h, grid.h_, -1.0))
        it = (C.c_int * 2)()
        ctx.check(lib.mcs_poisson_run(solver.h, spec.eb, it))
        return it[0], it[1]

    iters = []
    for _ in range(args.warmup):
        solver.zero(L.PSN_U)
        iters.append(step())
    assert np.array_equal(grid.read_fixed(L.Q_PART), qp_host), "device density! differs from the host restatement"
    n0 = C.c_int64(0)
    ctx.check(lib.mcs_poisson_launches(solver.h, C.byref(n0)))
    times = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        for _ in range(args.steps):
            solver.zero(L.PSN_U)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            iters.append(step())
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    n1 = C.c_int64(0)
    ctx.check(lib.mcs_poisson_launches(solver.h, C.byref(n1)))
    total_ms = float(sum(times))
    if ws > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = ws * 1e3 / ms
    gs_ms, res_ms, tile_ms = solver.profile(20)
    pk, src = peaks()
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    ach = poisson_alg_bytes_tile(spec.M, spec.N) / (tile_ms * 1e-3) / 1e9

    # end to end: host int64 charges in, host face fields out, pinned buffers
    nq = (spec.M + 2) * (spec.N + 2)
    nf = 2 * (spec.M + 3) * (spec.N + 3)
    h_qf = torch.from_numpy(qf).pin_memory()
    h_qp = torch.from_numpy(qp_host).pin_memory()
    h_e = torch.empty(nf, dtype=torch.float64).pin_memory()
    pi64 = C.POINTER(C.c_int64)
    pd = C.POINTER(C.c_double)
    e2e_t = []
    for k in range(max(1, args.e2e_steps) + 1):
        solver.zero(L.PSN_U)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.check(lib.mcs_grid_write_fixed(grid.h_, L.Q_FIXED, C.cast(h_qf.data_ptr(), pi64)))
        ctx.check(lib.mcs_grid_write_fixed(grid.h_, L.Q_PART, C.cast(h_qp.data_ptr(), pi64)))
        it = (C.c_int * 2)()
        ctx.check(lib.mcs_poisson_run(solver.h, spec.eb, it))
        ctx.check(lib.mcs_grid_read_efield(grid.h_, C.cast(h_e.data_ptr(), pd)))
        if k:
            e2e_t.append(time.perf_counter() - t0)
    e2e_v = 1.0 / statistics.median(e2e_t)

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sec, it_cpu = poisson_oracle_call(spec, qf, qp_host, threads)
        cpu = {"value": 1.0 / sec, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"one full poisson! (this workload) by the oracle on {threads} threads: {sec:.2f} s, "
                         f"fmg! calls {it_cpu}"}
    launches = int((n1.value - n0.value) / args.steps)
    it_set = sorted({tuple(i) for i in iters})
    line = {
        "metric": POISSON_METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": poisson_config(spec, {"fmg_calls_per_solve": it_set}),
        "roofline": {"kernel": "k_smooth_tile<2, TILE_POST> (interpolation + 2 red-black sweeps, finest level)",
                     "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": profiled_traffic("k_smooth_tile_post_sample_grid"), "peak_source": src, "launch_ms": tile_ms,
                     "alg_bytes_per_launch": poisson_alg_bytes_tile(spec.M, spec.N),
                     "unfused_k_gs_launch_ms": gs_ms,
                     "unfused_k_gs_gbs": poisson_alg_bytes_gs(spec.M, spec.N) / (gs_ms * 1e-3) / 1e9,
                     "residual_norm_launch_ms": res_ms},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "solves/s", "h2d_bytes_per_step": 2 * nq * 8, "d2h_bytes_per_step": nf * 8,
                "path": "mcs_grid_write_fixed (qfixed, qpart from pinned host) -> mcs_poisson_run -> "
                        "mcs_grid_read_efield (er, ez to pinned host)"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close(); pop.close(); grid.close(); tab.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_poisson(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.poisson_spec()
    _, qf, qp = poisson_inputs(spec)
    threads = os.cpu_count() or 1
    runs = [poisson_oracle_call(spec, qf, qp, threads) for _ in range(max(1, min(args.steps, 3)))]
    sec = statistics.median(r[0] for r in runs)
    v = 1.0 / sec
    line = {
        "impl": "reference", "metric": POISSON_METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": len(runs), "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": poisson_config(spec),
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{len(runs)} full poisson! calls of the oracle, fmg! calls {runs[0][1]}"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


PHOTON_METRIC = "electron and photon steps/s"
PHOTON_SAMPLE = (1_048_576, 262_144)   # CPU sample: electrons, photons


def photon_alg_bytes(n_photons: float) -> float:
    """Algorithmic HBM bytes of one photon step over n photons: each photon read once
    (x, v 48 B, nu, w, s 24 B, active 1 B) and written once (x 24 B, s 8 B, active 1 B, its
    photo-ionization count 4 B)."""
    return n_photons * (73.0 + 37.0)


def photon_setup_table():
    from mcstreamer_b200 import lxcat, workloads
    spec = workloads.photon_step_spec()
    t = lxcat.synthetic_photo_table(0, photon_multiplier=spec.photon_multiplier, photon_weight=spec.photon_weight)
    j = list(t.kinds).index(6)
    return spec, t, float(t.pe_lmin[j]), float(t.pe_lmax[j])


def photon_cpu_sample(threads: int) -> dict:
    """advance! over electrons and photons by the oracle on a bounded sample of the workload."""
    from mcstreamer_b200 import workloads
    from oracle import pyoracle as po
    spec, t, lmin, lmax = photon_setup_table()
    ne, nph = PHOTON_SAMPLE
    e = workloads.photon_step_electrons(spec, ne)
    x, v, nu, w, s, act = workloads.photon_step_photons(spec, lmin, lmax, nph)
    opop = po.OraclePop(e.x, e.v, e.w, e.s, e.active, cap=3 * ne, seed=spec.seed)
    oph = po.OraclePhotons(nph + ne, t.photon_numax, seed=spec.seed + 2, x=x, v=v, nu=nu, w=w, s=s, active=act)
    otab = po.OracleTable.from_lxcat(t)
    otrk = po.tracker_cyl(spec.R, spec.L, spec.M, spec.N)
    t0 = time.perf_counter()
    po.advance_mixed(opop, oph, otab, po.field_uniform(0.0, 0.0, spec.ez), spec.dt, otrk, threads=threads)
    sec = time.perf_counter() - t0
    return {"value": (ne + nph) / sec, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": f"one mixed step of {ne} electrons and {nph} photons of this workload (FP64 oracle, "
                      f"uniform field, cyl tracker): {sec:.2f} s"}


def photon_config(spec, extra=None):
    c = {"workload": f"advance! over electrons and photons: cyl grid R={spec.R:g} m, L={spec.L:g} m, "
                     f"{spec.M}x{spec.N} cells, face field ez={spec.ez:g} V/m (FieldInterp), tracker on; "
                     f"{spec.n_e} electrons (FP32, w={spec.weight:g}, 5 eV Maxwellian, Gaussian cloud sigma "
                     f"{spec.sigma:g} m) and {spec.n_ph} photons (FP64) restored before every step; synthetic gas 0 "
                     f"+ photo-emission (photon_multiplier {spec.photon_multiplier:g}, photon_weight "
                     f"{spec.photon_weight:g}); dt={spec.dt:g} s, seed {spec.seed}",
         "l2": "particle state (4.2M x 33 B + 1M x 73 B) exceeds L2", "parallelism": "1 GPU"}
    if extra:
        c.update(extra)
    return c


def run_photons(args):
    import ctypes as C

    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import jumc, streamer, workloads

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl")
    torch.cuda.set_device(local)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spec, t, lmin, lmax = photon_setup_table()
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(spec.R, spec.L, spec.M, spec.N, ctx=ctx)
    er = np.zeros((spec.M + 3, spec.N + 3))
    grid.set_efield(er, np.full_like(er, spec.ez))
    fld = streamer.FieldInterp(grid)
    trk = streamer.CollisionTracker(grid)
    parts = workloads.photon_step_electrons(spec)
    ph0 = jumc.PhotonArrays(*workloads.photon_step_photons(spec, lmin, lmax))
    snap_e = jumc.Population(spec.n_e, parts, tab, precision="fp32", seed=spec.seed + 100 * rank)
    pop = jumc.Population(4 * spec.n_e, None, tab, precision="fp32", seed=spec.seed + 100 * rank)
    snap_p = jumc.Photons(spec.n_ph, t.photon_numax, seed=spec.seed + 2, ctx=ctx, photons=ph0)
    phs = jumc.Photons(8 * spec.n_ph, t.photon_numax, seed=spec.seed + 2, ctx=ctx)
    lib = ctx.lib

    def restore():
        ctx.check(lib.mcs_pop_copy(pop.h, snap_e.h))
        ctx.check(lib.mcs_photons_copy(phs.h, snap_p.h))

    def step():
        ctx.check(lib.mcs_advance_mixed(pop.h, phs.h, tab.h, fld.h, spec.dt, trk.h))

    grid.zero(L.Q_FIXED)
    for _ in range(args.warmup):
        restore()
        step()
    torch.cuda.synchronize()
    times, emitted, ph_ms, ph_n, e_after = [], [], [], [], []
    with ClockSampler(local) as clk:
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            em, ne_, sm, ns = C.c_float(), C.c_int64(), C.c_float(), C.c_int64()
            ctx.check(lib.mcs_photons_last_timing(phs.h, C.byref(em), C.byref(ne_), C.byref(sm), C.byref(ns)))
            emitted.append(ne_.value)
            ph_ms.append(sm.value)
            ph_n.append(ns.value)
        torch.cuda.synchronize()
    total_ms = float(sum(times))
    if ws > 1:
        tt = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms = total_ms / args.steps
    n_part = spec.n_e + spec.n_ph
    value = ws * n_part * 1e3 / ms
    pk, src = peaks()
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    step_ms = statistics.median(ph_ms)
    n_step = statistics.median(ph_n)
    ach = photon_alg_bytes(n_step) / (step_ms * 1e-3) / 1e9 if step_ms > 0 else 0.0

    # end to end: both populations uploaded from host arrays (Julia layout) into the
    # workspaces, the mixed step, both downloaded
    e2e_t, d2h = [], 0
    for k in range(max(1, args.e2e_steps) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pop.upload(parts)
        phs.upload(ph0)
        ctx.check(lib.mcs_advance_mixed(pop.h, phs.h, tab.h, fld.h, spec.dt, trk.h))
        out_e, out_p = pop.download(), phs.download()
        dt_ = time.perf_counter() - t0
        d2h = out_e.n * (8 * 8 + 1) + len(out_p.w) * (10 * 8 + 1)
        if k:
            e2e_t.append(dt_)
    e2e_v = n_part / statistics.median(e2e_t)
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = photon_cpu_sample(os.cpu_count() or 1)
    line = {
        "metric": PHOTON_METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 electrons, f64 photons", "data": "synthetic",
        "config": photon_config(spec, {"photons_emitted_per_step": int(statistics.median(emitted)),
                                       "photons_stepped_per_step": int(n_step),
                                       "electron_steps_per_s": ws * spec.n_e * 1e3 / ms}),
        "roofline": {"kernel": "k_photon_step (photon flight + photo-ionization)", "bound": "hbm",
                     "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm, "traffic": None,
                     "peak_source": src, "launch_ms": step_ms, "alg_bytes_per_launch": photon_alg_bytes(n_step)},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "particle-steps/s",
                "h2d_bytes_per_step": spec.n_e * (8 * 8 + 1) + spec.n_ph * (10 * 8 + 1),
                "d2h_bytes_per_step": d2h,
                "path": "mcs_pop_upload + mcs_photons_upload (host arrays) -> mcs_advance_mixed -> "
                        "mcs_pop_download + mcs_photons_download"},
        "clocks": clk.summary(),
        # k_step_abs, 3 scan kernels, k_photon_emit, k_photon_step, 3 scan kernels,
        # k_ion_scatter, k_set_count
        "gpu_launches": 11,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    fld.close(); trk_close = getattr(trk, "close", None)
    if trk_close:
        trk_close()
    phs.close(); snap_p.close(); pop.close(); snap_e.close(); grid.close(); tab.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_photons(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.photon_step_spec()
    threads = os.cpu_count() or 1
    runs = [photon_cpu_sample(threads) for _ in range(max(1, min(args.steps, 3)))]
    v = statistics.median(r["value"] for r in runs)
    line = {
        "impl": "reference", "metric": PHOTON_METRIC, "value": v, "unit": "particle-steps/s", "n_gpus": args.gpus,
        "steps": len(runs), "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": photon_config(spec),
        "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": runs[-1]["sample"]},
        "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batch(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.batched_swarms()
    threads = os.cpu_count() or 1
    per = min(20.0, max(4.0, 120.0 / max(1, args.steps + args.warmup)))
    vals = [batch_cpu_sample(spec, per, threads) for _ in range(max(1, min(args.steps, 3)))]
    v = statistics.median(x["value"] for x in vals)
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": v, "unit": BATCH_UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched swarms cfg3", "instances": spec.k, "electrons": int(spec.n.sum())},
        "cpu_baseline": {"value": v, "unit": BATCH_UNIT, "cores": threads, "kind": "port", "sample": vals[-1]["sample"]},
        "e2e": {"value": v, "unit": BATCH_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


FLUID_METRIC = "fluid cell updates/s"


def fluid_alg_bytes(M: int, N: int) -> float:
    """Algorithmic HBM bytes of one fused setdne! + euler! over the (M+4) x (N+4) padded
    cells: ne, er and ez read once (8 + 8 + 8 B per cell), dne and the updated ne written
    once (8 + 8 B per cell)."""
    return 40.0 * (M + 4) * (N + 4)


def fluid_config(spec, extra=None):
    p = spec.poisson
    c = {"workload": f"setdne! + euler! of the electron fluid on the sample grid: R={p.R:g} m, L={p.L:g} m, "
                     f"{p.M}x{p.N} cells; fluid where a channel of peak density {spec.peak:g} m^-3 (Gaussian in "
                     f"r, sigma {p.sigma_r:g} m, z in [{p.z0:g}, {p.z1:g}] m) exceeds {spec.threshold:g} m^-3 "
                     f"(fluid_threshold); faces from one poisson! of the channel charge (eb={p.eb:g} V/m), "
                     f"mobility 1e24/nair, dt={spec.dt:g} s",
         "cells": p.M * p.N, "l2": "ne, dne and the face fields (500 MB) exceed L2", "parallelism": "1 GPU"}
    if extra:
        c.update(extra)
    return c


def fluid_oracle_step(spec, ne, er, ez):
    """One setdne! + euler! of the oracle on all host threads; returns seconds."""
    from oracle import fluid_ref as F
    p = spec.poisson
    dne = F.centers(p.M, p.N)
    t0 = time.perf_counter()
    F.setdne(ne, dne, er, ez, p.R, p.L, p.M, p.N)
    F.euler(ne, dne, spec.dt, p.M, p.N)
    return time.perf_counter() - t0


def fluid_faces(spec):
    """The face fields of one poisson! of the channel charge, computed by the oracle (for the
    CPU arms, which have no device)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    from oracle import poisson_ref as P
    p = spec.poisson
    _, qf, qp = poisson_inputs(p)
    u = P.cells(p.M, p.N)
    er, ez = P.faces(p.M, p.N), P.faces(p.M, p.N)
    P.poisson(P.default_conf(p.R, p.L, p.M, p.N, levels=p.levels), qf, qp, u, er, ez, p.eb, p.R, p.L)
    return er, ez


def profiled_traffic(name: str):
    """DRAM bytes per launch from a committed ncu summary (profiles/traffic_<name>.json)."""
    f = ROOT / "profiles" / f"traffic_{name}.json"
    return json.loads(f.read_text()).get("bytes_per_launch") if f.exists() else None


def run_fluid(args):
    import ctypes as C

    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import jumc, lxcat, streamer, workloads
    from mcstreamer_b200.fluid import MOBILITY, Fluid
    from mcstreamer_b200.poisson import MGConfig, PoissonSolver, read_faces

    ws, rank, local = dist_env()
    if ws > 1:
        # replicas only: the fluid step is not sharded
        import torch.distributed as dist
        dist.init_process_group("nccl")
    torch.cuda.set_device(local)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spec = workloads.fluid_spec()
    p = spec.poisson
    parts, qf, _ = poisson_inputs(p)
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.GridCyl(p.R, p.L, p.M, p.N, ctx=ctx)
    pop = jumc.Population(p.n, parts, tab, precision="fp64")
    solver = PoissonSolver(grid, MGConfig(levels=p.levels))
    grid.write_fixed(L.Q_FIXED, qf)
    grid.zero(L.Q_PART)
    streamer.density(grid, pop, -1.0)
    solver.run(p.eb)
    pop.close(); tab.close()
    ne0 = workloads.fluid_density(spec)
    fl = Fluid(grid)
    fl.upload(ne=ne0)
    lib = ctx.lib
    for _ in range(args.warmup):
        ctx.check(lib.mcs_fluid_step(fl.h, MOBILITY, spec.dt))
    n0 = fl.launches()
    times = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.mcs_fluid_step(fl.h, MOBILITY, spec.dt))
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
    times = [a.elapsed_time(b) for a, b in times]
    launches = (fl.launches() - n0) // args.steps
    total_ms = float(sum(times))
    if ws > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = ws * p.M * p.N / (ms * 1e-3)
    pk, src = peaks()
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    ach = fluid_alg_bytes(p.M, p.N) / (ms * 1e-3) / 1e9

    # end to end: ne from pinned host, the step, ne and dne back to pinned host
    npad = (p.M + 4) * (p.N + 4)
    h_ne = torch.from_numpy(np.ascontiguousarray(ne0.ravel(order="F"))).pin_memory()
    h_out = torch.empty(2 * npad, dtype=torch.float64).pin_memory()
    pd = C.POINTER(C.c_double)
    e2e_t = []
    for k in range(max(1, args.e2e_steps) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.check(lib.mcs_fluid_upload(fl.h, C.cast(h_ne.data_ptr(), pd), None))
        ctx.check(lib.mcs_fluid_step(fl.h, MOBILITY, spec.dt))
        ctx.check(lib.mcs_fluid_download(fl.h, C.cast(h_out.data_ptr(), pd),
                                         C.cast(h_out.data_ptr() + 8 * npad, pd), None))
        if k:
            e2e_t.append(time.perf_counter() - t0)
    e2e_v = p.M * p.N / statistics.median(e2e_t)

    cpu = None
    if rank == 0 and not args.no_cpu:
        er, ez = read_faces(grid)
        ne = ne0.copy(order="F")
        sec = fluid_oracle_step(spec, ne, np.asfortranarray(er), np.asfortranarray(ez))
        cpu = {"value": p.M * p.N / sec, "unit": "cell-updates/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"one setdne! + euler! of this workload by the oracle (OpenMP over the inner "
                         f"index, as the reference's @batch): {sec:.2f} s"}
    line = {
        "metric": FLUID_METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": fluid_config(spec, {"fluid_cells": int((ne0 > 0).sum())}),
        "roofline": {"kernel": "k_fluid<true> (setnebc! + setdne! + euler!, one launch)", "bound": "hbm",
                     "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": profiled_traffic("k_fluid_sample_grid"),
                     "peak_source": src, "launch_ms": ms, "alg_bytes_per_launch": fluid_alg_bytes(p.M, p.N)},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "cell-updates/s", "h2d_bytes_per_step": 8 * npad,
                "d2h_bytes_per_step": 16 * npad,
                "path": "mcs_fluid_upload (ne from pinned host) -> mcs_fluid_step -> mcs_fluid_download "
                        "(ne, dne to pinned host)"},
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    fl.close(); solver.close(); grid.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_fluid(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.fluid_spec()
    p = spec.poisson
    er, ez = fluid_faces(spec)
    ne = workloads.fluid_density(spec)
    runs = [fluid_oracle_step(spec, ne, er, ez) for _ in range(max(1, min(args.steps, 3)))]
    sec = statistics.median(runs)
    v = p.M * p.N / sec
    line = {
        "impl": "reference", "metric": FLUID_METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": len(runs), "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": fluid_config(spec),
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": f"{len(runs)} setdne! + euler! steps of the oracle (OpenMP over the inner "
                                   f"index, as the reference's @batch)"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


INIT_METRIC = "initfromfiles! electrons/s"


def init_alg_bytes(cells: int, electrons: int, esz: int) -> float:
    """Algorithmic HBM bytes of one initfromfiles!: ne and q read once (16 B per cell),
    qfixed's density part written (8 B per cell), each electron's x, v, w, s written (8 values
    of esz bytes) and its active flag (1 B).  The two-pass implementation also moves the
    counts and bases and reads ne and q twice; the ncu traffic shows that excess."""
    return cells * (16.0 + 8.0) + electrons * (8.0 * esz + 1.0)


def init_config(spec, extra=None):
    f = spec.fluid
    p = f.poisson
    c = {"workload": f"initfromfiles!(PoissonInitSampling({spec.p}), ...) on the sample grid: R={p.R:g} m, "
                     f"L={p.L:g} m, {p.M}x{p.N} cells; ne a channel of peak {f.peak:g} m^-3 (Gaussian in r, sigma "
                     f"{p.sigma_r:g} m, z in [{p.z0:g}, {p.z1:g}] m), q = 1 % of its charge; fluid_threshold "
                     f"{f.threshold:g} m^-3 (cells above go to the fluid); FP32 electrons, seed {spec.seed}",
         "cells": p.M * p.N, "l2": "ne, q (252 MB) and the electrons exceed L2", "parallelism": "1 GPU"}
    if extra:
        c.update(extra)
    return c


def init_oracle_call(spec, ne, q):
    """One initfromfiles! of the oracle (serial, as the reference's loop); returns (s, n)."""
    from oracle import initdens_ref as I
    p = spec.fluid.poisson
    t0 = time.perf_counter()
    x, w, s, qfd, nf = I.initfromfiles(ne, q, p.R, p.L, p.M, p.N, I.POISSON, spec.p,
                                       fluid_threshold=spec.fluid.threshold, seed=spec.seed, cap=12_000_000)
    return time.perf_counter() - t0, len(w)


def run_init(args):
    import ctypes as C

    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import jumc, lxcat, streamer, workloads
    from mcstreamer_b200.fluid import Fluid

    ws, rank, local = dist_env()
    if ws > 1:
        # replicas only: one grid's initialisation is not sharded
        import torch.distributed as dist
        dist.init_process_group("nccl")
    torch.cuda.set_device(local)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spec = workloads.init_spec()
    p = spec.fluid.poisson
    ne, q = workloads.init_densities(spec)
    cap = 12_000_000
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    grid = streamer.GridCyl(p.R, p.L, p.M, p.N, ctx=ctx)
    fl = Fluid(grid)
    pop = jumc.Population(cap, None, tab, precision="fp32", seed=spec.seed)
    lib = ctx.lib
    d_ne = torch.from_numpy(np.ascontiguousarray(ne.ravel(order="F"))).cuda()
    d_q = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).cuda()
    added = C.c_int64()

    def step():
        ctx.check(lib.mcs_pop_upload(pop.h, None, None, None, None, None, 0))
        ctx.check(lib.mcs_init_from_density_device(pop.h, grid.h_, C.c_void_p(d_ne.data_ptr()),
                                                   C.c_void_p(d_q.data_ptr()), L.INIT_POISSON, spec.p,
                                                   spec.fluid.threshold, spec.seed, C.byref(added)))

    for _ in range(args.warmup):
        step()
    times = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        for _ in range(args.steps):
            ctx.check(lib.mcs_pop_upload(pop.h, None, None, None, None, None, 0))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.mcs_init_from_density_device(pop.h, grid.h_, C.c_void_p(d_ne.data_ptr()),
                                                       C.c_void_p(d_q.data_ptr()), L.INIT_POISSON, spec.p,
                                                       spec.fluid.threshold, spec.seed, C.byref(added)))
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    n_el = added.value
    total_ms = float(sum(times))
    if ws > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    value = ws * n_el / (ms * 1e-3)
    pk, src = peaks()
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    alg = init_alg_bytes(p.M * p.N, n_el, 4)
    ach = alg / (ms * 1e-3) / 1e9

    # end to end: ne, q from pinned host memory; the electrons back into pinned host arrays
    h_ne = torch.from_numpy(np.ascontiguousarray(ne.ravel(order="F"))).pin_memory()
    h_q = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).pin_memory()
    hx = torch.empty((cap, 3), dtype=torch.float64).pin_memory()
    hv = torch.empty((cap, 3), dtype=torch.float64).pin_memory()
    hw = torch.empty(cap, dtype=torch.float64).pin_memory()
    hs = torch.empty(cap, dtype=torch.float64).pin_memory()
    ha = torch.empty(cap, dtype=torch.uint8).pin_memory()
    pd = C.POINTER(C.c_double)
    e2e_t = []
    nn = C.c_int64()
    for k in range(max(1, args.e2e_steps) + 1):
        ctx.check(lib.mcs_pop_upload(pop.h, None, None, None, None, None, 0))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.check(lib.mcs_init_from_density(pop.h, grid.h_, C.cast(h_ne.data_ptr(), pd), C.cast(h_q.data_ptr(), pd),
                                            L.INIT_POISSON, spec.p, spec.fluid.threshold, spec.seed,
                                            C.byref(added)))
        ctx.check(lib.mcs_pop_download(pop.h, C.cast(hx.data_ptr(), pd), C.cast(hv.data_ptr(), pd),
                                       C.cast(hw.data_ptr(), pd), C.cast(hs.data_ptr(), pd),
                                       C.cast(ha.data_ptr(), C.POINTER(C.c_uint8)), cap, C.byref(nn)))
        if k:
            e2e_t.append(time.perf_counter() - t0)
    e2e_v = n_el / statistics.median(e2e_t)

    cpu = None
    if rank == 0 and not args.no_cpu:
        sec, n_cpu = init_oracle_call(spec, ne, q)
        cpu = {"value": n_cpu / sec, "unit": "electrons/s", "cores": 1, "kind": "port",
               "sample": f"one full initfromfiles! of this workload by the oracle's serial loop (the reference's "
                         f"loop is serial): {sec:.2f} s, {n_cpu} electrons"}
    line = {
        "metric": INIT_METRIC, "value": value, "unit": "electrons/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 sampling, f32 electrons", "data": "synthetic",
        "config": init_config(spec, {"electrons": n_el, "fluid_cells": int((ne > spec.fluid.threshold).sum())}),
        "roofline": {"kernel": "mcs_init_from_density_device (k_init_count, scan, k_init_place)", "bound": "hbm",
                     "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": profiled_traffic("init_from_density_sample_grid"),
                     "peak_source": src, "launch_ms": ms, "alg_bytes_per_launch": alg},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "electrons/s", "h2d_bytes_per_step": 16 * p.M * p.N,
                "d2h_bytes_per_step": 65 * n_el,
                "path": "mcs_init_from_density (ne, q from pinned host) -> mcs_pop_download (electrons to "
                        "pinned host, Julia layout)"},
        "clocks": clk.summary(),
        "gpu_launches": 6,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    pop.close(); fl.close(); grid.close(); tab.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_init(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    from mcstreamer_b200 import workloads
    spec = workloads.init_spec()
    ne, q = workloads.init_densities(spec)
    runs = [init_oracle_call(spec, ne, q) for _ in range(max(1, min(args.steps, 2)))]
    sec = statistics.median(r[0] for r in runs)
    v = runs[0][1] / sec
    line = {
        "impl": "reference", "metric": INIT_METRIC, "value": v, "unit": "electrons/s", "n_gpus": args.gpus,
        "steps": len(runs), "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": init_config(spec),
        "cpu_baseline": {"value": v, "unit": "electrons/s", "cores": 1, "kind": "port",
                         "sample": f"{len(runs)} full initfromfiles! calls of the oracle's serial loop"},
        "e2e": {"value": v, "unit": "electrons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


LOOP_METRIC = "streamer loop steps/s"


def loop_config(spec, extra=None):
    f = spec.fluid
    p = f.poisson
    c = {"workload": f"nsteps of the sample input on the sample grid: R={p.R:g} m, L={p.L:g} m, {p.M}x{p.N} cells, "
                     f"{p.levels} multigrid levels, eb={p.eb:g} V/m; electrons from initfromfiles!("
                     f"PoissonInitSampling({spec.p})) of a channel of peak {f.peak:g} m^-3, fluid above "
                     f"{f.threshold:g} m^-3; synthetic gas 0 + photo-emission (photon_multiplier 1000); dt=1e-12 s, "
                     f"poisson!, resample!(ntarget=10, nmax=15) and the fluid every step; FP32 electrons, FP64 "
                     f"photons; seed {spec.seed}",
         "cells": p.M * p.N, "l2": "fields (1.5 GB) and particles exceed L2", "parallelism": "1 GPU"}
    if extra:
        c.update(extra)
    return c


def loop_build(ctx, spec, precision="fp32"):
    """The device state of the loop benchmark, initialised from the init workload."""
    from mcstreamer_b200 import jumc, loop, lxcat, streamer, workloads
    from mcstreamer_b200.fluid import Fluid
    from mcstreamer_b200.initdens import PoissonInitSampling, initfromfiles
    from mcstreamer_b200.poisson import MGConfig, PoissonSolver
    p = spec.fluid.poisson
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    tab = jumc.CollisionTable(t, ctx)
    grid = streamer.GridCyl(p.R, p.L, p.M, p.N, ctx=ctx)
    solver = PoissonSolver(grid, MGConfig(levels=p.levels))
    fl = Fluid(grid)
    pop = jumc.Population(30_000_000, None, tab, precision=precision, seed=spec.seed)
    ne, q = workloads.init_densities(spec)
    initfromfiles(PoissonInitSampling(spec.p), grid, pop, ne=ne, q=q, fluid_threshold=spec.fluid.threshold,
                  seed=spec.seed)
    ph = jumc.Photons(8_000_000, t.photon_numax, seed=spec.seed + 1, ctx=ctx)
    st = loop.Streamer(grid, solver, pop, streamer.FieldInterp(grid), ph, fl)
    return st, tab, t


def loop_close(st, tab):
    st.efield.close(); st.photons.close(); st.fluid.close(); st.electrons.close(); st.solver.close(); st.grid.close()
    tab.close()


def loop_oracle_step(spec, x, w, s, er, ez, qfixed, qpart, qfd, ne, u):
    """One nsteps step of the oracle chain over the given state (FP64, all host threads):
    poisson!, advance! (electrons, photons, tracker), repack!, resample!, setdne!/euler!,
    repack!.  Returns (seconds, electrons after the step)."""
    import numpy as np

    from mcstreamer_b200 import lxcat
    from oracle import fluid_ref as F
    from oracle import poisson_ref as P
    from oracle import pyoracle as po
    p = spec.fluid.poisson
    t = lxcat.synthetic_photo_table(0, photon_multiplier=1000.0, photon_weight=1.0)
    n = len(w)
    opop = po.OraclePop(x, np.zeros((n, 3)), w, s, np.ones(n, np.uint8), cap=3 * n + 1000, seed=spec.seed)
    oph = po.OraclePhotons(8_000_000, t.photon_numax, seed=spec.seed + 1)
    otab = po.OracleTable.from_lxcat(t)
    otrk = po.tracker_cyl(p.R, p.L, p.M, p.N)
    t0 = time.perf_counter()
    P.poisson(P.default_conf(p.R, p.L, p.M, p.N, levels=p.levels), qfixed, qpart, u, er, ez, p.eb, p.R, p.L,
              qfd=qfd, ne=ne)
    ofield = po.field_cyl(p.R, p.L, p.M, p.N, er.T.ravel(), ez.T.ravel())
    po.advance_mixed(opop, oph, otab, ofield, 1e-12, otrk, clamp=True)
    po.photons_repack(oph)
    po.repack(opop)
    po.sort_cells(opop, ofield)
    po.resample_cells(opop, ofield, 10, 15, 0)
    ne2 = np.asfortranarray(ne.reshape((p.M + 4, p.N + 4), order="F").copy())
    dne = F.centers(p.M, p.N)
    F.setdne(ne2, dne, er, ez, p.R, p.L, p.M, p.N)
    F.euler(ne2, dne, 1e-12, p.M, p.N)
    po.repack(opop)
    return time.perf_counter() - t0, opop.n


def run_loop(args):
    import ctypes as C
    import tempfile

    import torch

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200 import fieldsio, jumc, loop, workloads

    ws, rank, local = dist_env()
    if ws > 1:
        # replicas only: one streamer's loop is not sharded
        import torch.distributed as dist
        dist.init_process_group("nccl")
    torch.cuda.set_device(local)
    ctx = jumc.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    spec = workloads.loop_spec()
    p = spec.fluid.poisson
    st, tab, _ = loop_build(ctx, spec)
    n_init = st.electrons.nparticles()
    kw = dict(ntarget=10, nmax=15, eb=p.eb, dt=1e-12, dt_poisson=1e-12, dt_output=1e-10, dt_resample=1e-12)
    loop.nsteps(st, args.warmup, **kw)
    launches0 = st.solver.launches() + st.fluid.launches()
    times, electron_steps, phases = [], 0, {}
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        for _ in range(args.steps):
            n_before = st.electrons.nparticles() + st.photons.count()
            marks = []

            def mark(name):
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(stream)
                marks.append((name, ev))

            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            loop.nsteps(st, 1, mark=mark, **kw)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            for (name, a), (_, b) in zip(marks, marks[1:]):
                phases.setdefault(name, []).append(a.elapsed_time(b))
            electron_steps += n_before
        torch.cuda.synchronize()
    total_ms = float(sum(times))
    if ws > 1:
        tt = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms = total_ms / args.steps
    value = ws * 1e3 / ms
    last = st.log[-1]
    launches = (st.solver.launches() + st.fluid.launches() - launches0) // args.steps
    gs_ms, res_ms, tile_ms = st.solver.profile(5)
    pk, src = peaks()
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    ach = poisson_alg_bytes_tile(p.M, p.N) / (tile_ms * 1e-3) / 1e9
    loop_close(st, tab)

    # end to end: host init densities in, K steps with their diagnostics lines, one savefields
    ne, q = workloads.init_densities(spec)
    k_e2e = max(1, args.e2e_steps)
    with tempfile.TemporaryDirectory() as tmp:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, tab, _ = loop_build(ctx, spec)
        loop.nsteps(st, k_e2e, **kw)
        fieldsio.savefields(f"{tmp}/fields.h5", st.grid, st.solver, st.fluid)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        loop_close(st, tab)
    e2e_v = k_e2e / e2e_s

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = loop_cpu_sample(ctx, spec)
    line = {
        "metric": LOOP_METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 electrons, f64 fields and photons", "data": "synthetic",
        "config": loop_config(spec, {"electrons_initial": n_init, "electrons_last": last["active_superelectrons"],
                                     "photons_last": last["active_superphotons"],
                                     "particle_steps_per_s": ws * electron_steps / (total_ms * 1e-3),
                                     "phase_ms": {k: statistics.mean(v) for k, v in phases.items()},
                                     "step_ms_each": times}),
        "roofline": {"kernel": "k_smooth_tile<2, TILE_POST> (poisson!, the loop's largest fixed cost)",
                     "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": profiled_traffic("k_smooth_tile_post_sample_grid"), "peak_source": src, "launch_ms": tile_ms,
                     "alg_bytes_per_launch": poisson_alg_bytes_tile(p.M, p.N)},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_v, "unit": "steps/s", "h2d_bytes_per_step": 16 * p.M * p.N / k_e2e,
                "d2h_bytes_per_step": 48 * k_e2e + (2 * (p.M + 2) * (p.N + 2) * 8 * 6) / k_e2e,
                "path": f"initfromfiles! from host densities, {k_e2e} nsteps with their diagnostics lines, one "
                        "savefields (h5export layout) to disk"},
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "gpu_launches_counts": "per step, poisson! and the fluid only (the advance, resample! and repack! kernels "
                               "are not counted)",
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def loop_cpu_sample(ctx, spec):
    """One oracle-chain step from the state the device loop starts from."""
    import numpy as np

    from mcstreamer_b200 import _lib as L
    from mcstreamer_b200.poisson import read_faces
    p = spec.fluid.poisson
    st, tab, _ = loop_build(ctx, spec, precision="fp64")
    g = st.electrons.download()
    ne, _, qfd = st.fluid.download()
    qf = st.grid.read_fixed(L.Q_FIXED)
    from mcstreamer_b200.streamer import density
    st.grid.zero(L.Q_PART)
    density(st.grid, st.electrons, -1.0)
    qp = st.grid.read_fixed(L.Q_PART)
    loop_close(st, tab)
    from oracle import poisson_ref as P
    u = P.cells(p.M, p.N)
    er, ez = P.faces(p.M, p.N), P.faces(p.M, p.N)
    sec, n_after = loop_oracle_step(spec, g.x, g.w, g.s, er, ez, qf, qp, qfd.ravel(order="F"), ne.ravel(order="F"), u)
    threads = os.cpu_count() or 1
    return {"value": 1.0 / sec, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"one nsteps step of this workload by the oracle chain on {threads} threads (poisson!, advance!, "
                      f"repack!, resample!, fluid; {len(g.w)} electrons): {sec:.1f} s"}


def run_reference_loop(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    import numpy as np

    from mcstreamer_b200 import workloads
    from oracle import initdens_ref as I
    from oracle import poisson_ref as P
    spec = workloads.loop_spec()
    p = spec.fluid.poisson
    ne, q = workloads.init_densities(spec)
    x, w, s, qfd, nf = I.initfromfiles(ne, q, p.R, p.L, p.M, p.N, I.POISSON, spec.p,
                                       fluid_threshold=spec.fluid.threshold, seed=spec.seed, cap=12_000_000)
    qp = workloads.poisson_electron_charge(p, x, w)
    u = P.cells(p.M, p.N)
    er, ez = P.faces(p.M, p.N), P.faces(p.M, p.N)
    qf = np.zeros_like(qp)
    sec, n_after = loop_oracle_step(spec, x, w, s, er, ez, qf, qp, qfd.ravel(order="F"), nf.ravel(order="F"), u)
    v = 1.0 / sec
    threads = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": LOOP_METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus,
        "steps": 1, "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": loop_config(spec),
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"one nsteps step of the oracle chain ({len(w)} electrons)"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "cfg2":
        return run_reference_cfg2(args) if args.impl == "reference" else run_cfg2(args)
    if args.workload == "cfg0":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the oracle replicas run inside the cfg0 line "
                              "(cpu_baseline); no separate reference arm"}))
            return 0
        return run_cfg0(args)
    if args.workload == "cfg3":
        return run_reference_batch(args) if args.impl == "reference" else run_batch(args)
    if args.workload == "poisson":
        return run_reference_poisson(args) if args.impl == "reference" else run_poisson(args)
    if args.workload == "photons":
        return run_reference_photons(args) if args.impl == "reference" else run_photons(args)
    if args.workload == "fluid":
        return run_reference_fluid(args) if args.impl == "reference" else run_fluid(args)
    if args.workload == "init":
        return run_reference_init(args) if args.impl == "reference" else run_init(args)
    if args.workload == "loop":
        return run_reference_loop(args) if args.impl == "reference" else run_loop(args)
    if args.workload == "cfg4":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the served workload has no CPU reference arm; "
                              "the oracle's swarm rate is reported by --workload cfg3 --impl reference"}))
            return 0
        return run_serve(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_mine(args)


if __name__ == "__main__":
    sys.exit(main())
