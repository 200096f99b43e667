"""Batched swarms: many independent Swarm.swarm solves advanced together on one GPU.

The reference solves one E/N point of one gas per call (Swarm/src/Swarm.jl:102-173) and
sweeps them in a host loop (:48-186).  A SwarmBatch keeps every solve resident as an
instance of one device population; a step is the fixed kernel sequence advance! ->
Swarm.resample! -> repack! over all instances (one CUDA graph when `graph=True`), and each
instance's particles evolve exactly as a single FP32 population does under
mcs_swarm_run(..., repack_every=1) with the same table, field and seed.

BatchedSwarms runs whole solves on top of it: instances join when there is room, leave
when they have run their steps, and their coefficients are formed from the per-step sums
exactly as swarm_one forms them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from . import constants as co
from .jumc import CollisionTable, Context, ParticleArrays


class SwarmBatch:
    """Device-resident set of FP32 swarm instances (mcs_batch)."""

    def __init__(self, ctx: Context, max_instances: int, total_capacity: int):
        self.ctx = ctx
        self.max_instances = int(max_instances)
        self.total_capacity = int(total_capacity)
        h = C.c_void_p()
        ctx.check(ctx.lib.mcs_batch_create(ctx.h, self.max_instances, self.total_capacity, C.byref(h)))
        self.h = h

    def add(self, table: CollisionTable, ez: float, seed: int, n0: int, capacity: int, particles: ParticleArrays,
            tol: float = 0.1, ex: float = 0.0, ey: float = 0.0) -> int:
        """Join an instance in field (ex, ey, ez); n0 <= 0 disables Swarm.resample!."""
        p = particles
        x = np.ascontiguousarray(p.x, dtype=np.float64)
        v = np.ascontiguousarray(p.v, dtype=np.float64)
        w = np.ascontiguousarray(p.w, dtype=np.float64)
        s = np.ascontiguousarray(p.s, dtype=np.float64)
        a = np.ascontiguousarray(p.active, dtype=np.uint8)
        slot = C.c_int(-1)
        self.ctx.check(self.ctx.lib.mcs_batch_add(
            self.h, table.h, float(ex), float(ey), float(ez), C.c_uint64(seed), int(n0), float(tol), int(capacity),
            L.dptr(x), L.dptr(v), L.dptr(w), L.dptr(s), L.u8ptr(a), len(w), C.byref(slot)))
        return slot.value

    def add_maxwellian(self, table: CollisionTable, ez: float, seed: int, n0: int, capacity: int, n: int,
                       mean_ev: float = 1.0, tol: float = 0.1, ex: float = 0.0, ey: float = 0.0) -> int:
        """Join with n electrons drawn on the device (stream-ordered, no host wait)."""
        slot = C.c_int(-1)
        self.ctx.check(self.ctx.lib.mcs_batch_add_maxwellian(
            self.h, table.h, float(ex), float(ey), float(ez), C.c_uint64(seed), int(n0), float(tol), int(capacity),
            int(n), float(mean_ev), C.byref(slot)))
        return slot.value

    def logs_enqueue(self, buf: int) -> None:
        self.ctx.check(self.ctx.lib.mcs_batch_logs_enqueue(self.h, int(buf)))

    def logs_wait(self, buf: int) -> tuple[np.ndarray, np.ndarray]:
        """Views of pinned buffer `buf` (ring, logged steps); valid until its next enqueue."""
        ring = L.pd()
        pos = C.POINTER(C.c_uint32)()
        self.ctx.check(self.ctx.lib.mcs_batch_logs_wait(self.h, int(buf), C.byref(ring), C.byref(pos)))
        r = np.ctypeslib.as_array(ring, shape=(self.max_instances, L.BATCH_LOG, L.BATCH_MOMENTS))
        p = np.ctypeslib.as_array(pos, shape=(self.max_instances,))
        return r, p

    def remove(self, slot: int) -> None:
        self.ctx.check(self.ctx.lib.mcs_batch_remove(self.h, int(slot)))

    def step(self, dt: float, nsteps: int = 1, graph: bool = True) -> None:
        """Enqueue nsteps batched steps on the context's stream (asynchronous)."""
        self.ctx.check(self.ctx.lib.mcs_batch_step(self.h, float(dt), int(nsteps), 1 if graph else 0))

    def sync(self) -> None:
        self.ctx.check(self.ctx.lib.mcs_batch_sync(self.h))

    def state(self) -> tuple[np.ndarray, np.ndarray]:
        """(particle count, completed steps) per instance slot."""
        n = np.zeros(self.max_instances, np.int64)
        st = np.zeros(self.max_instances, np.uint32)
        self.ctx.check(self.ctx.lib.mcs_batch_state(self.h, L.i64ptr(n), st.ctypes.data_as(C.POINTER(C.c_uint32))))
        return n, st

    def read_log(self, slot: int, count: int) -> np.ndarray:
        """(count, BATCH_MOMENTS) per-step sums of the last `count` steps, oldest first."""
        out = np.zeros((count, L.BATCH_MOMENTS))
        self.ctx.check(self.ctx.lib.mcs_batch_read_log(self.h, int(slot), L.dptr(out), int(count)))
        return out

    def read_current(self) -> np.ndarray:
        """(max_instances, BATCH_MOMENTS) sums of every slot's most recent step."""
        out = np.zeros((self.max_instances, L.BATCH_MOMENTS))
        self.ctx.check(self.ctx.lib.mcs_batch_read_current(self.h, L.dptr(out)))
        return out

    def read_logs(self) -> tuple[np.ndarray, np.ndarray]:
        """(ring, logged steps) of every slot: ring[k, t % BATCH_LOG] holds step t's sums."""
        ring = np.zeros((self.max_instances, L.BATCH_LOG, L.BATCH_MOMENTS))
        pos = np.zeros(self.max_instances, np.uint32)
        self.ctx.check(self.ctx.lib.mcs_batch_read_logs(self.h, L.dptr(ring), pos.ctypes.data_as(C.POINTER(C.c_uint32))))
        return ring, pos

    def download(self, slot: int) -> ParticleArrays:
        n, _ = self.state()
        m = int(n[slot])
        out = ParticleArrays.empty(m)
        got = C.c_int64(0)
        self.ctx.check(self.ctx.lib.mcs_batch_download(
            self.h, int(slot), L.dptr(out.x), L.dptr(out.v), L.dptr(out.w), L.dptr(out.s), L.u8ptr(out.active), m,
            C.byref(got)))
        return out

    def autotune(self, dt: float, trial_steps: int = 3) -> tuple[int, np.ndarray]:
        """Time all (block, particles-per-thread) variants on the current state, keep the fastest."""
        chosen = C.c_int(-1)
        times = np.zeros(L.BATCH_VARIANTS, np.float32)
        self.ctx.check(self.ctx.lib.mcs_batch_autotune(self.h, float(dt), int(trial_steps), C.byref(chosen),
                                                       times.ctypes.data_as(C.POINTER(C.c_float))))
        return chosen.value, times

    def profile(self, dt: float, nsteps: int) -> tuple[float, float]:
        """(advance! kernel ms, whole step ms) per step over nsteps steps without the graph."""
        k, t = C.c_float(0), C.c_float(0)
        self.ctx.check(self.ctx.lib.mcs_batch_profile(self.h, float(dt), int(nsteps), C.byref(k), C.byref(t)))
        return k.value, t.value

    def set_variant(self, variant: int) -> None:
        self.ctx.check(self.ctx.lib.mcs_batch_set_variant(self.h, int(variant)))

    @staticmethod
    def variant_shape(variant: int) -> tuple[int, int]:
        b, p = C.c_int(0), C.c_int(0)
        L.check(L.lib().mcs_batch_variant_shape(int(variant), C.byref(b), C.byref(p)))
        return b.value, p.value

    def close(self) -> None:
        if self.h:
            self.ctx.lib.mcs_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class Solve:
    """One swarm solve: a gas table at one reduced field (Td) with its own seed."""
    table: CollisionTable
    en_td: float
    seed: int
    n0: int
    nt: int
    density: float
    init: str = "maxwellian"
    mean_ev: float = 1.0
    tol: float = 0.1
    capacity: Optional[int] = None
    tag: object = None


@dataclass
class SolveResult:
    tag: object
    en_td: float
    steps: int
    sums: np.ndarray = field(repr=False)    # (steps, BATCH_MOMENTS) per-step sums
    k_ion: float = 0.0                       # <nu_ion> / N over the averaging window
    k_ion_rel_err: float = float("inf")      # 3 sigma / k_ion of that mean
    drift: float = 0.0


def solve_metrics(sums: np.ndarray, density: float, window: int) -> tuple[float, float, float]:
    """Per-step ionization-rate and drift estimates over the last `window` steps: k_ion =
    mean over steps of sum(nu_ion)/count / N, with 3 sigma of that mean from the step-to-step
    scatter (steps are correlated, so the scatter is an estimate, not a bound)."""
    s = sums[-window:]
    cnt = np.maximum(s[:, L.S_COUNT], 1.0)
    nu = s[:, L.B_NU] / cnt / density
    k = float(nu.mean())
    err = float(3.0 * nu.std(ddof=1) / np.sqrt(len(nu))) if len(nu) > 1 else float("inf")
    W = float((s[:, L.S_V + 2] / cnt).mean())
    return k, (err / abs(k) if k != 0 else float("inf")), W


class BatchedSwarms:
    """Run many Solves through one SwarmBatch: fill free instance slots, step everything
    together, collect each solve's per-step sums as it finishes its nt steps."""

    def __init__(self, ctx: Context, max_instances: int, total_capacity: int, dt: float, graph: bool = True,
                 chunk: int = 16):
        self.ctx = ctx
        self.batch = SwarmBatch(ctx, max_instances, total_capacity)
        self.dt = dt
        self.graph = graph
        self.chunk = max(1, min(int(chunk), L.BATCH_LOG))
        self.free_cap = total_capacity

    def run(self, solves: Sequence[Solve], window: int = 100) -> list[SolveResult]:
        from .swarm import initial_particles
        pending = list(range(len(solves)))
        live: dict[int, tuple[int, list[np.ndarray], int]] = {}   # slot -> (solve index, chunks, done)
        results: list[Optional[SolveResult]] = [None] * len(solves)
        while pending or live:
            # admit while there is room (instances and capacity)
            while pending and len(live) < self.batch.max_instances:
                i = pending[0]
                sv = solves[i]
                cap = sv.capacity or 4 * sv.n0
                if cap > self.free_cap:
                    break
                p0 = initial_particles(sv.n0, sv.init, sv.seed, mean_ev=sv.mean_ev)
                ez = sv.en_td * sv.density * co.Td
                try:
                    slot = self.batch.add(sv.table, ez, sv.seed, sv.n0, cap, p0, tol=sv.tol)
                except L.MCSError as e:
                    if e.code != L.ERR_NOMEM or not live:   # a fragmented region: wait for a leave
                        raise
                    break
                self.free_cap -= cap
                live[slot] = (i, [], 0)
                pending.pop(0)
            if not live:
                raise RuntimeError("a solve does not fit the batch capacity")
            k = min(self.chunk, min(solves[i].nt - done for i, _, done in live.values()))
            self.batch.step(self.dt, k, graph=self.graph)
            for slot in list(live):
                i, chunks, done = live[slot]
                chunks.append(self.batch.read_log(slot, k))
                done += k
                if done >= solves[i].nt:
                    sums = np.concatenate(chunks)
                    sv = solves[i]
                    kk, rel, W = solve_metrics(sums, sv.density, min(window, len(sums)))
                    results[i] = SolveResult(sv.tag, sv.en_td, done, sums, kk, rel, W)
                    self.batch.remove(slot)
                    self.free_cap += sv.capacity or 4 * sv.n0
                    del live[slot]
                else:
                    live[slot] = (i, chunks, done)
        return results  # type: ignore[return-value]

    def close(self) -> None:
        self.batch.close()
