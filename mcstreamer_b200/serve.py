"""Serving swarm solves: continuous batching of requests on one GPU.

A request is one Swarm.swarm solve (Swarm/src/Swarm.jl:102-173) -- a gas, a reduced field
E/N and an electron count -- that runs until its ionization-rate estimate is statistically
settled.  The server keeps every admitted request resident as an instance of one
SwarmBatch, advances all of them together (one CUDA graph per batched step), and between
chunks of steps retires the requests whose stopping rule holds and admits waiting ones
while an instance slot and a free particle region of the batch's memory pool are
available (first fit; the pool is sized from the memory budget).

Each request's result is a function of its own per-step sums only (its particles evolve
exactly as they do alone) and the stopping step is the first step at which the rule holds,
whatever the chunking, so a result is the same alone and in any mix.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib as L
from . import constants as co
from .batch import SwarmBatch
from .jumc import CollisionTable, Context

# bytes of batch memory per particle slot: 8 FP32 fields + active byte + two u32 scan words
BYTES_PER_SLOT = 8 * 4 + 1 + 2 * 4
MAX_POOL_SLOTS = 0x7FFFFFFF


@dataclass
class SwarmRequest:
    rid: int
    gas: int                 # index into the server's tables
    en_td: float             # reduced field, Td
    n: int                   # electrons (also the Swarm.resample! target)
    seed: int
    arrival: float = 0.0     # seconds after the start of the run
    mean_ev: float = 1.0     # initial isotropic Maxwellian


@dataclass
class StopRule:
    """Run until 3 sigma of the mean ionization rate is within `rel` of it.

    The rate per step is <nu_ion(eps)> over active electrons (the estimator of collrate,
    Swarm.jl:242-248, for the ionization row).  Steps before `min_steps` are relaxation and
    not averaged; sigma comes from the means of consecutive blocks of `block` steps (the
    batch-means method, which absorbs the step-to-step correlation within a block), and
    needs at least `min_blocks` blocks.  A solve with no ionization at all after the
    minimum (rate and spread exactly 0) is settled at 0; `max_steps` bounds every solve."""
    rel: float = 0.01
    min_steps: int = 200
    block: int = 20
    min_blocks: int = 5
    max_steps: int = 2000

    def first_check(self) -> int:
        return self.min_steps + self.min_blocks * self.block

    def evaluate(self, nu: np.ndarray, start_T: Optional[int] = None) -> tuple[int, float, float, bool, int]:
        """First step count T >= start_T (on the block grid) at which the rule holds over
        the per-step rates nu[0..T).  Returns (T, mean, 3 sigma, settled, next T to check);
        T = -1 when no decision is possible yet."""
        T = self.first_check() if start_T is None else start_T
        while T <= len(nu):
            if T >= self.max_steps:
                k, err = self.stats(nu[:self.max_steps])
                settled = (k == 0.0 and err == 0.0) or (k != 0.0 and err <= self.rel * abs(k))
                return self.max_steps, k, err, settled, T
            k, err = self.stats(nu[:T])
            if (k == 0.0 and err == 0.0) or (k != 0.0 and err <= self.rel * abs(k)):
                return T, k, err, True, T
            T += self.block
        if len(nu) >= self.max_steps:
            k, err = self.stats(nu[:self.max_steps])
            return self.max_steps, k, err, False, T
        return -1, 0.0, float("inf"), False, T

    def stats(self, nu: np.ndarray) -> tuple[float, float]:
        b = self.block
        w = nu[self.min_steps:]
        nb = len(w) // b
        if nb < 2:
            return float(w.mean()) if len(w) else 0.0, float("inf")
        blocks = w[len(w) - nb * b:].reshape(nb, b).mean(axis=1)
        return float(blocks.mean()), float(3.0 * blocks.std(ddof=1) / np.sqrt(nb))


@dataclass
class SwarmResponse:
    rid: int
    gas: int
    en_td: float
    n: int
    steps: int               # stopping step
    k_ion: float             # m^3/s
    k_ion_err3: float        # 3 sigma of k_ion
    settled: bool
    drift: float             # <v_z> over the averaged steps, m/s
    mean_energy: float       # eV, over the averaged steps
    arrival: float
    admitted: float
    finished: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Live:
    req: SwarmRequest
    slot: int
    cap: int
    admitted: float
    next_T: int = 0
    first_chunk: int = 0                        # first chunk whose steps include this request
    rows: list = field(default_factory=list)    # per-step sums, in step order
    nu: list = field(default_factory=list)      # per-step mean ionization rate

    def sums(self) -> np.ndarray:
        return np.concatenate(self.rows) if self.rows else np.zeros((0, L.BATCH_MOMENTS))


class SwarmServer:
    """Continuous-batching swarm server over one SwarmBatch."""

    def __init__(self, ctx: Context, tables: Sequence[CollisionTable], dt: float, density: float,
                 budget_bytes: float = 160e9, rule: Optional[StopRule] = None, max_instances: int = 1024,
                 chunk: int = 16, graph: bool = True, capacity_factor: float = 2.0):
        self.ctx = ctx
        self.tables = list(tables)
        self.dt = float(dt)
        self.density = float(density)
        self.rule = rule or StopRule()
        self.chunk = max(1, min(int(chunk), L.BATCH_LOG))
        self.graph = graph
        self.capacity_factor = capacity_factor
        pool = int(budget_bytes // BYTES_PER_SLOT)
        try:
            import torch
            free, _ = torch.cuda.mem_get_info(ctx.device)
            pool = min(pool, int(0.9 * free // BYTES_PER_SLOT))
        except Exception:
            pass
        self.pool_slots = max(1, min(pool, MAX_POOL_SLOTS))
        self.batch = SwarmBatch(ctx, max_instances, self.pool_slots)
        self.live: dict[int, _Live] = {}
        self.free_slots = self.pool_slots
        self.gpu_steps = 0

    def capacity_of(self, req: SwarmRequest) -> int:
        return max(64, int(self.capacity_factor * req.n))

    def _admit(self, req: SwarmRequest, now: float, first_chunk: int) -> bool:
        cap = self.capacity_of(req)
        if cap > self.free_slots or len(self.live) >= self.batch.max_instances:
            return False
        ez = req.en_td * self.density * co.Td
        try:
            slot = self.batch.add_maxwellian(self.tables[req.gas], ez, req.seed, req.n, cap, req.n, req.mean_ev)
        except L.MCSError as e:
            if e.code in (L.ERR_NOMEM, L.ERR_CAPACITY):   # fragmented pool / no instance slot
                return False
            raise
        self.free_slots -= cap
        lv = _Live(req, slot, cap, now, self.rule.first_check())
        lv.first_chunk = first_chunk
        self.live[slot] = lv
        return True

    def _retire(self, slot: int) -> None:
        self.batch.remove(slot)
        self.free_slots += self.live.pop(slot).cap

    def _respond(self, lv: _Live, T: int, k: float, err: float, settled: bool, now: float) -> SwarmResponse:
        s = lv.sums()[:T]
        w = s[self.rule.min_steps:] if T > self.rule.min_steps else s
        cnt = np.maximum(w[:, L.S_COUNT], 1.0)
        drift = float((w[:, L.S_V + 2] / cnt).mean()) if len(w) else 0.0
        energy = float((w[:, L.S_E] / cnt).mean() / co.eV) if len(w) else 0.0
        return SwarmResponse(lv.req.rid, lv.req.gas, lv.req.en_td, lv.req.n, T, k / self.density,
                             err / self.density, settled, drift, energy, lv.req.arrival, lv.admitted, now)

    def _collect(self, ring: np.ndarray, pos: np.ndarray, chunk_id: int, nsteps: int, now: float
                 ) -> list[SwarmResponse]:
        done = []
        for slot, lv in list(self.live.items()):
            if lv.first_chunk > chunk_id:        # joined after this chunk was enqueued
                continue
            p = int(pos[slot])
            rows = ring[slot, [(t % L.BATCH_LOG) for t in range(p - nsteps, p)]]
            lv.rows.append(rows)
            lv.nu.extend((rows[:, L.B_NU] / np.maximum(rows[:, L.S_COUNT], 1.0)).tolist())
            T, k, err, settled, lv.next_T = self.rule.evaluate(np.asarray(lv.nu), lv.next_T)
            if T > 0:
                done.append(self._respond(lv, T, k, err, settled, now))
                self._retire(slot)
        return done

    def run(self, requests: Sequence[SwarmRequest], clock: Callable[[], float] = time.perf_counter,
            realtime: bool = True, on_response: Optional[Callable[[SwarmResponse], None]] = None,
            deadline: Optional[float] = None) -> list[SwarmResponse]:
        """Serve `requests` (arrival times relative to the start).  realtime=False admits
        every request at once in arrival order (the arrival clock is ignored).  With a
        deadline (seconds) the run stops there; unfinished requests are left out of the
        result and counted in self.unfinished.

        The device always has the next chunk queued while the host reads the previous
        chunk's per-step sums (two pinned log buffers): joins, leaves and the log copies are
        stream-ordered, so the host never waits for the GPU except for the oldest chunk."""
        order = sorted(requests, key=lambda r: (r.arrival, r.rid))
        t0 = clock()
        nxt = 0
        queue: list[SwarmRequest] = []
        out: list[SwarmResponse] = []
        inflight: list[tuple[int, int]] = []     # (chunk id, steps) enqueued, not yet read
        chunk_id = 0
        self.unfinished = 0
        while True:
            now = clock() - t0
            if deadline is not None and now > deadline:
                for cid, k in inflight:
                    self.batch.logs_wait(cid % 2)
                self.unfinished = len(order) - nxt + len(queue) + len(self.live)
                for slot in list(self.live):
                    self._retire(slot)
                self.batch.sync()
                break
            while nxt < len(order) and (not realtime or order[nxt].arrival <= now):
                queue.append(order[nxt])
                nxt += 1
            while queue and self._admit(queue[0], now, chunk_id):
                queue.pop(0)
            if self.live and len(inflight) < 2:
                k = self.chunk
                self.batch.step(self.dt, k, graph=self.graph)
                self.batch.logs_enqueue(chunk_id % 2)
                inflight.append((chunk_id, k))
                chunk_id += 1
                self.gpu_steps += k
                continue
            if inflight:
                cid, k = inflight.pop(0)
                ring, pos = self.batch.logs_wait(cid % 2)
                for r in self._collect(ring, pos, cid, k, clock() - t0):
                    out.append(r)
                    if on_response:
                        on_response(r)
                continue
            if queue:
                raise RuntimeError(f"request {queue[0].rid} does not fit the memory pool")
            if nxt >= len(order):
                break
            time.sleep(max(0.0, min(0.01, order[nxt].arrival - (clock() - t0))))
        self.batch.sync()
        return sorted(out, key=lambda r: r.rid)

    def close(self) -> None:
        self.batch.close()


def percentiles(lat: Sequence[float]) -> dict:
    a = np.asarray(lat, dtype=np.float64)
    if len(a) == 0:
        return {"p50": None, "p95": None, "p99": None}
    return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
            "p99": float(np.percentile(a, 99))}


def serial_latencies(arrivals: Sequence[float], service: Sequence[float]) -> np.ndarray:
    """Latencies of a single FIFO server that runs one request at a time (Lindley)."""
    free = 0.0
    lat = np.zeros(len(arrivals))
    for i, (a, s) in enumerate(sorted(zip(arrivals, service))):
        start = max(a, free)
        free = start + s
        lat[i] = free - a
    return lat


def poisson_requests(rate: float, duration: float, seed: int, n_range=(1024, 2_097_152), en_range=(10.0, 1000.0),
                     gases: int = 4) -> list[SwarmRequest]:
    """Poisson arrivals at `rate` per second over `duration` seconds; gas uniform over
    `gases`, E/N and electron count log-uniform over their ranges."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        n = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        en = float(np.exp(rng.uniform(np.log(en_range[0]), np.log(en_range[1]))))
        out.append(SwarmRequest(len(out), int(rng.integers(0, gases)), en, n, int(rng.integers(0, 2**62)), t))
    return out
