"""jumc_ref -- TEST INFRASTRUCTURE (the checker, never the product).

A second CPU restatement of JuMC's electron step, in plain Python loops, written from the
Julia source line by line and independently of oracle/oracle.cpp (it shares no code with
it: its own Philox4x32-10, its own LinRange arithmetic, its own loops).  tests/ use it to
pin oracle.cpp -- and through oracle.cpp the CUDA kernels -- bit for bit on small cases, and
to check the device's injected-uniform mode (mcs_set_uniform_source) per particle.  It is
slow (pure Python): a few thousand particles and a few steps at most.

What it restates (paths inside the reference project):
  advance!            JuMC/src/mixed_population.jl:24-54
  collisions!         JuMC/src/mixed_population.jl:61-77
  advance_free_yoshida, energy, collide
                      JuMC/src/electron.jl:27,38-62,108-139
  do_one_collision!, rate, presample
                      JuMC/src/collisions.jl:26-39,159-192
  apply!              JuMC/src/collisions.jl:96-123
  randsphere, nextcoll, indweight
                      JuMC/src/util.jl:4-30
  add_particle!, remove_particle!, repack!
                      JuMC/src/population.jl:88-106,191-215
  FixedField          Swarm/src/Swarm.jl:28-32
  Swarm.resample!     Swarm/src/Swarm.jl:193-223
  Grid, cellindex, dV, inside
                      MCStreamer/src/grid.jl:33-90
  FieldInterp, track1 MCStreamer/src/gridfields.jl:94-224
  density!            MCStreamer/src/poisson.jl:65-84
  resample!, samplemin
                      MCStreamer/src/resample.jl:7-84
  LinRange (start, stop, len, lendiv; step, lerpi getindex, sub-range, +, scalar *)
                      Julia 1.8 Base range.jl, the semantics Grid and the energy grid rely on

Random numbers.  Every place the Julia code calls rand() calls `rng.rand(role)` here, in the
same order; `role` names the draw (xi, phi1, u1, phi2, u2, s2, share, s) so that a source
can map it.  Two sources exist:
  * SerialDraws -- the reference's own order: one particle's draws one after the other from
    a caller-given list (what a single-threaded Julia run consumes for that particle);
  * PhiloxEventDraws -- the library's counter-based stream: event j of particle `slot`
    during step `step` owns Philox4x32-10 block {slot, step, j, tag} (xi, s, phi1, u1) and,
    only when needed, block {slot, step, j | 2^31, tag} (phi2, u2, s2, share); a word w is
    the uniform (w + 0.5) * 2^-32.
The 3-D node mesh (trilinear field, CIC int64 deposit at 2^-32 e) is the configurations'
extension, not reference code; it is restated from its definition.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

# JuMC/src/constants.jl:50-54
ELEMENTARY_CHARGE = 1.6021766208e-19
ELECTRON_MASS = 9.10938356e-31

NULL, ELASTIC, EXCITATION, IONIZATION, ATTACHMENT, IONIZATION_UNIFORM = 0, 1, 2, 3, 4, 5
TAG_ADVANCE, TAG_SWARM_RESAMPLE, TAG_CELL_RESAMPLE, TAG_COLLISIONS = 0, 1, 2, 4

M32 = 0xFFFFFFFF


# ---------------------------------------------------------------------------------------
# Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), written out from the paper.
# ---------------------------------------------------------------------------------------
def philox4x32_10(ctr: Sequence[int], key: Sequence[int]) -> tuple[int, int, int, int]:
    c0, c1, c2, c3 = (int(c) & M32 for c in ctr)
    k0, k1 = int(key[0]) & M32, int(key[1]) & M32
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & M32
            k1 = (k1 + 0xBB67AE85) & M32
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M32, p1 & M32, ((p0 >> 32) ^ c3 ^ k1) & M32, p0 & M32
    return c0, c1, c2, c3


def word_uniform(w: int) -> float:
    return (w + 0.5) * 2.0 ** -32


def key_of(seed: int) -> tuple[int, int]:
    return seed & M32, (seed >> 32) & M32


class Stream:
    """Word k of entity `a` in call `b`: block {a, b, k/4, tag}, lane k % 4."""

    def __init__(self, seed: int, a: int, b: int, tag: int):
        self.key = key_of(seed)
        self.a, self.b, self.tag, self.k = a, b, tag, 0
        self.buf = (0, 0, 0, 0)

    def rand(self, role: str = "") -> float:
        if self.k % 4 == 0:
            self.buf = philox4x32_10((self.a, self.b, self.k // 4, self.tag), self.key)
        w = self.buf[self.k % 4]
        self.k += 1
        return word_uniform(w)


class PhiloxEventDraws:
    """The library's per-event stream of one particle in one step (see the module text)."""

    SLOT = {"xi": 0, "s": 1, "phi1": 2, "u1": 3, "phi2": 4, "u2": 5, "s2": 6, "share": 7}

    def __init__(self, seed: int, slot: int, step: int, tag: int):
        self.key = key_of(seed)
        self.slot, self.step, self.tag = slot, step, tag
        self.j = 0
        self.b = self.c = None

    def rand(self, role: str) -> float:
        if role == "xi":    # the first draw of every event opens its block
            self.b = philox4x32_10((self.slot, self.step, self.j, self.tag), self.key)
            self.c = None
            self.j += 1
        q = self.SLOT[role]
        if q < 4:
            return word_uniform(self.b[q])
        if self.c is None:
            self.c = philox4x32_10((self.slot, self.step, (self.j - 1) | 0x80000000, self.tag), self.key)
        return word_uniform(self.c[q - 4])


class SerialDraws:
    """One particle's uniforms in the order a serial run of the reference draws them."""

    def __init__(self, values: Sequence[float]):
        self.values = list(values)
        self.k = 0

    def rand(self, role: str = "") -> float:
        if self.k >= len(self.values):
            raise IndexError("the particle's uniforms are used up")
        u = self.values[self.k]
        self.k += 1
        return u


class CountingSource:
    """Serial order drawn from a generator, recording each particle's values (used to make
    injected-uniform inputs: the recorded lists replayed through SerialDraws, or through the
    device's injected mode, reproduce the run)."""

    def __init__(self, gen: Callable[[], float]):
        self.gen = gen
        self.values: list[float] = []

    def rand(self, role: str = "") -> float:
        u = self.gen()
        self.values.append(u)
        return u


# ---------------------------------------------------------------------------------------
# Julia's LinRange (Base range.jl): lerpi getindex, step = (stop - start) / lendiv.
# ---------------------------------------------------------------------------------------
@dataclass(frozen=True)
class LinRange:
    start: float
    stop: float
    len: int

    @property
    def lendiv(self) -> int:
        return max(1, self.len - 1)

    def step(self) -> float:
        return (self.stop - self.start) / self.lendiv

    def __getitem__(self, i: int) -> float:       # 1-based, like Julia
        t = (i - 1) / self.lendiv
        return (1 - t) * self.start + t * self.stop

    def first(self) -> float:
        return self.start

    def last(self) -> float:
        return self.stop

    def sub(self, a: int, b: int) -> "LinRange":  # r[a:b]
        return LinRange(self[a], self[b], b - a + 1)

    def __add__(self, o: "LinRange") -> "LinRange":
        assert self.len == o.len
        return LinRange(self.start + o.start, self.stop + o.stop, self.len)

    def scale(self, x: float) -> "LinRange":      # x * r
        return LinRange(x * self.start, x * self.stop, self.len)


def julia_mod(x: float, y: float) -> float:
    r = math.fmod(x, y)
    if r == 0.0:
        return math.copysign(0.0, y)
    if (r > 0) != (y > 0):
        return r + y
    return r


def fld(x: float, y: float) -> float:
    """Base fld for floats: round((x - mod(x, y)) / y), round half to even."""
    return float(round((x - julia_mod(x, y)) / y))


# ---------------------------------------------------------------------------------------
# Tables and the collision processes
# ---------------------------------------------------------------------------------------
@dataclass
class Table:
    """CollisionTable (collisions.jl:9-22): proc kinds/params, energy LinRange, rate[j, k]."""

    kinds: list
    params: list
    energy: LinRange
    rate: np.ndarray        # (nrows, neps): rate[j, k] with j the process
    maxrate: float

    @classmethod
    def from_lxcat(cls, t) -> "Table":
        e = t.energy
        return cls([int(k) for k in t.kinds], [float(p) for p in t.params], LinRange(float(e.e0), float(e.emax), int(e.n)),
                   np.asarray(t.rate, dtype=np.float64), float(t.maxrate))


class EnergyRangeError(Exception):
    """indweight's @assert 0 <= w <= 1 / BoundsError (util.jl:28)."""


def indweight(r: LinRange, x: float) -> tuple[int, float]:
    """util.jl:23-30 (1-based index i)."""
    i = int(fld(x - r.first(), r.step())) + 1
    if not (1 <= i and i + 1 <= r.len):
        raise EnergyRangeError(x)
    w = (r[i + 1] - x) / r.step()
    if not (0 <= w <= 1):
        raise EnergyRangeError(x)
    return i, w


def rate(tab: Table, j: int, pre: tuple[int, float]) -> float:
    """collisions.jl:35-39 (j, k 1-based)."""
    k, w = pre
    return w * tab.rate[j - 1, k - 1] + (1 - w) * tab.rate[j - 1, k]


def sq(x: float) -> float:
    """x^2 with a literal integer exponent: Julia lowers it to x * x (Base.literal_pow)."""
    return x * x


def energy(v) -> float:
    """electron.jl:27."""
    return 0.5 * ELECTRON_MASS * (sq(v[0]) + sq(v[1]) + sq(v[2]))


def randsphere(rng) -> list:
    """util.jl:4-12."""
    phi = 2 * math.pi * rng.rand("phi")
    sinphi, cosphi = math.sin(phi), math.cos(phi)
    u = 2 * rng.rand("u") - 1
    v = math.sqrt(1 - sq(u))
    return [v * cosphi, v * sinphi, u]


class _Role:
    """Renames randsphere's draws to the event roles of the first or second direction."""

    def __init__(self, rng, which: int):
        self.rng, self.which = rng, which

    def rand(self, role: str) -> float:
        return self.rng.rand(("phi" if role == "phi" else "u") + str(self.which))


def nextcoll(rng, role: str = "s") -> float:
    """util.jl:17."""
    return -math.log(rng.rand(role))


def norm3(a) -> float:
    return math.sqrt(sq(a[0]) + sq(a[1]) + sq(a[2]))


@dataclass
class State:
    """ElectronState (electron.jl:9-15)."""

    x: list
    v: list
    w: float
    s: float
    active: bool

    def copy(self) -> "State":
        return State(list(self.x), list(self.v), self.w, self.s, self.active)


def collide(kind: int, par: float, p: State, eng: float, rng):
    """electron.jl:108-139.  Returns (outcome, state1, state2)."""
    m = ELECTRON_MASS
    if kind == EXCITATION:
        E1 = max(0.0, eng - par)
        vabs = math.sqrt(2 * E1 / m)
        d = randsphere(_Role(rng, 1))
        return "change", State(p.x, [c * vabs for c in d], p.w, p.s, p.active), None
    if kind == IONIZATION:
        E1 = max(0.0, eng - par) / 2
        vabs = math.sqrt(2 * E1 / m)
        v = [c * vabs for c in randsphere(_Role(rng, 1))]
        v1 = [c * vabs for c in randsphere(_Role(rng, 2))]
        p1 = State(p.x, v, p.w, p.s, p.active)
        p2 = State(list(p.x), v1, p.w, nextcoll(rng, "s2"), p.active)
        return "new", p1, p2
    if kind == IONIZATION_UNIFORM:
        # the configurations' ionization (not in JuMC): secondary energy uniform on
        # [0, eps - threshold], the share drawn first
        Ea = max(0.0, eng - par)
        E2 = rng.rand("share") * Ea
        E1 = Ea - E2
        va1, va2 = math.sqrt(2 * E1 / m), math.sqrt(2 * E2 / m)
        v = [c * va1 for c in randsphere(_Role(rng, 1))]
        v1 = [c * va2 for c in randsphere(_Role(rng, 2))]
        return "new", State(p.x, v, p.w, p.s, p.active), State(list(p.x), v1, p.w, nextcoll(rng, "s2"), p.active)
    if kind == ATTACHMENT:
        return "remove", p, None
    if kind == ELASTIC:
        f = par / (1 + par)
        v_cm = [f * c for c in p.v]
        nrm = norm3([p.v[q] - v_cm[q] for q in range(3)])
        d = randsphere(_Role(rng, 1))
        return "change", State(p.x, [d[q] * nrm + v_cm[q] for q in range(3)], p.w, p.s, p.active), None
    raise ValueError(f"process kind {kind} is not restated here")


# ---------------------------------------------------------------------------------------
# Populations
# ---------------------------------------------------------------------------------------
class Population:
    """Population (population.jl:4-36): particles 1..n of capacity maxp (0-based storage)."""

    def __init__(self, x, v, w, s, active, maxp: int):
        n = len(w)
        self.maxp = maxp
        self.p = [State([float(c) for c in x[i]], [float(c) for c in v[i]], float(w[i]), float(s[i]), bool(active[i]))
                  for i in range(n)]

    @property
    def n(self) -> int:
        return len(self.p)

    def add_particle(self, st: State) -> int:
        """population.jl:88-97."""
        assert self.n < self.maxp, "Maximum number of particles reached"
        self.p.append(st.copy())
        return self.n - 1

    def remove_particle(self, i: int) -> None:
        """population.jl:104-106."""
        self.p[i].active = False

    def arrays(self):
        n = self.n
        x = np.array([q.x for q in self.p], dtype=np.float64).reshape(n, 3)
        v = np.array([q.v for q in self.p], dtype=np.float64).reshape(n, 3)
        w = np.array([q.w for q in self.p], dtype=np.float64)
        s = np.array([q.s for q in self.p], dtype=np.float64)
        a = np.array([q.active for q in self.p], dtype=np.uint8)
        return x, v, w, s, a


def repack(popl: Population) -> None:
    """population.jl:191-215 (1-based l and i).  The reference throws when nothing is active;
    the population then becomes empty here, as in the library."""
    l = popl.n
    if l == 0:
        return
    while l >= 1 and not popl.p[l - 1].active:
        l -= 1
    if l == 0:
        popl.p = []
        return
    i = 1
    while i <= l:
        if not popl.p[i - 1].active:
            popl.p[i - 1] = popl.p[l - 1].copy()
            l -= 1
            while not popl.p[l - 1].active:
                l -= 1
        i += 1
    del popl.p[l:]


# ---------------------------------------------------------------------------------------
# Fields and trackers
# ---------------------------------------------------------------------------------------
class FixedField:
    """Swarm.jl:28-32: a constant field (given here as its vector)."""

    def __init__(self, e):
        self.e = [float(c) for c in e]

    def __call__(self, x):
        return list(self.e)


class GridCyl:
    """Grid (grid.jl:33-41): rf, zf face ranges and rc, zc centre ranges as LinRanges."""

    def __init__(self, R: float, L: float, M: int, N: int):
        self.R, self.L, self.M, self.N = R, L, M, N
        self.rf = LinRange(0.0, R, M + 1)
        self.zf = LinRange(0.0, L, N + 1)
        self.rc = (self.rf.sub(2, M + 1) + self.rf.sub(1, M)).scale(0.5)
        self.zc = (self.zf.sub(2, N + 1) + self.zf.sub(1, N)).scale(0.5)

    def dr(self) -> float:
        return self.rc.step()

    def dz(self) -> float:
        return self.zc.step()

    def dV(self, i: int) -> float:
        return 2 * math.pi * self.rc[i] * self.dr() * self.dz()

    def inside(self, x) -> bool:
        r = math.sqrt(sq(x[0]) + sq(x[1]))
        return (self.rf[1] < r < self.rf[self.M + 1]) and (self.zf[1] < x[2] < self.zf[self.N + 1])

    def cellindex(self, x) -> tuple[int, int]:
        rho = math.sqrt(sq(x[0]) + sq(x[1]))
        i = int(fld(rho - self.rf.first(), self.rf.step())) + 1
        j = int(fld(x[2] - self.zf.first(), self.zf.step())) + 1
        return i, j


class FieldInterp:
    """gridfields.jl:94-190.  er, ez: face arrays over (0:M+2, 0:N+2), stored as
    [i + (M+3) j] (i fastest)."""

    class TooHigh(Exception):
        pass

    def __init__(self, grid: GridCyl, er, ez):
        self.g = grid
        self.ld = grid.M + 3
        self.er = np.asarray(er, dtype=np.float64).ravel(order="F")
        self.ez = np.asarray(ez, dtype=np.float64).ravel(order="F")

    @staticmethod
    def normdivrem(x, y):
        r = x / y
        m = int(math.trunc(r))
        return m, r - m

    @staticmethod
    def staggered(i, d):
        if d < 1 / 2:
            return i, d + 1 / 2
        return i + 1, d - 1 / 2

    def __call__(self, x):
        g = self.g
        if not g.inside(x):
            return [0.0, 0.0, 0.0]
        r = math.sqrt(sq(x[0]) + sq(x[1]))
        i, dr_ = self.normdivrem(r - g.rf.first(), g.dr())
        i1, dr1 = self.staggered(i, dr_)
        j, dz_ = self.normdivrem(x[2] - g.zf.first(), g.dz())
        j1, dz1 = self.staggered(j, dz_)
        i += 1
        j += 1
        ld = self.ld
        ER = lambda a, b: self.er[a + b * ld]   # noqa: E731
        EZ = lambda a, b: self.ez[a + b * ld]   # noqa: E731
        er1 = (ER(i, j1) * (1 - dr_) * (1 - dz1) + ER(i + 1, j1) * dr_ * (1 - dz1) +
               ER(i, j1 + 1) * (1 - dr_) * dz1 + ER(i + 1, j1 + 1) * dr_ * dz1)
        ez1 = (EZ(i1, j) * (1 - dr1) * (1 - dz_) + EZ(i1 + 1, j) * dr1 * (1 - dz_) +
               EZ(i1, j + 1) * (1 - dr1) * dz_ + EZ(i1 + 1, j + 1) * dr1 * dz_)
        e = [er1 * x[0] / r, er1 * x[1] / r, ez1]
        if norm3(e) > 1e8:
            raise FieldInterp.TooHigh(x)
        return e


class NodeField3D:
    """Trilinear interpolation of node values on an (nx, ny, nz)-cell mesh of spacing h with
    origin (x0, y0, z0); zero outside the open box.  enodes: (nodes, 3), x fastest."""

    def __init__(self, nx, ny, nz, h, origin, enodes):
        self.nx, self.ny, self.nz, self.h = nx, ny, nz, h
        self.o = [float(c) for c in origin]
        self.e = np.asarray(enodes, dtype=np.float64).reshape(-1, 3)

    def __call__(self, x):
        u = [(x[d] - self.o[d]) / self.h for d in range(3)]
        nc = (self.nx, self.ny, self.nz)
        ic, fr = [], []
        for d in range(3):
            if not (0.0 < u[d] < nc[d]):
                return [0.0, 0.0, 0.0]
            fl = math.floor(u[d])
            fl = min(fl, nc[d] - 1)
            ic.append(int(fl))
            fr.append(u[d] - fl)
        sy, sz = self.nx + 1, (self.nx + 1) * (self.ny + 1)
        base = ic[0] + ic[1] * sy + ic[2] * sz
        out = []
        for c in range(3):
            acc = 0.0
            for b in range(8):
                a0, a1, a2 = b & 1, (b >> 1) & 1, (b >> 2) & 1
                wgt = (fr[0] if a0 else 1.0 - fr[0]) * (fr[1] if a1 else 1.0 - fr[1]) * (fr[2] if a2 else 1.0 - fr[2])
                acc += wgt * self.e[base + a0 + a1 * sy + a2 * sz, c]
            out.append(acc)
        return out


class TrackerCyl:
    """CollisionTracker (gridfields.jl:198-224): qfixed over (0:M+1, 0:N+1), one slice."""

    def __init__(self, grid: GridCyl):
        self.g = grid
        self.q = np.zeros((grid.M + 2) * (grid.N + 2))

    def track1(self, x, val) -> None:
        i, j = self.g.cellindex(x)
        if not (0 <= i <= self.g.M + 1 and 0 <= j <= self.g.N + 1):   # checkbounds(qfixed, I)
            return
        if not (1 <= i <= self.g.M):                                  # checkbounds(grid.rc, i)
            return
        self.q[i + j * (self.g.M + 2)] += val / self.g.dV(i)


class TrackerNodes3D:
    """Int64 CIC at 2^-32 e on the nodes of the 3-D mesh: the charge W = round(q 2^32) is
    split over the cell's 8 nodes with weights (gx gy) gz, seven corners rounded and the
    last taking the remainder, so a node sum is exactly W."""

    def __init__(self, nx, ny, nz, h, origin):
        self.nx, self.ny, self.nz, self.h = nx, ny, nz, h
        self.o = [float(c) for c in origin]
        self.q = np.zeros((nx + 1) * (ny + 1) * (nz + 1), dtype=np.int64)

    def locate(self, x):
        u = [(x[d] - self.o[d]) / self.h for d in range(3)]
        nc = (self.nx, self.ny, self.nz)
        ic, fr = [], []
        for d in range(3):
            fl = math.floor(u[d])
            if not (0 <= fl < nc[d]):
                return None
            ic.append(int(fl))
            fr.append(u[d] - fl)
        return ic, fr

    def deposit(self, ic, fr, charge) -> None:
        W = int(np.rint(charge * 2.0 ** 32))
        Wd = float(W)
        g = [(1.0 - fr[0], fr[0]), (1.0 - fr[1], fr[1]), (1.0 - fr[2], fr[2])]
        sy, sz = self.nx + 1, (self.nx + 1) * (self.ny + 1)
        base = ic[0] + ic[1] * sy + ic[2] * sz
        acc = 0
        for b in range(7):
            a0, a1, a2 = b & 1, (b >> 1) & 1, (b >> 2) & 1
            qb = int(np.rint(Wd * ((g[0][a0] * g[1][a1]) * g[2][a2])))
            acc += qb
            self.q[base + a0 + a1 * sy + a2 * sz] += qb
        self.q[base + 1 + sy + sz] += W - acc

    def track1(self, x, val) -> None:
        loc = self.locate(x)
        if loc is not None:
            self.deposit(loc[0], loc[1], val)


# ---------------------------------------------------------------------------------------
# advance!, do_one_collision!, collisions!
# ---------------------------------------------------------------------------------------
YW0 = -2 ** (1 / 3) / (2 - 2 ** (1 / 3))
YW1 = 1 / (2 - 2 ** (1 / 3))
YC1 = YW1 / 2
YC2 = (YW0 + YW1) / 2
YC3 = YC2
YC4 = YC1
YD1 = YW1
YD2 = YW0
YD3 = YD1


def advance_free_yoshida(p: State, efield, dt: float) -> State:
    """electron.jl:51-62."""
    qm = (-ELEMENTARY_CHARGE) / ELECTRON_MASS
    x1 = [p.x[q] + YC1 * dt * p.v[q] for q in range(3)]
    E = efield(x1)
    v1 = [p.v[q] + YD1 * dt * qm * E[q] for q in range(3)]
    x2 = [x1[q] + YC2 * dt * v1[q] for q in range(3)]
    E = efield(x2)
    v2 = [v1[q] + YD2 * dt * qm * E[q] for q in range(3)]
    x3 = [x2[q] + YC3 * dt * v2[q] for q in range(3)]
    E = efield(x3)
    v3 = [v2[q] + YD3 * dt * qm * E[q] for q in range(3)]
    x4 = [x3[q] + YC4 * dt * v3[q] for q in range(3)]
    return State(x4, v3, p.w, p.s, p.active)


def do_one_collision(popl: Population, tab: Table, state: State, i: int, tracker, rng) -> None:
    """collisions.jl:159-192 (the generated scan over rows j = 1..L), with track and apply!."""
    eng = energy(state.v)
    pre = indweight(tab.energy, eng)
    xi = rng.rand("xi") * tab.maxrate
    for j in range(1, len(tab.kinds) + 1):
        nu = rate(tab, j, pre)
        if nu > xi:
            kind = tab.kinds[j - 1]
            if kind == NULL:
                return                                   # NullOutcome: track/apply! do nothing
            out, s1, s2 = collide(kind, tab.params[j - 1], state, eng, rng)
            if out == "change":                          # apply!(StateChangeOutcome)
                popl.p[i] = s1.copy()
            elif out == "new":
                if tracker is not None:
                    tracker.track1(s1.x, s1.w)           # track(NewParticleOutcome): +w
                popl.p[i] = s1.copy()                    # apply!(NewParticleOutcome)
                popl.add_particle(s2)
            elif out == "remove":
                if tracker is not None:
                    tracker.track1(s1.x, -s1.w)          # track(RemoveParticleOutcome): -w
                popl.remove_particle(i)
            return
        xi -= nu


def advance(popl: Population, tab: Table, efield, dt: float, tracker=None,
            draws: Optional[Callable[[int], object]] = None) -> None:
    """advance! (mixed_population.jl:24-54) of one population, serially over i = 1..n.
    draws(i) gives particle i's uniform source (0-based i)."""
    n = popl.n
    for i in range(n):
        if not popl.p[i].active:
            continue
        rng = draws(i)
        trem = dt
        while trem > 0:
            l = popl.p[i]
            tnextcoll = l.s / tab.maxrate
            if trem > tnextcoll:
                t = tnextcoll
                collides = True
            else:
                t = trem
                collides = False
                l.s -= t * tab.maxrate
            new_state = advance_free_yoshida(l, efield, t)
            popl.p[i] = new_state
            if collides:
                do_one_collision(popl, tab, new_state, i, tracker, rng)
                popl.p[i].s = nextcoll(rng, "s")
            trem -= t


def collisions(popl: Population, tab: Table, dt: float, tracker=None,
               draws: Optional[Callable[[int], object]] = None) -> None:
    """collisions! (mixed_population.jl:61-77)."""
    for i in range(popl.n):
        l = popl.p[i]
        if not l.active:
            continue
        l.s -= dt * tab.maxrate
        if l.s <= 0:
            rng = draws(i)
            do_one_collision(popl, tab, l.copy(), i, tracker, rng)
            popl.p[i].s = nextcoll(rng, "s")


def philox_draws(seed: int, step: int, tag: int = TAG_ADVANCE):
    return lambda i: PhiloxEventDraws(seed, i, step, tag)


# ---------------------------------------------------------------------------------------
# Swarm.resample!, resample!, density!
# ---------------------------------------------------------------------------------------
def poisson_draw(rng, lam: float) -> int:
    """The library's Poisson sampler (the reference draws Distributions.Poisson; only the law
    is matched): inversion of the cdf below lam = 10; above, PTRS, the transformed
    rejection method of Hoermann (1993), with its published constants."""
    if lam <= 0:
        return 0
    if lam < 10.0:
        u = rng.rand()
        pr = math.exp(-lam)
        F = pr
        k = 0
        while u > F and k < 1000:
            k += 1
            pr *= lam / k
            F += pr
        return k
    slam, loglam = math.sqrt(lam), math.log(lam)
    b = 0.931 + 2.53 * slam
    a = -0.059 + 0.02483 * b
    invalpha = 1.1239 + 1.1328 / (b - 3.4)
    vr = 0.9277 - 3.6224 / (b - 2.0)
    for _ in range(1000):
        U = rng.rand() - 0.5
        V = rng.rand()
        us = 0.5 - abs(U)
        kf = math.floor((2.0 * a / us + b) * U + lam + 0.43)
        if us >= 0.07 and V <= vr:
            return int(kf)
        if kf < 0 or (us < 0.013 and V > us):
            continue
        if math.log(V) + math.log(invalpha) - math.log(a / (us * us) + b) <= -lam + kf * loglam - math.lgamma(kf + 1.0):
            return int(kf)
    return int(math.floor(lam))


def swarm_resample(popl: Population, n0: int, tol: float, seed: int, call: int) -> None:
    """Swarm.jl:193-223.  Particle i's draws: Stream(seed, i, call, TAG_SWARM_RESAMPLE)."""
    ncur = sum(1 for q in popl.p if q.active)
    if abs((ncur - n0) / n0) < tol:
        return
    n_entry = popl.n
    if ncur > n0:
        for i in range(n_entry):
            if not popl.p[i].active:
                continue
            if Stream(seed, i, call, TAG_SWARM_RESAMPLE).rand() < (ncur - n0) / ncur:
                popl.remove_particle(i)
    else:
        for i in range(n_entry):
            if not popl.p[i].active:
                continue
            nnew = poisson_draw(Stream(seed, i, call, TAG_SWARM_RESAMPLE), (n0 - ncur) / ncur)
            for _ in range(nnew):
                popl.add_particle(popl.p[i])


def samplemin(rng, m: float) -> float:
    """resample.jl:84."""
    return 1 - (1 - rng.rand()) ** (1 / m)


def resample(popl: Population, cellindex: Callable, ntarget: int, nmax: int, seed: int, call: int) -> None:
    """resample.jl:7-77.  cellindex(x) gives a cell key or None (checkbounds fails); cell c's
    draws come from Stream(seed, c, call, TAG_CELL_RESAMPLE), in the order the serial passes
    visit its particles."""
    p, pk, wtotal, wcum, x, rngs = {}, {}, {}, {}, {}, {}
    n = popl.n
    keys = [None] * n
    for i in range(n):
        k = popl.p[i]
        if not k.active:
            continue
        I = cellindex(k.x)
        keys[i] = I
        if I is None:
            continue
        if I not in p:
            p[I], pk[I], wtotal[I], wcum[I], x[I] = 0, 0, 0.0, 0.0, 0.0
            rngs[I] = Stream(seed, I, call, TAG_CELL_RESAMPLE)
        p[I] += 1
        wtotal[I] += k.w
        if p[I] == nmax:
            x[I] = samplemin(rngs[I], ntarget)
    for i in range(n):
        k = popl.p[i]
        if not k.active:
            continue
        I = keys[i]
        if I is None:
            continue
        if p[I] > nmax:
            while (wtotal[I] * x[I] < wcum[I] + k.w) and pk[I] < ntarget:
                pk[I] += 1
                index = popl.add_particle(popl.p[i])
                popl.p[index].w = wtotal[I] / ntarget
                if pk[I] < ntarget:
                    x[I] += samplemin(rngs[I], ntarget - pk[I]) * (1 - x[I])
            wcum[I] += k.w
            popl.remove_particle(i)
        elif p[I] < ntarget and k.w > 2:
            wnew = float(round(k.w / 2))
            index = popl.add_particle(popl.p[i])
            popl.p[index].w = wnew
            k.w = k.w - wnew
            p[I] += 1


def cell_key_cyl(grid: GridCyl):
    """cellindex on (0:M+1, 0:N+1) as the linear key i + (M+2) j, None outside."""
    def f(x):
        i, j = grid.cellindex(x)
        if not (0 <= i <= grid.M + 1 and 0 <= j <= grid.N + 1):
            return None
        return i + (grid.M + 2) * j
    return f


def cell_key_3d(nx, ny, nz, h, origin):
    def f(x):
        ic = []
        for d, nc in enumerate((nx, ny, nz)):
            fl = math.floor((x[d] - origin[d]) / h)
            if not (0 <= fl < nc):
                return None
            ic.append(int(fl))
        return ic[0] + nx * (ic[1] + ny * ic[2])
    return f


def density_cyl(grid: GridCyl, popl: Population, val: float) -> np.ndarray:
    """density! (poisson.jl:65-84) into a fresh (0:M+1, 0:N+1) array."""
    arr = np.zeros((grid.M + 2) * (grid.N + 2))
    for q in popl.p:
        if not q.active:
            continue
        i, j = grid.cellindex(q.x)
        if not (0 <= i <= grid.M + 1 and 0 <= j <= grid.N + 1):
            continue
        if not (1 <= i <= grid.M):
            continue
        arr[i + j * (grid.M + 2)] += q.w * val / grid.dV(i)
    return arr


def sort_by_cell(popl: Population, cellindex: Callable) -> None:
    """Stable sort by cell key; inactive and outside particles last (the library sorts before
    resample!, so its serial pass order is the cell order)."""
    big = float("inf")

    def key(q):
        if not q.active:
            return big
        k = cellindex(q.x)
        return big if k is None else k
    popl.p = sorted(popl.p, key=key)
