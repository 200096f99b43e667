"""Cross-section input: load_lxcat (JuMC/src/lxcat.jl:17-134) and the synthetic gases.

load_lxcat reads LXCat-format JSON records (kind, target, threshold | mass_ratio,
comment, data=[[eV, m^2], ...]; the format of JuMC/data/LXCat-June2013.json), turns each
cross section into a collision rate nu_j(eps) = N * v(eps) * sigma_j(eps) on a uniform
energy grid, adds the null-collision row and sorts the rows by their sum over the grid.
The result feeds mcs_table_create unchanged (CollisionTable, collisions.jl:9-22).

PHOTOEMISSION records (lxcat.jl:57-60,86-93) give rows of kind PHOTOEMISSION: their cross
section is scaled by photon_multiplier, and their absorption band nu_min..nu_max = c *
N(absorber) * chi_min..chi_max is kept as log(nu) per row (PhotoEmission, electron.jl:88-105);
photon_numax is the photon population's maxrate (MCStreamer/src/main.jl:115-118).
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable, Mapping, Sequence

import numpy as np

from . import constants as co
from ._lib import ATTACHMENT, ELASTIC, EXCITATION, IONIZATION, IONIZATION_UNIFORM, NULL, PHOTOEMISSION

KIND_NAMES = {NULL: "NULL", ELASTIC: "ELASTIC", EXCITATION: "EXCITATION", IONIZATION: "IONIZATION",
              ATTACHMENT: "ATTACHMENT", IONIZATION_UNIFORM: "IONIZATION_UNIFORM", PHOTOEMISSION: "PHOTOEMISSION"}


@dataclass(frozen=True)
class EnergyGrid:
    """LinRange(e0, emax, n) in joules."""

    e0: float
    emax: float
    n: int

    def values(self) -> np.ndarray:
        # Base.LinRange getindex: lerpi(j, lendiv, start, stop) = (1 - j/lendiv)*a + (j/lendiv)*b
        lendiv = float(self.n - 1)
        t = np.arange(self.n, dtype=np.float64) / lendiv
        return (1.0 - t) * self.e0 + t * self.emax

    @property
    def step(self) -> float:
        return (self.emax - self.e0) / float(self.n - 1)


# Swarm.jl:66 and MCStreamer main.jl:52: LinRange(0, 1000 eV, 100_000)
DEFAULT_ENERGY = EnergyGrid(0.0, 1000 * co.eV, 100_000)


@dataclass
class Process:
    kind: int
    param: float          # threshold (J) or mass ratio
    target: str
    signature: str
    lmin: float = 0.0     # PHOTOEMISSION: log(nu_min), log(nu_max) (1/s)
    lmax: float = 0.0


@dataclass
class LXCatTable:
    """Return value of load_lxcat: (proc, rate, maxrate, origperm) of lxcat.jl:133."""

    proc: list[Process]
    rate: np.ndarray       # (nrows, neps), rows sorted by integral (descending)
    maxrate: float
    origperm: np.ndarray   # invperm(perm)
    energy: EnergyGrid
    perm: np.ndarray = field(default=None)
    photon_multiplier: float = 1.0
    photon_weight: float = 1.0

    @property
    def kinds(self) -> np.ndarray:
        return np.array([p.kind for p in self.proc], dtype=np.int32)

    @property
    def has_photoemission(self) -> bool:
        return any(p.kind == PHOTOEMISSION for p in self.proc)

    @property
    def pe_lmin(self) -> np.ndarray:
        return np.array([p.lmin for p in self.proc], dtype=np.float64)

    @property
    def pe_lmax(self) -> np.ndarray:
        return np.array([p.lmax for p in self.proc], dtype=np.float64)

    @property
    def photon_numax(self) -> float:
        """ZhelezniakCollisions(exp(log_numax)) of the first PhotoEmission row
        (MCStreamer/src/main.jl:115-118)."""
        for p in self.proc:
            if p.kind == PHOTOEMISSION:
                return float(np.exp(p.lmax))
        raise ValueError("no PHOTOEMISSION process")

    @property
    def params(self) -> np.ndarray:
        return np.array([p.param for p in self.proc], dtype=np.float64)

    def rate_energy_major(self) -> np.ndarray:
        """(neps, nrows) C-contiguous == Julia's column-major (nrows, neps) memory layout."""
        return np.ascontiguousarray(self.rate.T)


def _interp_flat(x0: np.ndarray, y0: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Piecewise-linear interpolation on knots x0 with flat extrapolation, the semantics of
    extrapolate(interpolate((x0,), y0, Gridded(Linear())), Flat()) (Interpolations.jl)."""
    x0 = np.asarray(x0, dtype=np.float64)
    y0 = np.asarray(y0, dtype=np.float64)
    out = np.empty_like(x)
    lo = x <= x0[0]
    hi = x >= x0[-1]
    out[lo] = y0[0]
    out[hi] = y0[-1]
    mid = ~(lo | hi)
    xm = x[mid]
    i = np.searchsorted(x0, xm, side="right") - 1
    i = np.clip(i, 0, len(x0) - 2)
    t = (xm - x0[i]) / (x0[i + 1] - x0[i])
    out[mid] = (1.0 - t) * y0[i] + t * y0[i + 1]
    return out


def _kind_of(item: Mapping) -> int:
    k = item["kind"]
    if k == "ELASTIC":
        return ELASTIC
    if k == "EXCITATION":
        return EXCITATION
    if k == "IONIZATION":
        return IONIZATION_UNIFORM if item.get("sharing") == "uniform" else IONIZATION
    if k == "ATTACHMENT":
        return ATTACHMENT
    if k == "PHOTOEMISSION":
        return PHOTOEMISSION
    raise ValueError(f"unknown process kind {k!r}")


def _signature(item: Mapping) -> str:
    # lxcat.jl:159-164
    product = item.get("product", "")
    return f"e + {item['target']} -> {product}... ({item['kind']})"


def load_lxcat_records(db: Sequence[Mapping], densities: Mapping[str, float],
                       energy: EnergyGrid = DEFAULT_ENERGY, photon_weight: float = 1.0,
                       photon_multiplier: float = 1.0) -> LXCatTable:
    """load_lxcat on already-parsed records (lxcat.jl:17-134)."""
    eng = energy.values()
    v = np.sqrt(2.0 * eng / co.electron_mass)
    targets: dict[str, list[dict]] = {}
    nprocs = 0
    for raw in db:
        item = dict(raw)
        dens = float(densities.get(item["target"], 0.0))
        if dens == 0.0:
            continue
        tgt = targets.setdefault(item["target"], [])
        data = np.asarray(item["data"], dtype=np.float64)
        energy0 = data[:, 0] * co.eV
        cs0 = data[:, 1].copy()
        if "3-body" in item.get("comment", ""):
            cs0 *= densities[item["target"]] / co.centi ** -3
        if "rescale" in item:
            cs0 *= item["rescale"]
        if "weight_scale" in item:
            cs0 *= item["weight_scale"]
        if item["kind"] == "PHOTOEMISSION":
            cs0 *= photon_multiplier
        item["nu"] = dens * v * _interp_flat(energy0, cs0, eng)
        tgt.append(item)
        nprocs += 1

    proc: list[Process] = []
    rate = np.zeros((nprocs + 1, energy.n), dtype=np.float64)
    i = 0
    for name, ps in targets.items():
        # ensure_elastic, lxcat.jl:146-156
        for p in ps:
            if p["kind"] != "EFFECTIVE":
                continue
            for p2 in ps:
                if p2 is not p and p2["kind"] in ("EXCITATION", "IONIZATION"):
                    p["nu"] = p["nu"] - p2["nu"]
            p["kind"] = "ELASTIC"
        for item in ps:
            kind = _kind_of(item)
            par = float(item["mass_ratio"]) if kind == ELASTIC else float(item.get("threshold", 0.0)) * co.eV
            pr = Process(kind, par, name, _signature(item))
            if kind == PHOTOEMISSION:
                par = 0.0
                nu_abs = co.speed_of_light * densities[item["absorber"]]
                pr = Process(kind, 0.0, name, _signature(item), float(np.log(nu_abs * item["chi_min"])),
                             float(np.log(nu_abs * item["chi_max"])))
            proc.append(pr)
            rate[i, :] = item["nu"]
            i += 1

    nutotal = rate.sum(axis=0)
    maxrate = float(nutotal.max())
    rate[nprocs, :] = maxrate - nutotal
    proc.append(Process(NULL, 0.0, "", "null collision"))
    inteng = rate.sum(axis=1)
    perm = np.argsort(-inteng, kind="stable")      # sortperm(inteng, rev=true)
    origperm = np.argsort(perm, kind="stable")      # invperm(perm)
    return LXCatTable([proc[k] for k in perm], np.ascontiguousarray(rate[perm, :]), maxrate, origperm,
                      energy, perm, photon_multiplier, photon_weight)


def load_lxcat(fnames: Iterable[str | Path], densities: Mapping[str, float],
               energy: EnergyGrid = DEFAULT_ENERGY, photon_weight: float = 1.0,
               photon_multiplier: float = 1.0) -> LXCatTable:
    """load_lxcat(fnames, densities, energy; photon_weight, photon_multiplier)
    (JuMC/src/lxcat.jl:17)."""
    db: list[dict] = []
    for fn in fnames:
        with open(fn) as fd:
            db.extend(json.load(fd))
    return load_lxcat_records(db, densities, energy, photon_weight, photon_multiplier)


# ---------------------------------------------------------------------------------------
# Synthetic gases of the benchmark configurations, written as LXCat records.
# ---------------------------------------------------------------------------------------
SYNTHETIC_DENSITY = 2.5e25  # m^-3
LOG_GRID_EV = np.logspace(-3.0, 3.0, 1000)


def _ramp(e: np.ndarray, th: float, top_e: float, top: float) -> np.ndarray:
    s = np.where(e < th, 0.0, top * (e - th) / (top_e - th))
    return np.where(e >= top_e, top, s)


def synthetic_records(variant: int = 0, target: str = "SYN", uniform_sharing: bool = True) -> list[dict]:
    """The synthetic gases of the workloads, sampled on a 1000-point log grid 1e-3..1e3 eV.

    variant 0: elastic 6e-20 m^2 (m/M = 1.96e-5); excitations at 6.2/8.4/11.0 eV rising
               linearly to 1e-21 m^2 at twice threshold, then flat; ionization at 15.6 eV
               rising linearly to 2.5e-20 m^2 at 100 eV, then flat, secondary energy uniform
               on [0, eps - 15.6 eV]; attachment 1e-22 m^2 below 3 eV.
    variant 1: as 0 with ionization threshold 12.1 eV and attachment 5e-22 m^2.
    variant 2: as 0 with twice the elastic cross section.
    variant 3: as 0 with five excitation levels at 2, 4.5, 7, 9.5 and 12 eV.
    """
    e = LOG_GRID_EV
    el = 6e-20 * (2.0 if variant == 2 else 1.0)
    exc = [2.0, 4.5, 7.0, 9.5, 12.0] if variant == 3 else [6.2, 8.4, 11.0]
    ion_th = 12.1 if variant == 1 else 15.6
    att = 5e-22 if variant == 1 else 1e-22

    def rec(kind, sig, **kw):
        r = {"kind": kind, "target": target, "comment": f"synthetic gas {variant}",
             "data": [[float(a), float(b)] for a, b in zip(e, sig)]}
        r.update(kw)
        return r

    recs = [rec("ELASTIC", np.full_like(e, el), mass_ratio=1.96e-5)]
    for th in exc:
        recs.append(rec("EXCITATION", _ramp(e, th, 2 * th, 1e-21), threshold=th, product=f"{target}*{th}"))
    ion = rec("IONIZATION", _ramp(e, ion_th, 100.0, 2.5e-20), threshold=ion_th, product=f"{target}+")
    if uniform_sharing:
        ion["sharing"] = "uniform"
    recs.append(ion)
    recs.append(rec("ATTACHMENT", np.where(e < 3.0, att, 0.0), threshold=0.0, product=f"{target}-"))
    return recs


def synthetic_table(variant: int = 0, energy: EnergyGrid = DEFAULT_ENERGY, density: float = SYNTHETIC_DENSITY,
                    uniform_sharing: bool = True) -> LXCatTable:
    return load_lxcat_records(synthetic_records(variant, uniform_sharing=uniform_sharing), {"SYN": density}, energy)


def synthetic_photo_records(target: str = "SYN", absorber: str = "ABS", chi_min: float = 1e-23,
                            chi_max: float = 6e-21, rescale: float = 2e-3) -> list[dict]:
    """A synthetic PHOTOEMISSION record in the format the reference reads (kind, target,
    absorber, chi_min, chi_max, rescale; lxcat.jl:57-60,86-93): a cross section rising
    linearly from 15.6 eV to 2.5e-20 m^2 at 100 eV, then flat, on the log grid."""
    e = LOG_GRID_EV
    return [{"kind": "PHOTOEMISSION", "target": target, "absorber": absorber, "chi_min": chi_min,
             "chi_max": chi_max, "rescale": rescale, "comment": "synthetic photo-emission",
             "data": [[float(a), float(b)] for a, b in zip(e, _ramp(e, 15.6, 100.0, 2.5e-20))]}]


def synthetic_photo_table(variant: int = 0, energy: EnergyGrid = DEFAULT_ENERGY, density: float = SYNTHETIC_DENSITY,
                          absorber_density: float = 0.2 * SYNTHETIC_DENSITY, photon_weight: float = 1.0,
                          photon_multiplier: float = 1000.0, **photo) -> LXCatTable:
    """Synthetic gas `variant` plus one photo-emission process whose photons are absorbed by a
    species of density `absorber_density` (the reference's sample input uses
    photon_multiplier = 1000, photon_weight = 1)."""
    recs = synthetic_records(variant) + synthetic_photo_records(**photo)
    return load_lxcat_records(recs, {"SYN": density, "ABS": absorber_density}, energy, photon_weight,
                              photon_multiplier)
