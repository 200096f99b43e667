"""Run a streamer from the reference's TOML input: MCStreamer.main(finput)
(MCStreamer/src/main.jl:15-196) over the device.

`main(finput)` reads the same keys as the reference and sets up the same objects:

* the grid from [domain] (R, L, M, N), the collision table from `cross_sections` (paths
  relative to the input file) with N2 and O2 at 0.79 and 0.21 of `nair`, on the energy grid
  LinRange(0, 1000 eV, 100000), and the photo-emission parameters of [photoionization];
* the background field from `eb` and `field_units` (geteb, main.jl:349-360);
* the electrons: without [init_files], `n` electrons at rest from sampseg(z0, z1, w) of
  [seed], of weight `initial_weight`, whose charge goes into qfixed (main.jl:88-94,126-128);
  with [init_files], initfromfiles! with the `method`, `format` and `fluid_threshold` given
  there (main.jl:95-112);
* a photon population when the table has a photo-emission process (main.jl:115-121);
* the needle fluid of [needle] (main.jl:169-179);
* the multigrid with `poisson_levels` (main.jl:130-148);

then runs nsteps for fld(tmax, dt) steps with the intervals of [interval], writing the
output files next to the input (main.jl:152-193).  `rng_seed` keys the random streams.

Not carried over: the TensorFlow denoiser ([denoise]); an input that names one runs with the
NullDenoiser and a warning.  `maxp` sizes the electron and photon populations; `capacity`
and `photon_capacity` override it, since the reference's host arrays can be far larger
than a device population needs to be.
"""
from __future__ import annotations

import math
import os
import tomllib
import warnings
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _lib as L
from . import constants as co
from . import jumc, loop, lxcat, streamer
from .fluid import Fluid
from .initdens import AfivoLoader, AMLoader, NoiselessInitSampling, PoissonInitSampling, initfromfiles
from .poisson import MGConfig, PoissonSolver

FIELD_UNITS = {"kV/cm": 1e5, "MV/m": 1e6, "V/m": 1.0, "": 1.0}


def geteb(inp: dict) -> float:
    """geteb(input) (main.jl:349-360): -eb in V/m."""
    units = inp.get("field_units", "Td")
    nair = float(inp.get("nair", co.nair))
    scale = co.Td * nair if units == "Td" else FIELD_UNITS[units]
    return -float(inp["eb"]) * scale


def sampseg(z0: float, z1: float, w: float, n: int, rng: np.random.Generator) -> np.ndarray:
    """n draws of sampseg(z0, z1, w) (main.jl:320-341): a segment on the axis blurred by a
    Gaussian of width w."""
    if not z1 >= z0:
        raise ValueError("sampseg needs z1 >= z0")
    length = z1 - z0
    p = length / (length + math.sqrt(2 * math.pi) * w)
    x = np.empty((n, 3))
    for k in range(n):
        if rng.random() < p:
            u = rng.random()
            x[k] = (w * rng.standard_normal(), w * rng.standard_normal(), z0 + u * length)
        else:
            s = w * rng.standard_normal(3)
            x[k] = s + (0.0, 0.0, z1 if s[2] > 0 else z0)
    return x


@dataclass
class Run:
    """What main returns: the device objects and the per-step diagnostics."""
    streamer: loop.Streamer
    table: jumc.CollisionTable
    eb: float
    dt: float
    steps: int
    diagnostics: List[dict]
    outpath: str

    def close(self) -> None:
        s = self.streamer
        s.efield.close()
        if s.photons is not None:
            s.photons.close()
        if s.fluid is not None:
            s.fluid.close()
        s.electrons.close()
        s.solver.close()
        s.grid.close()
        self.table.close()


def read_input(finput: str, tmax: Optional[float] = None) -> dict:
    """The settings main takes from the input file, resolved as main.jl does: the parsed
    TOML under "input", with the cross-section and init-file paths made relative to the
    input's folder, the background field eb (V/m), the number of steps fld(tmax, dt), the
    Poisson levels and the output path."""
    with open(finput, "rb") as f:
        inp = tomllib.load(f)
    here = os.path.dirname(os.path.abspath(finput))
    dt = float(inp["dt"])
    tmax = float(inp["tmax"]) if tmax is None else float(tmax)
    out = {"input": inp, "here": here, "dt": dt, "tmax": tmax, "steps": int(tmax // dt),   # fld(tmax, dt)
           "eb": geteb(inp), "seed": int(inp.get("rng_seed", 0)), "nair": float(inp.get("nair", co.nair)),
           "poisson_levels": int(inp.get("poisson_levels", 9)),
           "cross_sections": [os.path.join(here, f) for f in inp["cross_sections"]],
           "outpath": os.path.splitext(os.path.abspath(finput))[0]}
    if "init_files" in inp:
        init = inp["init_files"]
        out["init_files"] = {"ne_file": os.path.join(here, init["ne_file"]),
                             "q_file": os.path.join(here, init["q_file"]),
                             "method": init.get("method", "noiseless"), "format": init.get("format", "am"),
                             "fluid_threshold": float(init.get("fluid_threshold", math.inf))}
    return out


def main(finput: str, tmax: Optional[float] = None, run: bool = True, precision: str = "fp32",
         capacity: Optional[int] = None, photon_capacity: Optional[int] = None,
         ctx: Optional[jumc.Context] = None) -> Run:
    """MCStreamer.main(finput; tmax, run) on the device."""
    cfg = read_input(finput, tmax)
    inp = cfg["input"]
    here = cfg["here"]
    ctx = ctx or jumc.Context.default()
    seed, nair = cfg["seed"], cfg["nair"]
    dom = inp["domain"]
    R, Lz, M, N = float(dom["R"]), float(dom["L"]), int(dom["M"]), int(dom["N"])
    nmax, ntarget, maxp, n = int(inp["nmax"]), int(inp["ntarget"]), int(float(inp["maxp"])), int(inp["n"])
    pi = inp.get("photoionization", {})
    table = lxcat.load_lxcat(cfg["cross_sections"],
                             {"N2": nair * 0.79, "O2": nair * 0.21}, lxcat.DEFAULT_ENERGY,
                             photon_weight=float(pi.get("photon_weight", 1.0)),
                             photon_multiplier=float(pi.get("photon_multiplier", 1.0)))
    tab = jumc.CollisionTable(table, ctx)
    dt, eb = cfg["dt"], cfg["eb"]
    if "denoise" in inp:
        warnings.warn("the [denoise] model is not supported; poisson! runs with the NullDenoiser")

    grid = streamer.GridCyl(R, Lz, M, N, ctx=ctx)
    solver = PoissonSolver(grid, MGConfig(levels=cfg["poisson_levels"]))
    cap = int(capacity) if capacity is not None else maxp
    try:
        electrons = jumc.Population(cap, None, tab, precision=precision, seed=seed)
    except L.MCSError as e:
        solver.close(); grid.close(); tab.close()
        if e.code != L.ERR_NOMEM:
            raise
        raise L.MCSError(e.code, f"{cap} electrons do not fit on the device (maxp = {maxp} sizes the "
                                 f"reference's host arrays); pass capacity= and photon_capacity=") from e
    fluid = None
    if "init_files" in cfg:
        init = cfg["init_files"]
        method = {"poisson": PoissonInitSampling, "noiseless": NoiselessInitSampling}[init["method"]](ntarget)
        loader = {"am": AMLoader, "afivo": AfivoLoader}[init["format"]](init["ne_file"], init["q_file"])
        threshold = init["fluid_threshold"]
        if math.isfinite(threshold):
            fluid = Fluid(grid)
        initfromfiles(method, grid, electrons, loader, fluid_threshold=threshold, seed=seed)
    else:
        sd = inp["seed"]
        z0 = float(sd["z0"])
        z1 = float(sd.get("z1", z0))
        x = sampseg(z0, z1, float(sd["w"]), n, np.random.default_rng(seed))
        p = jumc.ParticleArrays(x, np.zeros((n, 3)), np.full(n, float(inp.get("initial_weight", 1.0))),
                                -np.log(np.random.default_rng(seed + 1).random(n)), np.ones(n, np.uint8))
        electrons.upload(p)
        # density!(grid, qfixed, mpopl, Electron, fields, 1.0): the seed's ions
        grid.zero(L.Q_PART)
        streamer.density(grid, electrons, 1.0)
        grid.write_fixed(L.Q_FIXED, grid.read_fixed(L.Q_PART))
        grid.zero(L.Q_PART)
    if "needle" in inp:
        nd = inp["needle"]
        fluid = fluid or Fluid(grid)
        fluid.set_needle(float(nd["sigma_z"]), float(nd["sigma_r"]), float(nd["position_z"]),
                         float(nd["position_r"]), float(nd["ne0"]))
    photons = None
    if table.has_photoemission:
        photons = jumc.Photons(int(photon_capacity) if photon_capacity is not None else maxp, table.photon_numax,
                               seed=seed + 1, ctx=ctx)
    # main.jl:173-180 sets hasfluid from [needle] alone, after initfromfiles! set it for a
    # finite fluid_threshold: an init-file fluid without a needle is never stepped
    s = loop.Streamer(grid, solver, electrons, streamer.FieldInterp(grid), photons, fluid,
                      hasfluid="needle" in inp)
    outpath = cfg["outpath"]
    iv = inp["interval"]
    steps = cfg["steps"]
    diags: List[dict] = []
    if run:
        diags = loop.nsteps(s, steps, ntarget, nmax, eb, dt, float(iv["poisson"]), float(iv["output"]),
                            float(iv["resample"]), outpath=outpath)
    return Run(s, tab, eb, dt, steps, diags, outpath)
