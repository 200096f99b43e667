"""The streamer loop: `nsteps` (MCStreamer/src/main.jl:218-318) over the device state.

Every step i (t = (i - 1) dt), in the reference's order:

1. at the Poisson times: poisson! (density! of the electrons into qpart, the charge, the
   free-boundary solve and the face fields; the potential warm-starts from the last solve);
2. at the output times: savefields (h5export's layout) and the output line;
3. advance!(mpopl, efield, dt, tracker) over electrons and, when present, photons;
4. the per-step diagnostics line (main.jl:269-279);
5. at the resample times: repack!(photons), repack!(electrons), resample!(electrons,
   ntarget, nmax), with the reference's weight-conservation checks (rtol 1e-5);
6. with a fluid: setdne! + euler!;
7. repack!(electrons).

`TimeStepper` is timesteps.jl's: `atstep` fires when t >= step * i and then counts i up; the
resample stepper is built as TimeStepper(dt, dt_resample), whose start the reference never
reads, and so is this one.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Callable, List, Optional

from . import fieldsio, jumc
from .streamer import CollisionTracker, GridCyl, density, diagnostics, reserve_resample, resample


class TimeStepper:
    """timesteps.jl:5-28."""

    def __init__(self, step: float, start: Optional[float] = None):
        self.i = 0
        self.start = 0.0 * step if start is None else start
        self.step = step

    def atstep(self, t: float) -> Optional[int]:
        """The counter before the increase when it is time, else None."""
        if t >= self.step * self.i:
            i = self.i
            self.i += 1
            return i
        return None


@dataclass
class Streamer:
    """The device objects nsteps works on (the reference's mpopl, efield, fields, mg, ws)."""
    grid: GridCyl
    solver: object                      # poisson.PoissonSolver
    electrons: jumc.Population
    efield: object                      # streamer.FieldInterp(grid)
    photons: Optional[jumc.Photons] = None
    fluid: Optional[object] = None      # fluid.Fluid: its ne enters poisson!'s charge (poisson.jl:24)
    tracker: Optional[CollisionTracker] = None
    # the reference's hasfluid (MCStreamer/src/main.jl:173-180): setdne! + euler! run only
    # when the input has a [needle]; an init-file fluid without one keeps its ne fixed
    hasfluid: Optional[bool] = None
    log: List[dict] = field(default_factory=list)

    def __post_init__(self):
        if self.tracker is None:
            self.tracker = CollisionTracker(self.grid)
        if self.hasfluid is None:
            self.hasfluid = self.fluid is not None


def poisson_step(s: Streamer, eb: float):
    """poisson!(fields, mpopl, eb, mg, ws, NullDenoiser(), t, outpath) (poisson.jl:6-58)."""
    from . import _lib as L
    s.grid.zero(L.Q_PART)
    density(s.grid, s.electrons, -1.0)
    return s.solver.run(eb)


def nsteps(s: Streamer, n: int, ntarget: int, nmax: int, eb: float, dt: float, dt_poisson: float,
           dt_output: float, dt_resample: float, outpath: Optional[str] = None, check_weights: bool = True,
           on_step: Optional[Callable[[int, dict], None]] = None,
           mark: Optional[Callable[[str], None]] = None) -> List[dict]:
    """Advance the simulation by n steps; returns the per-step diagnostics.  `mark(name)`, if
    given, is called as each part of a step begins ("poisson", "output", "advance",
    "diagnostics", "resample", "fluid", "repack") and with "end" after the last, e.g. to
    record a CUDA event on the context's stream."""
    poisson = TimeStepper(dt_poisson)
    output = TimeStepper(dt_output)
    resampler = TimeStepper(dt_resample, start=dt)
    reserve_resample(s.electrons)
    out: List[dict] = []
    tick = mark if mark is not None else (lambda name: None)
    for i in range(1, n + 1):
        t = (i - 1) * dt
        tick("poisson")
        if poisson.atstep(t) is not None:
            poisson_step(s, eb)
        tick("output")
        j = output.atstep(t)
        if j is not None and outpath:
            os.makedirs(outpath, exist_ok=True)
            fieldsio.savefields(os.path.join(outpath, f"{j:04d}.h5"), s.grid, s.solver, s.fluid)
        tick("advance")
        if s.photons is not None:
            jumc.advance_mixed(s.electrons, s.photons, s.efield, dt, s.tracker)
        else:
            jumc.advance(s.electrons, s.efield, dt, s.tracker)
        tick("diagnostics")
        d = diagnostics(s.electrons, s.photons)
        d.update(step=i, t=t)
        tick("resample")
        if resampler.atstep(t) is not None:
            if s.photons is not None:
                s.photons.repack()
            pre = s.electrons.weight() if check_weights else 0.0
            jumc.repack(s.electrons)
            if check_weights:
                post = s.electrons.weight()
                if not math.isclose(pre, post, rel_tol=1e-5):
                    raise AssertionError("repackaging is not conserving the number of particles")
            resample(s.electrons, s.grid, ntarget, nmax)
            if check_weights:
                post2 = s.electrons.weight()
                if not math.isclose(post, post2, rel_tol=1e-5):
                    raise AssertionError("resampling is not conserving the number of particles")
            d["resampled"] = True
        tick("fluid")
        if s.fluid is not None and s.hasfluid:
            s.fluid.step(dt)
        tick("repack")
        jumc.repack(s.electrons)
        tick("end")
        out.append(d)
        s.log.append(d)
        if on_step is not None:
            on_step(i, d)
    return out
