"""nsteps' schedule and call order (MCStreamer/src/main.jl:218-318, timesteps.jl) without a
GPU: every device call of the loop is replaced by a recorder."""
import pytest

from mcstreamer_b200 import loop


def test_timestepper_is_the_reference_one():
    ts = loop.TimeStepper(1.5, start=10.0)       # start is never read (timesteps.jl:23-28)
    fired = [ts.atstep(t) for t in (0.0, 0.5, 1.5, 2.0, 3.0, 4.4, 4.5)]
    assert fired == [0, None, 1, None, 2, None, 3]


class _Rec:
    def __init__(self):
        self.calls = []

    def __call__(self, name):
        def f(*a, **k):
            self.calls.append(name)
            return (1, 1) if name == "solve" else None
        return f


class _Pop:
    def __init__(self, rec):
        self.rec = rec

    def weight(self):
        return 1.0


class _Obj:
    def __init__(self, rec, name):
        self.rec, self.name = rec, name

    def __getattr__(self, item):
        return self.rec(f"{self.name}.{item}")


def test_nsteps_call_order(monkeypatch, tmp_path):
    rec = _Rec()
    monkeypatch.setattr(loop, "density", rec("density"))
    monkeypatch.setattr(loop, "diagnostics", lambda e, p: {})
    monkeypatch.setattr(loop, "resample", rec("resample"))
    monkeypatch.setattr(loop, "reserve_resample", lambda p: None)   # scratch allocation only
    monkeypatch.setattr(loop.jumc, "advance_mixed", rec("advance"))
    monkeypatch.setattr(loop.jumc, "repack", rec("repack"))
    monkeypatch.setattr(loop.fieldsio, "savefields", rec("save"))
    s = loop.Streamer(grid=_Obj(rec, "grid"), solver=_Obj(rec, "solver"), electrons=_Pop(rec), efield=None,
                      photons=_Obj(rec, "photons"), fluid=_Obj(rec, "fluid"), tracker=object())
    # dt 0.5; Poisson every 1.0, output every 2.0, resample every 1.5: steps at t = 0, 0.5, ... 2.0
    out = loop.nsteps(s, 5, 10, 15, -1.5e6, 0.5, 1.0, 2.0, 1.5, outpath=str(tmp_path))
    poisson = ["grid.zero", "density", "solver.run"]
    res = ["photons.repack", "repack", "resample"]
    tail = ["fluid.step", "repack"]
    want = (poisson + ["save", "advance"] + res + tail                       # t = 0
            + ["advance"] + tail                                             # t = 0.5
            + poisson + ["advance"] + tail                                   # t = 1.0
            + ["advance"] + res + tail                                       # t = 1.5
            + poisson + ["save", "advance"] + tail)                          # t = 2.0
    assert rec.calls == want
    assert [d["step"] for d in out] == [1, 2, 3, 4, 5]
    assert [bool(d.get("resampled")) for d in out] == [True, False, False, True, False]


def test_nsteps_without_photons_or_fluid(monkeypatch):
    """Electrons only: advance! instead of the mixed advance, no photon repack!, no fluid;
    a weight change across resample! fails as the reference's assertion does."""
    rec = _Rec()
    monkeypatch.setattr(loop, "density", rec("density"))
    monkeypatch.setattr(loop, "diagnostics", lambda e, p: {})
    monkeypatch.setattr(loop, "resample", rec("resample"))
    monkeypatch.setattr(loop, "reserve_resample", lambda p: None)   # scratch allocation only
    monkeypatch.setattr(loop.jumc, "advance", rec("advance"))
    monkeypatch.setattr(loop.jumc, "advance_mixed", rec("mixed"))
    monkeypatch.setattr(loop.jumc, "repack", rec("repack"))
    s = loop.Streamer(grid=_Obj(rec, "grid"), solver=_Obj(rec, "solver"), electrons=_Pop(rec), efield=None,
                      tracker=object())
    loop.nsteps(s, 2, 10, 15, -1.5e6, 1.0, 1.0, 10.0, 1.0)
    assert rec.calls == ["grid.zero", "density", "solver.run", "advance", "repack", "resample", "repack"] * 2

    class Shrinking(_Pop):
        def __init__(self, rec):
            super().__init__(rec)
            self.w = [1.0, 0.5]

        def weight(self):
            return self.w.pop(0) if len(self.w) > 1 else self.w[0]

    s.electrons = Shrinking(rec)
    with pytest.raises(AssertionError, match="repackaging"):
        loop.nsteps(s, 1, 10, 15, -1.5e6, 1.0, 1.0, 10.0, 1.0)
