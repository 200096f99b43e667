"""Pure-Python (loop) restatement of load_lxcat (JuMC/src/lxcat.jl:17-134) for small
grids -- TEST INFRASTRUCTURE, the checker of mcstreamer_b200.lxcat."""
from __future__ import annotations

import math

ELECTRON_MASS = 9.10938356e-31
EV = 1.6021766208e-19


def linrange(a, b, n):
    # Base.LinRange getindex: (1 - j/lendiv)*a + (j/lendiv)*b
    return [(1.0 - j / (n - 1)) * a + (j / (n - 1)) * b for j in range(n)]


def interp_flat(xs, ys, x):
    # extrapolate(interpolate((xs,), ys, Gridded(Linear())), Flat())
    if x <= xs[0]:
        return ys[0]
    if x >= xs[-1]:
        return ys[-1]
    for i in range(len(xs) - 1):
        if xs[i] <= x < xs[i + 1]:
            t = (x - xs[i]) / (xs[i + 1] - xs[i])
            return (1.0 - t) * ys[i] + t * ys[i + 1]
    return ys[-1]


def load_lxcat(db, densities, e0, emax, n):
    energy = linrange(e0, emax, n)
    v = [math.sqrt(2 * e / ELECTRON_MASS) for e in energy]
    targets = {}
    for item in db:
        dens = densities.get(item["target"], 0.0)
        if dens == 0.0:
            continue
        item = dict(item)
        e_0 = [d[0] * EV for d in item["data"]]
        cs = [d[1] for d in item["data"]]
        if "3-body" in item.get("comment", ""):
            cs = [c * dens / 1e6 for c in cs]
        if "rescale" in item:
            cs = [c * item["rescale"] for c in cs]
        item["nu"] = [dens * v[k] * interp_flat(e_0, cs, energy[k]) for k in range(n)]
        targets.setdefault(item["target"], []).append(item)
    rows, procs = [], []
    for name, ps in targets.items():
        for p in ps:
            if p["kind"] == "EFFECTIVE":
                for p2 in ps:
                    if p2 is not p and p2["kind"] in ("EXCITATION", "IONIZATION"):
                        p["nu"] = [a - b for a, b in zip(p["nu"], p2["nu"])]
                p["kind"] = "ELASTIC"
        for p in ps:
            procs.append(p["kind"])
            rows.append(p["nu"])
    total = [sum(r[k] for r in rows) for k in range(n)]
    maxrate = max(total)
    rows.append([maxrate - t for t in total])
    procs.append("NULL")
    integ = [sum(r) for r in rows]
    perm = sorted(range(len(rows)), key=lambda i: -integ[i])
    return [procs[i] for i in perm], [rows[i] for i in perm], maxrate
