"""initfromfiles!'s CPU restatement (orc_init_from_density) pinned without a GPU against what
the reference's code defines (MCStreamer/src/initdens.jl:64-159): the noiseless sampler's
three regimes, the Poisson sampler's expected counts and charge, the fluid cells, electrons
placed in their own cell at rest, in the serial cell order, with s ~ Exp(1).  No reference
test exists for initfromfiles!."""
import math

import numpy as np
import pytest
import scipy.stats as ss

from oracle import initdens_ref as I

E = 1.6021766208e-19
R, LEN = 1e-3, 2e-3


def _vol(M, N):
    dr, dz = R / M, LEN / N
    rc = (np.arange(M) + 0.5) * dr
    return (2.0 * np.pi * rc * dr * dz)[:, None] * np.ones((1, N))


def _cells(x, M, N):
    r = np.hypot(x[:, 0], x[:, 1])
    return np.floor(r / (R / M)).astype(int), np.floor(x[:, 2] / (LEN / N)).astype(int)


def test_noiseless_regimes_and_charge():
    M, N, p = 12, 10, 10
    V = _vol(M, N)
    n = np.empty((M, N))
    n[:4] = 0.4            # Poisson(n)
    n[4:8] = 3.6           # randround(n)
    n[8:] = 57.0           # p electrons of weight n / p
    ne = n / V
    q = 0.3 * E * ne
    x, w, s, qfd, nf = I.initfromfiles(ne, q, R, LEN, M, N, I.NOISELESS, p, seed=4)
    i, j = _cells(x, M, N)
    cnt = np.zeros((M, N), int)
    np.add.at(cnt, (i, j), 1)
    assert set(np.unique(cnt[4:8])) <= {3, 4}
    assert (cnt[8:] == p).all()
    assert cnt[:4].max() <= 6
    np.testing.assert_allclose(w[i >= 8], 57.0 / p, rtol=1e-15)
    assert (w[i < 8] == 1.0).all()
    # qf = q / e + w nume / V
    wc = np.where(np.arange(M)[:, None] >= 8, 57.0 / p, 1.0)
    np.testing.assert_allclose(qfd[1:M + 1, 1:N + 1], q / E + wc * cnt / V, rtol=1e-14)
    assert (nf == 0).all()
    # electrons at rest in their own cell, in serial cell order (r fastest)
    order = i + M * j
    assert (np.diff(order) >= 0).all()
    assert ss.kstest(s, "expon").pvalue > 1e-4


def test_noiseless_means():
    M, N, p = 40, 50, 10
    V = _vol(M, N)
    for nval, tol in ((0.4, 0.05), (3.6, 0.02)):
        ne = np.full((M, N), nval) / V
        x, w, s, qfd, nf = I.initfromfiles(ne, 0 * ne, R, LEN, M, N, I.NOISELESS, p, seed=7)
        assert abs(len(w) / (M * N) - nval) < 5 * np.sqrt(nval / (M * N)) + 1e-9, (len(w), nval)


def test_poisson_sampler_expectations():
    """PoissonInitSampling: E[nume] w = ne V; E[qf] V = |ni| V sign(ni) with ni = ne + q/e."""
    M, N, p = 30, 40, 10
    V = _vol(M, N)
    ne = np.full((M, N), 23.0) / V          # w = 2.3, nume ~ Poisson(10)
    q = -1.7 * E * ne                        # ni = -0.7 ne
    x, w, s, qfd, nf = I.initfromfiles(ne, q, R, LEN, M, N, I.POISSON, p, seed=2)
    np.testing.assert_allclose(w, 2.3, rtol=1e-14)
    tot = len(w) * 2.3
    assert abs(tot - 23.0 * M * N) < 5 * 2.3 * np.sqrt(10 * M * N)
    charge = (qfd[1:M + 1, 1:N + 1] * V).sum()
    assert charge < 0
    assert abs(charge + 0.7 * 23.0 * M * N) < 5 * np.sqrt(0.7 * 23.0 * 1.61 * M * N)
    # the ions' weight wi = max(1, |ni| V / p): qf is a multiple of wi / V
    k = -qfd[1:M + 1, 1:N + 1] * V / 1.61
    np.testing.assert_allclose(k, np.round(k), atol=1e-9)


def test_fluid_cells_and_capacity():
    M, N, p = 8, 6, 5
    V = _vol(M, N)
    ne = np.full((M, N), 2.0) / V
    ne[2:4, 1:3] = 1e21
    q = np.full((M, N), 1e-3)
    x, w, s, qfd, nf = I.initfromfiles(ne, q, R, LEN, M, N, I.NOISELESS, p, fluid_threshold=1e20, seed=1)
    np.testing.assert_array_equal(nf[4:6, 3:5], 1e21)
    assert (nf > 0).sum() == 4
    np.testing.assert_array_equal(qfd[3:5, 2:4], 1e-3 / E + 1e21)
    i, j = _cells(x, M, N)
    assert not ((i >= 2) & (i < 4) & (j >= 1) & (j < 3)).any()
    n, *_ = I.initfromfiles(ne, q, R, LEN, M, N, I.NOISELESS, p, fluid_threshold=1e20, seed=1, cap=len(w) - 1)
    assert n == -1


def test_empty_and_single_particle_cells():
    """ne = 0 samples nothing (qfixed = q/e); p = 1 keeps one electron per dense cell."""
    M, N = 5, 4
    V = _vol(M, N)
    x, w, s, qfd, nf = I.initfromfiles(np.zeros((M, N)), np.full((M, N), 2 * E), R, LEN, M, N, I.NOISELESS, 10)
    assert len(w) == 0
    np.testing.assert_allclose(qfd[1:M + 1, 1:N + 1], 2.0, rtol=1e-15)
    x, w, s, qfd, nf = I.initfromfiles(np.zeros((M, N)), np.zeros((M, N)), R, LEN, M, N, I.POISSON, 10)
    assert len(w) == 0 and (qfd == 0).all()
    ne = 50.0 / V
    x, w, s, qfd, nf = I.initfromfiles(ne, 0 * ne, R, LEN, M, N, I.NOISELESS, 1)
    assert len(w) == M * N
    np.testing.assert_allclose(w, 50.0, rtol=1e-14)


def _py_initfromfiles(ne, q, M, N, method, p, thr, seed):
    """initfromfiles! restated in plain Python from the reference's statements (the draws
    taken word by word from the same Philox streams, the Poisson sampler written out
    again), for a small grid."""
    from oracle import pyoracle as po
    dr, dz = R / M, LEN / N

    class Stream:
        def __init__(self, c0, c1, tag):
            self.c0, self.c1, self.tag, self.k = c0, c1, tag, 0

        def next(self):
            u = po.uniform(seed, self.c0, self.c1, self.tag, self.k)
            self.k += 1
            return u

    def poisson(rng, lam):
        if lam <= 0:
            return 0
        if lam < 10.0:
            u = rng.next()
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
            U = rng.next() - 0.5
            V = rng.next()
            us = 0.5 - abs(U)
            kf = math.floor((2.0 * a / us + b) * U + lam + 0.43)
            if us >= 0.07 and V <= vr:
                return kf
            if kf < 0 or (us < 0.013 and V > us):
                continue
            if math.log(V) + math.log(invalpha) - math.log(a / (us * us) + b) <= -lam + kf * loglam - math.lgamma(kf + 1.0):
                return kf
        return math.floor(lam)

    xs, ws, ss = [], [], []
    qfd = np.zeros((M + 2, N + 2))
    nf = np.zeros((M + 4, N + 4))
    for j in range(1, N + 1):
        for i in range(1, M + 1):
            c = (i - 1) + (j - 1) * M
            V = 2.0 * math.pi * (((i - 1) + 0.5) * dr) * dr * dz
            nec, qc = ne[i - 1, j - 1], q[i - 1, j - 1]
            if nec > thr:
                nf[i + 1, j + 1] = nec
                qfd[i, j] = qc / E + nec
                continue
            rng = Stream(c, 0, 6)
            if method == I.NOISELESS:
                n = nec * V
                if n < 1:
                    nume, w = poisson(rng, n), 1.0
                elif n < p:
                    m = math.floor(n)
                    nume, w = (int(m) if rng.next() > n - m else int(m) + 1), 1.0
                else:
                    nume, w = p, n / p
                qf = qc / E + w * nume / V
            else:
                w = max(1.0, nec * V / p)
                nume = poisson(rng, nec * V / w)
                ni = nec + qc / E
                wi = max(1.0, abs(ni) * V / p)
                numi = poisson(rng, abs(ni) * V / wi)
                qf = math.copysign(1.0, ni) * numi * wi / V if ni != 0 else 0.0 * numi * wi / V
            qfd[i, j] = qf
            for k in range(nume):
                u = [po.uniform(seed, c, k, 6 | 0x40000000, t) for t in range(4)]
                r = dr * u[0] + (i - 1) * dr
                z = dz * u[1] + (j - 1) * dz
                phi = 2.0 * math.pi * u[2]
                xs.append((r * math.cos(phi), r * math.sin(phi), z))
                ws.append(w)
                ss.append(-math.log(u[3]))
    return np.array(xs).reshape(-1, 3), np.array(ws), np.array(ss), qfd, nf


@pytest.mark.parametrize("method", [I.NOISELESS, I.POISSON])
def test_oracle_agrees_with_a_python_restatement(method):
    """The C++ loop and a plain-Python restatement written apart agree bit for bit: counts,
    weights, positions, s, qfixed and the fluid cells, over all sampler branches."""
    M, N, p = 6, 8, 10
    V = _vol(M, N)
    rng = np.random.default_rng(4)
    n = 10 ** rng.uniform(-2, 2.5, (M, N))            # Poisson(n < 1), randround, p electrons
    n[0, 0] = 0.0
    ne = np.asfortranarray(n / V)
    ne[5, 7] = 3e21                                    # one fluid cell
    q = np.asfortranarray(E * ne * rng.uniform(-1.5, 1.5, (M, N)))
    x, w, s, qfd, nf = I.initfromfiles(ne, q, R, LEN, M, N, method, p, fluid_threshold=1e21, seed=9)
    x2, w2, s2, qfd2, nf2 = _py_initfromfiles(ne, q, M, N, method, p, 1e21, 9)
    assert len(w) == len(w2) > 50
    np.testing.assert_array_equal(w, w2)
    np.testing.assert_array_equal(x, x2)
    np.testing.assert_array_equal(s, s2)
    np.testing.assert_array_equal(qfd, qfd2)
    np.testing.assert_array_equal(nf, nf2)
