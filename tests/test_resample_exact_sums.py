"""The arithmetic that lets resample!'s merging cells run without the serial pass
(csrc/sort_resample.cu, merge_select_warp), checked on the CPU.

A merging cell (MCStreamer/src/resample.jl:31-76) sums its weights in FP64 in slot order
and picks, for clone k, the first particle whose running sum exceeds wtotal * x_k.  When
every weight is a non-negative multiple of 2^lmin below 2^(emax+1) and
p * 2^(emax+1) <= 2^(lmin+53), every partial sum is an integer multiple of 2^lmin below
2^53 of them: FP64 adds it exactly, in any order.  Then the running sums of a parallel
scan are the serial ones, and the clone sources are a search over them.  These tests
restate the serial loop and the condition in Python and compare the two selections on
random cells, with weights as the streamer run makes them (FP32 values, integers, dyadic
fractions) and with full FP64 mantissas (which must fail the condition)."""
import math

import numpy as np
import pytest


def serial_select(w, f, nt):
    """resample.jl's merge loop: wtotal, then the clone sources in slot order."""
    wtotal = 0.0
    for wj in w:
        wtotal = wtotal + wj
    x, pk, wcum, src = f[0], 0, 0.0, []
    for j, wj in enumerate(w):
        while wtotal * x < wcum + wj and pk < nt:
            pk += 1
            src.append(j)
            if pk < nt:
                x = x + f[pk] * (1.0 - x)
        wcum = wcum + wj
    return wtotal, src


def exact_condition(w):
    """p * 2^(emax+1) <= 2^(lmin+53) over the non-zero weights (all finite, >= 0)."""
    emax, lmin = None, None
    for v in w:
        if v == 0.0:
            continue
        m, e = math.frexp(v)                    # v = m * 2^e, 0.5 <= m < 1
        mi = int(m * 2 ** 53)                   # the 53-bit significand as an integer
        lsb = (e - 53) + ((mi & -mi).bit_length() - 1)
        emax = e - 1 if emax is None else max(emax, e - 1)
        lmin = lsb if lmin is None else min(lmin, lsb)
    if emax is None:
        return True
    lg = (len(w) - 1).bit_length()              # ceil(log2 p)
    return lg + emax + 1 <= lmin + 53


def scan_select(w, f, nt, rng):
    """The warp's form: a total summed in another order, running sums, a search per clone."""
    order = rng.permutation(len(w))
    wtotal = 0.0
    for j in order:                             # any order: exact under the condition
        wtotal += w[j]
    A = np.cumsum(w)
    t, x = [], f[0]
    for k in range(nt):
        if k > 0:
            x = x + f[k] * (1.0 - x)
        t.append(wtotal * x)
    jk = np.searchsorted(A, np.array(t), side="right")   # first j with t_k < A_j
    return wtotal, [int(j) for j in jk if j < len(w)]


def factors(rng, nt):
    u = rng.random(nt)
    return 1.0 - (1.0 - u) ** (1.0 / (nt - np.arange(nt)))


@pytest.mark.parametrize("kind", ["fp32", "integer", "dyadic"])
def test_exact_weights_give_the_serial_selection(kind):
    rng = np.random.default_rng({"fp32": 1, "integer": 2, "dyadic": 3}[kind])
    nt = 64
    for _ in range(400):
        p = int(rng.integers(97, 1200))
        u = 10 ** rng.uniform(0, 4, p)
        if kind == "fp32":
            w = u.astype(np.float32).astype(np.float64)
        elif kind == "integer":
            w = np.rint(u)
        else:
            w = np.rint(u * 2 ** 20) / 2 ** 20
        assert exact_condition(w)
        f = factors(rng, nt)
        assert scan_select(w, f, nt, rng) == serial_select(w, f, nt)


def test_full_mantissas_fail_the_condition():
    rng = np.random.default_rng(4)
    for _ in range(50):
        w = 10 ** rng.uniform(0, 4, int(rng.integers(97, 400)))
        assert not exact_condition(w)


def test_condition_bounds_the_worst_case():
    # p = 2: the bound p * 2^(emax+1) = 4 allows 2^(lmin+53) >= 4, i.e. lmin >= -51; at
    # lmin = -52 it fails although 1 + 2^-52 itself is a double (the bound is the worst
    # case of p weights just below 2^(emax+1)); zero weights do not count
    assert exact_condition(np.array([1.0, 2.0 ** -51]))
    assert not exact_condition(np.array([1.0, 2.0 ** -52]))
    assert exact_condition(np.array([0.0, 0.0, 3.0]))
