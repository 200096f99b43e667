"""mcs_moments_noalloc, the moments entry point that allocates nothing.

It exists for callers that may not allocate device memory when they want diagnostics (a
loop held to a memory budget fixed at start-up, an application whose allocator owns every
device byte): they pass their own device arrays and output.  The test calls it twice in a
row through the C ABI on device buffers it owns and compares each result with the sums the
population API (mcs_moments) computes for the same particles, at the 1e-12 relative
tolerance of the other moment tests.  This file is collected last so that a stop at the
first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from mcstreamer_b200 import _lib as L

MAX_PARTICLES = 67108864


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [100_003, 3 * 8192, 0])
def test_noalloc_moments_match_population_moments_on_two_calls(precision, n):
    """An uneven size, a size that ends exactly on a chunk boundary (8192 particles per
    chunk) and the empty population (counts and sums 0, the maximum energy -inf)."""
    import torch

    from mcstreamer_b200 import jumc, lxcat
    from tests.helpers import broad

    ctx = jumc.Context(0)
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    m = max(n, 1)
    p = broad(m, 13, spread=1e-4)
    p.w[:] = np.random.default_rng(5).uniform(0.5, 2.0, m)
    p.active[::5] = 0
    pop = jumc.Population(m, p if n else None, tab, precision=precision, seed=1)
    ref = pop.moments()  # the existing entry point, MCS_MOMENTS_BASE sums
    if n == 0:
        assert ref[L.M_COUNT] == 0 and ref[L.M_EMAX] == -np.inf

    dev = torch.device("cuda:0")
    dtype = torch.float32 if precision == "fp32" else torch.float64
    cols = [p.x[:, 0], p.x[:, 1], p.x[:, 2], p.v[:, 0], p.v[:, 1], p.v[:, 2], p.w]
    bufs = [torch.tensor(np.ascontiguousarray(c), dtype=torch.float64).to(dtype).to(dev) for c in cols]
    act = torch.tensor(p.active, dtype=torch.uint8, device=dev)
    out = torch.empty(L.MOMENTS_BASE, dtype=torch.float64, device=dev)
    ptrs = (C.c_void_p * 7)(*[b.data_ptr() for b in bufs])
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    prec = L.FP32 if precision == "fp32" else L.FP64
    lib = L.lib()
    for _ in range(2):
        out.fill_(np.nan)
        rc = lib.mcs_moments_noalloc(0, stream, prec, ptrs, C.cast(act.data_ptr(), L.pu8), n,
                                     C.cast(out.data_ptr(), L.pd))
        assert rc == L.OK
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=0)

    # sizes beyond the fixed scratch are refused before anything runs
    rc = lib.mcs_moments_noalloc(0, stream, prec, ptrs, C.cast(act.data_ptr(), L.pu8), MAX_PARTICLES + 1,
                                 C.cast(out.data_ptr(), L.pd))
    assert rc == L.ERR_ARG
    pop.close()
    tab.close()
    ctx.close()
