"""Failure detection without a GPU fault: a bounded wait whose predecessor never publishes
gives up, raises the status, and the next call reports MCS_ERR_TIMEOUT; the context then
runs normal work."""
import numpy as np
import pytest

from mcstreamer_b200 import _lib as L
from mcstreamer_b200 import constants as co
from mcstreamer_b200 import jumc, lxcat, swarm


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_survives(ctx):
    assert ctx.lib.mcs_diag_wait_timeout(ctx.h, 4096) == L.ERR_TIMEOUT
    assert ctx.lib.mcs_diag_wait_timeout(ctx.h, 1) == L.ERR_TIMEOUT
    # the status word was cleared and the context keeps working
    ctx.sync()
    tab = jumc.CollisionTable(lxcat.synthetic_table(0), ctx)
    n = 4096
    pop = jumc.Population(4 * n, swarm.initial_particles(n, "maxwellian", 1, mean_ev=2.0), tab, precision="fp32",
                          seed=1)
    fld = jumc.FixedField(100 * co.Td * 2.5e25, ctx)
    mom = np.zeros((5, L.STEP_MOMENTS))
    ctx.check(ctx.lib.mcs_swarm_run(pop.h, tab.h, fld.h, 1e-13, 5, n, 0.1, 1, L.dptr(mom)))
    assert (mom[:, L.S_COUNT] > 0).all()
    fld.close(); pop.close(); tab.close()


@pytest.mark.gpu
def test_diag_rejects_bad_limits(ctx):
    assert ctx.lib.mcs_diag_wait_timeout(ctx.h, 0) == L.ERR_ARG
    assert ctx.lib.mcs_diag_wait_timeout(ctx.h, (1 << 20) + 1) == L.ERR_ARG
