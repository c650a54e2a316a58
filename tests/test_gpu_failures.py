"""Failure detection on the GPU, made to happen without faulting it.

The reference has no counterpart: its ten Tusscher Newton loop has no
iteration cap (Tusscher.cc:150) and a failed solve only prints
(Tusscher.cc:182-184).  Here every in-kernel wait is bounded and the host
reads status words:

* a grid barrier that waits for one CTA more than the launch has (the
  ep_test_hold_barrier hook: the missing arrival never comes) gives up after
  a short poll limit; ep_step returns EP_ERR_TIMEOUT promptly, and after the
  hook is cleared and the state restored the handle steps on exactly like one
  that never failed;
* a non-finite voltage uploaded from the host shows up as EP_ERR_NAN with
  the step's statistics counting the nodes, and the CG solves stop at once
  instead of running to their iteration limit;
* a Newton cap of 1 is counted in newton_cap_hits.
"""
import time

import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu
D = M.sigma_to_D(1.2, 0.2)
AMP = 50.0 * 2000.0


def _handle(prec=capi.FP32, **kw):
    m = M.slab(15, 13, 4, 0.28, 0.24, 0.06)
    g = Monodomain(m, capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, D=D, tt_jacobian=capi.TT_JAC_TRUE, **kw)
    g.set_voltage(-85.423)
    g.set_stimulus(M.corner_block(m, 3, 3), 0.0, 1.0, AMP)
    return g


def test_grid_barrier_timeout(gpu):
    ref = _handle()
    g = _handle()
    ref.step(20)
    g.step(20)
    V0, S0 = g.voltage(), g.states()
    g.set_wait_limits(grid_polls=4096)
    g.test_hold_barrier(1)
    t0 = time.perf_counter()
    with pytest.raises(capi.EPError) as e:
        g.step(1)
    waited = time.perf_counter() - t0
    assert e.value.code == -8                              # EP_ERR_TIMEOUT
    assert g.last_stats["timeouts"] > 0
    assert waited < 5.0, waited                            # a short limit gives up promptly
    assert g.time()[1] == 20                               # the failed call took no step
    # clear the hook, put the state back: the handle steps on as if nothing
    # happened.  A voltage upload restarts the CG start predictor, so the
    # handle that never failed takes the same upload of its own voltage.
    g.test_hold_barrier(0)
    g.set_wait_limits(0, 0)
    g.set_voltage(V0)
    g.set_states(S0)
    ref.set_voltage(ref.voltage())
    st = g.step(30)
    ref.step(30)
    assert st["timeouts"] == 0 and st["cg_failures"] == 0
    assert np.array_equal(g.voltage(), ref.voltage())
    g.close()
    ref.close()


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_nonfinite_voltage_is_reported(gpu, prec):
    g = _handle(prec)
    g.step(5)
    V, S = g.voltage(), g.states()
    V0 = V.copy()
    V[17] = np.nan
    g.set_voltage(V)
    t0 = time.perf_counter()
    with pytest.raises(capi.EPError) as e:
        g.step(1)
    assert e.value.code == -7                              # EP_ERR_NAN
    st = g.last_stats
    assert st["nonfinite"] > 0 and st["timeouts"] == 0
    assert st["cg_failures"] >= 1 and st["cg_max_iters"] <= 2   # stopped at once, not at maxit
    assert time.perf_counter() - t0 < 5.0
    # the NaN spread through the diffusion and the cells; a clean state steps normally again
    g.set_voltage(V0)
    g.set_states(S)
    assert g.step(2)["nonfinite"] == 0
    g.close()


def test_newton_cap_is_counted(gpu):
    """FP64 ten Tusscher with the cap at one Newton iteration: the
    stimulated upstroke needs more, and the cap hits are counted."""
    capped = _handle(capi.FP64, newton_cap=1)
    st = capped.step(60)
    assert st["newton_cap_hits"] > 0
    assert st["newton_iters"] >= st["newton_cap_hits"]
    free = _handle(capi.FP64)
    assert free.step(60)["newton_cap_hits"] == 0
    capped.close()
    free.close()
