"""The device activation tracker against the same definitions applied on the
host to the voltage read back after every step (FP64 slab, dt 0.02 ms, one
beat from a corner stimulus).

Activation: first upward crossing of -40 mV.  APD90: first downward crossing
of v_peak - 0.9 (v_peak - v_rest) later than 5 ms after activation, v_rest =
the node's voltage when tracking starts (not the minimum before activation,
which takes in the undershoot the consistent-mass Crank-Nicolson step makes
ahead of a steep front).  The tracker sees the voltage inside the step (after
the first diffusion half step), the host only at step ends, so the times agree
to a step or two, not bit for bit.
"""
import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


def _host_times(t, V, v_rest, thr=-40.0):
    up = np.where((V[:-1] < thr) & (V[1:] >= thr))[0]
    if not len(up):
        return -1.0, -1.0
    k = up[0]
    ta = t[k] + (thr - V[k]) / (V[k + 1] - V[k]) * (t[k + 1] - t[k])
    vp = V[k + 1:].max()
    v90 = vp - 0.9 * (vp - v_rest)
    dn = np.where((t[:-1] > ta + 5.0) & (V[:-1] >= v90) & (V[1:] < v90))[0]
    if not len(dn):
        return ta, -1.0
    j = dn[0]
    tr = t[j] + (V[j] - v90) / (V[j] - V[j + 1]) * (t[j + 1] - t[j])
    return ta, tr - ta


def test_activation_and_apd90_match_the_voltage_trace(gpu):
    m = M.slab(9, 9, 3, 0.16, 0.16, 0.04)
    dt = 0.02
    g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=dt, ionic_dt=dt, D=M.sigma_to_D(1.2, 0.2),
                   tt_jacobian=capi.TT_JAC_TRUE)
    v0 = -85.423
    g.set_voltage(v0)
    g.set_stimulus(M.corner_block(m, 2, 2), 0.0, 1.0, 50.0 * 2000.0)
    watch = np.array([0, m.n // 2, m.n - 1])
    nsteps = 20000                                   # 400 ms: one whole beat
    t = np.arange(nsteps + 1) * dt
    V = np.empty((nsteps + 1, len(watch)))
    V[0] = g.voltage()[watch]
    for k in range(nsteps):
        g.step(1)
        V[k + 1] = g.voltage()[watch]
    ta, apd = g.activation()
    g.close()
    for j, i in enumerate(watch):
        hta, hapd = _host_times(t, V[:, j], v0)
        assert hta > 0.0 and hapd > 200.0, (i, hta, hapd)
        assert abs(ta[i] - hta) <= 2 * dt, (i, ta[i], hta)
        assert abs(apd[i] - hapd) <= 0.1, (i, apd[i], hapd)
