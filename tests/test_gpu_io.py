"""Host <-> device transfers of the per-node arrays through the C ABI on a
mesh large enough (>= 64K nodes) for the chunked, overlapped copies (the
host-side conversion of one chunk beside the copy of the next): what goes in
comes back, rounded to the handle's precision, node for node."""
import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_voltage_and_states_round_trip_in_chunks(gpu, prec):
    m = M.slab(61, 61, 21, 1.2, 1.2, 0.4)                 # 78,141 nodes
    assert m.n >= 1 << 16
    g = Monodomain(m, capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                   tt_jacobian=capi.TT_JAC_TRUE)
    rng = np.random.default_rng(3)
    cast = np.float64 if prec == capi.FP64 else np.float32
    V = rng.normal(-80.0, 10.0, m.n)
    g.set_voltage(V)
    assert np.array_equal(g.voltage(), V.astype(cast).astype(np.float64))
    S = g.states()
    S2 = S * (1.0 + 1e-3 * rng.standard_normal(S.shape))
    S2[:, 0] = V
    g.set_states(S2)
    back = g.states()
    assert back.shape == S2.shape
    assert np.array_equal(back[:, 1:], S2[:, 1:].astype(cast).astype(np.float64))
    assert np.array_equal(back[:, 0], V.astype(cast).astype(np.float64))
    g.close()
