"""The persistent CG half diffusion step vs the oracle's Jacobi-PCG on the
shell geometry (CG residual checks)."""
import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, workloads as W
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shell():
    wl = W.shell_c2(h=0.1)
    m = wl.mesh
    rng = np.random.default_rng(5)
    # a sharp front plus noise: the residual a propagating wave produces
    V = -85.0 + 120.0 * (m.xyz[:, 2] < -3.0) + rng.normal(0, 1.0, m.n)
    c = O.Csr(m.xyz, m.tets, m.fibers, wl.D, 1.0, wl.dt)
    return wl, V, c


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_half_step_matches_oracle(gpu, shell, prec):
    wl, V, c = shell
    B = c.scipy("B")
    x_ref, it_ref, rr_ref = c.pcg(B @ V, V.copy(), tol=1e-7, maxit=1000, jacobi_steps=1)
    g = Monodomain(wl.mesh, capi.TUSSCHER, prec, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
    g.set_voltage(V)
    it, rr = g.diffusion_half_step()
    x = g.voltage()
    g.close()
    assert it_ref > 3
    if prec == capi.FP64:
        assert abs(it - it_ref) <= 1, (it, it_ref)
        assert rr <= 1e-7
        assert np.max(np.abs(x - x_ref)) < 1e-6 * np.max(np.abs(x_ref))
    else:
        assert it <= it_ref + 2, (it, it_ref)
        assert np.max(np.abs(x - x_ref)) < 1e-4 * np.max(np.abs(x_ref))
