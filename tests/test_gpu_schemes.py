"""The backward-Euler and explicit operator splittings (EP_BackwardEuler,
EP_ExplicitSolver) with the reference's per-node ionic strides
(CardiacBody::getVoltageFromIonicCurrent), GPU FP64 against the CPU oracle's
restatement -- with the reference's own cell objects where they apply."""
import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu
D = M.sigma_to_D(1.2, 0.2)
AMP = 100000.0


def _oracle(m, scheme, cells, dt, idt, steps, blk, nstim):
    c = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, dt)
    s = O.Sim(c, cells, dt, idt, cg_tol=1e-12, cg_maxit=2000, jacobi_steps=1)
    s.set_scheme(scheme)
    s.V[:] = -85.423
    out = []
    for k in range(steps):
        s.istim[:] = 0.0
        if k < nstim:
            s.istim[blk] = AMP
        s.step()
        if (k + 1) % 50 == 0:
            out.append(s.V.copy())
    return out


def _gpu(m, scheme, prec, dt, idt, steps, blk, t_stim, tt_jac):
    g = Monodomain(m, capi.TUSSCHER, prec, dt=dt, ionic_dt=idt, D=D, cg_tol=1e-12 if scheme == capi.SCHEME_BE else 0.0,
                   cg_maxit=2000, tt_jacobian=tt_jac, scheme=scheme)
    g.set_voltage(-85.423)
    g.set_stimulus(blk, 0.0, t_stim, AMP)
    out = []
    for k in range(0, steps, 50):
        g.step(50)
        out.append(g.voltage())
    g.close()
    return out


@pytest.mark.parametrize("scheme", [capi.SCHEME_BE, capi.SCHEME_EXPLICIT])
def test_scheme_fp64_parity(gpu, scheme):
    m = M.slab(11, 11, 4, 0.2, 0.2, 0.06)
    blk = M.corner_block(m, 3, 3)
    dt, idt, steps = 0.05, 0.01, 200
    cells = O.Cells(O.TUSSCHER, m.n, tt_jac_true=1, newton_cap=100)
    ref = _oracle(m, scheme, cells, dt, idt, steps, blk, 20)
    got = _gpu(m, scheme, capi.FP64, dt, idt, steps, blk, 1.0, capi.TT_JAC_TRUE)
    assert np.max(ref[-1]) > 0.0                     # the slab has fired
    worst = max(np.max(np.abs(a - b)) / np.max(np.abs(a)) for a, b in zip(ref, got))
    assert worst <= 1e-6, worst


def test_backward_euler_reference_cells(gpu):
    """Same, with the reference's own ten Tusscher objects in the oracle
    (transposed Jacobian, stable at these sub-steps)."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    m = M.slab(11, 11, 4, 0.2, 0.2, 0.06)
    blk = M.corner_block(m, 3, 3)
    dt, idt, steps = 0.02, 0.005, 200
    ref = _oracle(m, capi.SCHEME_BE, O.RefCells(O.TUSSCHER, m.n), dt, idt, steps, blk, 50)
    got = _gpu(m, capi.SCHEME_BE, capi.FP64, dt, idt, steps, blk, 1.0, capi.TT_JAC_REFERENCE)
    worst = max(np.max(np.abs(a - b)) / np.max(np.abs(a)) for a, b in zip(ref, got))
    assert worst <= 1e-6, worst


@pytest.mark.parametrize("scheme", [capi.SCHEME_BE, capi.SCHEME_EXPLICIT])
def test_scheme_fp32_fires(gpu, scheme):
    m = M.slab(11, 11, 4, 0.2, 0.2, 0.06)
    blk = M.corner_block(m, 3, 3)
    a = _gpu(m, scheme, capi.FP32, 0.05, 0.01, 200, blk, 1.0, capi.TT_JAC_TRUE)
    b = _gpu(m, scheme, capi.FP64, 0.05, 0.01, 200, blk, 1.0, capi.TT_JAC_TRUE)
    assert np.max(a[-1]) > 0.0
    assert np.max(np.abs(a[-1] - b[-1])) < 2.0       # mV, FP32 against FP64 after 10 ms
