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


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("batch", [4, 8])
def test_single_reduction_variant_matches_oracle(gpu, shell, prec, batch):
    """The Chronopoulos-Gear launch option (one reduction per iteration)
    solves the same system to the same tolerance: iteration count within one
    of the oracle's PCG, solution within the tolerance the two-reduction
    kernel is held to."""
    wl, V, c = shell
    B = c.scipy("B")
    x_ref, it_ref, rr_ref = c.pcg(B @ V, V.copy(), tol=1e-7, maxit=1000, jacobi_steps=1)
    g = Monodomain(wl.mesh, capi.TUSSCHER, prec, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
    g.set_launch_config(cg_variant=1, cg_batch=batch, cg_per_sm=0)
    assert g.launch_config()["cg_variant"] == 1
    for rep in range(2):                      # the buffers' contents of one solve do not leak into the next
        g.set_voltage(V)
        it, rr = g.diffusion_half_step()
        x = g.voltage()
        if prec == capi.FP64:
            assert abs(it - it_ref) <= 1, (it, it_ref)
            assert rr <= 1e-7
            assert np.max(np.abs(x - x_ref)) < 1e-6 * np.max(np.abs(x_ref))
        else:
            assert it <= it_ref + 2, (it, it_ref)
            assert np.max(np.abs(x - x_ref)) < 1e-4 * np.max(np.abs(x_ref))
    g.close()


def test_single_reduction_variant_in_tissue(gpu):
    """Whole split steps with either CG variant (FP64, slab with a wave):
    the voltage fields agree to the CG tolerance's level."""
    from ucla_cmg_b200 import mesh as M
    m = M.slab(21, 21, 5, 0.4, 0.4, 0.08)
    blk = M.corner_block(m, 3, 3)
    out = []
    for var in (0, 1):
        g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                       cg_tol=1e-10, tt_jacobian=capi.TT_JAC_TRUE)
        g.set_launch_config(cg_variant=var)
        g.set_voltage(-85.423)
        g.set_stimulus(blk, 0.0, 1.0, 50.0 * 2000.0)
        g.step(400)
        out.append(g.voltage())
        g.close()
    assert np.max(out[0]) > 0.0
    assert np.max(np.abs(out[0] - out[1])) < 1e-6 * np.max(np.abs(out[0]))


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_gather_widths_are_bit_identical(gpu, shell, prec):
    """The gather width (4, 8, or 8 pipelined) changes which loads are in
    flight together, not the order of the additions: same bits."""
    wl, V, c = shell
    out = []
    for nb in (4, 8, 16):
        g = Monodomain(wl.mesh, capi.TUSSCHER, prec, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
        g.set_launch_config(cg_batch=nb, cg_per_sm=4)
        g.set_voltage(V)
        it, rr = g.diffusion_half_step()
        out.append((g.voltage(), it))
        g.close()
    for x, it in out[1:]:
        assert it == out[0][1]
        assert np.array_equal(x, out[0][0])
