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
    """The gather width (4, 8, 8 pipelined, or the staged kernel with its
    units of slice columns copied asynchronously into shared memory) changes
    which loads are in flight together, not the order of the additions: same
    bits on the same grid.  (The grid decides how the FP64 dot products are split over
    CTAs, so every kernel gets one CTA per SM: the staged kernel's ring can
    fill most of an SM's shared memory.)"""
    wl, V, c = shell
    out = []
    for nb, pf in ((4, 0), (8, 0), (16, 0), (32, 0), (32, 1), (32, 3), (32, 4)):   # pf: the staged ring's depth
        g = Monodomain(wl.mesh, capi.TUSSCHER, prec, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
        g.set_launch_config(cg_batch=nb, cg_per_sm=1, cg_prefetch=pf)
        g.set_voltage(V)
        it, rr = g.diffusion_half_step()
        out.append((g.voltage(), it))
        g.close()
    for x, it in out[1:]:
        assert it == out[0][1]
        assert np.array_equal(x, out[0][0])


def _slab_run(var=0, predict=0, prec=capi.FP64, steps=400, graph_steps=0):
    from ucla_cmg_b200 import mesh as M
    m = M.slab(21, 21, 5, 0.4, 0.4, 0.08)
    blk = M.corner_block(m, 3, 3)
    g = Monodomain(m, capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                   cg_tol=1e-10 if prec == capi.FP64 else 1e-7, tt_jacobian=capi.TT_JAC_TRUE)
    g.set_launch_config(cg_variant=var, cg_predict=predict, graph_steps=graph_steps)
    g.set_voltage(-85.423)
    g.set_stimulus(blk, 0.0, 1.0, 50.0 * 2000.0)
    st = g.step(steps)
    V = g.voltage()
    return g, V, st


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("predict", [1, 2])
def test_predictor_in_tissue(gpu, prec, predict):
    """Starting each solve from V + the previous correction of the same half
    step (or the linear extrapolation of the last two): the stop test is the
    reference's (relative to B V - A V), so the field agrees with the plain
    start to the CG tolerance's level, in fewer iterations, and no solve
    fails."""
    g0, V0, st0 = _slab_run(0, 0, prec)
    g0.close()
    g1, V1, st1 = _slab_run(0, predict, prec)
    assert g1.launch_config()["cg_predict"] == predict
    g1.close()
    assert np.max(V0) > 0.0
    assert st1["cg_failures"] == 0 and st1["nonfinite"] == 0
    tol = 1e-6 if prec == capi.FP64 else 2e-4
    assert np.max(np.abs(V0 - V1)) < tol * np.max(np.abs(V0)), np.max(np.abs(V0 - V1))
    assert st1["cg_iters"] < st0["cg_iters"], (st1["cg_iters"], st0["cg_iters"])


def test_predictor_restarts_on_voltage_upload(gpu):
    """A voltage upload restarts the predictor from zero, so a run from an
    uploaded state repeats bit for bit (also under graph replay)."""
    for gs, predict in ((0, 1), (50, 1), (50, 2)):
        g, V, st = _slab_run(0, predict, steps=100, graph_steps=gs)
        S = g.states()
        out = []
        for rep in range(2):
            g.set_states(S)
            g.set_voltage(V)
            g.step(100)
            out.append(g.voltage())
        g.close()
        assert np.max(out[0]) > 0.0
        assert np.array_equal(out[0], out[1])


def test_predictor_needs_two_reduction_variant(gpu):
    from ucla_cmg_b200 import mesh as M
    m = M.slab(6, 6, 3, 0.4, 0.4, 0.08)
    g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2))
    with pytest.raises(capi.EPError):
        g.set_launch_config(cg_variant=1, cg_predict=1)
    assert g.launch_config()["cg_predict"] == 0
    g.close()


def test_prefetch_changes_no_bits(gpu, shell):
    """The L2 prefetch of the next slice is a hint: same bits with it on."""
    wl, V, c = shell
    out = []
    for pf in (0, 2):
        g = Monodomain(wl.mesh, capi.TUSSCHER, capi.FP32, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
        g.set_launch_config(cg_batch=8, cg_per_sm=4, cg_prefetch=pf)
        g.set_voltage(V)
        it, rr = g.diffusion_half_step()
        out.append((g.voltage(), it))
        g.close()
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    with pytest.raises(capi.EPError):
        g = Monodomain(wl.mesh, capi.TUSSCHER, capi.FP32, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D)
        try:
            g.set_launch_config(cg_variant=1, cg_prefetch=2)
        finally:
            g.close()


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_staged_cg_in_tissue_is_bit_identical(gpu, prec):
    """The staged CG over a whole tissue run (predictor on, steps replayed
    from a CUDA graph): every step's solves give the bits of the gather-width
    8 kernel, so the fields after 400 steps are equal."""
    from ucla_cmg_b200 import mesh as M
    m = M.slab(23, 19, 5, 0.44, 0.36, 0.08)
    out = []
    for nb in (8, 32):
        g = Monodomain(m, capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                       tt_jacobian=capi.TT_JAC_TRUE)
        g.set_launch_config(cg_batch=nb, cg_predict=1, graph_steps=20)
        g.set_voltage(-85.423)
        g.set_stimulus(M.corner_block(m, 3, 3), 0.0, 1.0, 50.0 * 2000.0)
        st = g.step(400)
        assert st["cg_failures"] == 0 and st["timeouts"] == 0
        out.append((g.voltage(), st["cg_iters"]))
        g.close()
    assert np.max(out[0][0]) > 0.0
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


def test_staged_cg_batch_instances(gpu):
    """Independent instances in one staged launch (each CTA group streams
    its own instance's slices; the slices two instances share are masked):
    the same bits as gather width 8."""
    from ucla_cmg_b200 import mesh as M
    from ucla_cmg_b200.simulation import Batch
    insts = [dict(mesh=M.slab(nx, ny, 4, 0.02 * (nx - 1), 0.02 * (ny - 1), 0.06), D=M.sigma_to_D(1.2, 0.2))
             for nx, ny in ((13, 9), (21, 17), (7, 11))]
    out = []
    for nb in (8, 32):
        b = Batch(insts, capi.TUSSCHER, capi.FP32, dt=0.02, ionic_dt=0.02, tt_jacobian=capi.TT_JAC_TRUE)
        b.set_launch_config(cg_batch=nb)
        b.set_voltage(-85.423)
        ids = np.concatenate([M.corner_block(i["mesh"], 3, 3) + o for i, o in zip(insts, b.offsets[:-1])])
        b.set_stimulus(ids.astype(np.int32), 0.0, 1.0, 50.0 * 2000.0)
        st = b.step(200)
        assert st["cg_failures"] == 0
        out.append(b.voltage())
        b.close()
    assert np.array_equal(out[0], out[1])
