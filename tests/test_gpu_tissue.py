"""The full split step on the GPU vs the CPU oracle on small slabs.

FP64 bar: max |V_gpu - V_ref| <= 1e-6 * max |V_ref| at every checkpoint,
with the reference cell objects (oracle/_ref) or the C restatement in the
ionic phase and a tight CG tolerance on both sides so the two preconditioners
(AztecOO's and the GPU's) drop out.
"""
import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu
D = M.sigma_to_D(1.2, 0.2)


def _slab():
    return M.slab(13, 11, 5, 0.6, 0.5, 0.2)


def _oracle_sim(m, model, dt, idt, cg_tol, cells=None, jac=0):
    c = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, dt)
    if cells is None:
        cells = O.Cells(model, m.n, tt_jac_true=jac, newton_cap=100)
    s = O.Sim(c, cells, dt, idt, cg_tol=cg_tol, cg_maxit=2000, jacobi_steps=1)
    return c, cells, s


@pytest.mark.parametrize("use_ref", [True, False])
def test_tt_fp64_parity(gpu, use_ref):
    if use_ref and O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    m = _slab()
    dt = 0.01
    blk = M.corner_block(m, 3, 3)
    amp = 50.0 * 2000.0
    cells = O.RefCells(O.TUSSCHER, m.n) if use_ref else None
    c, cells, s = _oracle_sim(m, O.TUSSCHER, dt, dt, 1e-13, cells)
    s.V[:] = -85.423
    g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=dt, ionic_dt=dt, D=D, cg_tol=1e-13,
                   cg_maxit=2000)
    g.set_voltage(-85.423)
    g.set_stimulus(blk, 0.0, 1.0, amp)
    worst = 0.0
    for chk in range(4):                 # 4 x 5 ms
        for k in range(500):
            step = chk * 500 + k
            s.istim[:] = 0.0
            if step < 100:
                s.istim[blk] = amp
            s.step()
        g.step(500)
        Vg, Vo = g.voltage(), s.V.copy()
        worst = max(worst, np.max(np.abs(Vg - Vo)) / np.max(np.abs(Vo)))
    assert np.max(s.V) > 0.0                       # the wave is up
    assert worst <= 1e-6, worst
    g.close()


def test_mahajan_fp64_parity(gpu):
    m = _slab()
    dt, idt = 0.1, 0.05                             # the reference's own defaults
    types = (np.arange(m.n) % 9).astype(np.uint8)
    cells = O.Cells(O.MAHAJAN, m.n, types=types)
    c, cells, s = _oracle_sim(m, O.MAHAJAN, dt, idt, 1e-13, cells)
    V0 = cells.initial_voltage()
    s.V[:] = V0
    g = Monodomain(m, capi.MAHAJAN, capi.FP64, dt=dt, ionic_dt=idt, D=D, cg_tol=1e-13,
                   cg_maxit=2000, node_type=types)
    assert np.allclose(g.model_voltage(), V0)
    g.set_voltage(V0)
    blk = M.corner_block(m, 3, 3)
    amp = 50.0 * 1.55e-4 / 2.58e-8
    g.set_stimulus(blk, 0.0, 2.0, amp)
    worst = 0.0
    for chk in range(4):
        for k in range(100):
            step = chk * 100 + k
            s.istim[:] = 0.0
            if step < 20:
                s.istim[blk] = amp
            s.step()
        g.step(100)
        Vg, Vo = g.voltage(), s.V.copy()
        worst = max(worst, np.max(np.abs(Vg - Vo)) / np.max(np.abs(Vo)))
    assert np.max(s.V) > 0.0
    assert worst <= 1e-6, worst
    states = g.states()
    assert np.allclose(states[:, 1:], cells.state[:, 1:], rtol=1e-6, atol=1e-9)


def test_fp32_error_report(gpu):
    """FP32 vs FP64 on the GPU: errors are reported and bounded."""
    m = M.slab(21, 21, 4, 1.0, 1.0, 0.15)
    dt = 0.02
    blk = M.corner_block(m, 3, 3)
    amp = 50.0 * 2000.0
    runs = {}
    for prec in (capi.FP64, capi.FP32):
        g = Monodomain(m, capi.TUSSCHER, prec, dt=dt, ionic_dt=dt, D=D,
                       tt_jacobian=capi.TT_JAC_TRUE)
        g.set_voltage(-85.423)
        g.set_stimulus(blk, 0.0, 1.0, amp)
        g.step(2500)                             # 50 ms
        runs[prec] = (g.voltage(), g.activation()[0], g.last_stats)
        g.close()
    V64, ta64, st64 = runs[capi.FP64]
    V32, ta32, st32 = runs[capi.FP32]
    assert st64["cg_failures"] == 0 and st32["cg_failures"] == 0
    assert st64["nonfinite"] == 0 and st32["nonfinite"] == 0
    act64, act32 = ta64 >= 0, ta32 >= 0
    assert act64.mean() > 0.5                    # the wave crossed most of the slab
    assert np.mean(act64 != act32) < 0.01        # same activated set up to the front
    both = act64 & act32
    assert np.max(np.abs(ta32[both] - ta64[both])) < 0.1     # ms
    assert np.max(np.abs(V32 - V64)) < 5.0       # mV (behind a moving front)


def test_ecg_matches_oracle(gpu):
    m = _slab()
    g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=0.01, ionic_dt=0.01, D=D, ecg_every=50)
    g.set_voltage(-85.423)
    el = np.array([[2.3, 0.25, 0.1], [-1.7, 0.25, 0.1]])
    g.set_electrodes(el, D_ecg=[1e-3, 5e-4, 2.5e-4])
    g.set_stimulus(M.corner_block(m, 3, 3), 0.0, 1.0, 1e5)
    g.step(300)
    t, e = g.ecg()
    assert e.shape == (6, 2) and np.allclose(t, np.arange(1, 7) * 0.5)
    V = g.voltage()
    ref = O.ecg_elementwise(m.xyz, m.tets, m.fibers, [1e-3, 5e-4, 2.5e-4], el, V)
    now = g.compute_ecg()
    assert np.allclose(now, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    assert np.allclose(e[-1], now, rtol=1e-12)


def test_restart_round_trip(gpu, tmp_path):
    m = _slab()
    kw = dict(dt=0.02, ionic_dt=0.02, D=D, tt_jacobian=capi.TT_JAC_TRUE)
    a = Monodomain(m, capi.TUSSCHER, capi.FP64, **kw)
    a.set_voltage(-85.423)
    a.set_stimulus(M.corner_block(m, 3, 3), 0.0, 1.0, 1e5)
    a.step(200)
    a.write_output(4.0, tmp_path)
    a.write_restart(4.0, tmp_path)
    raw = np.fromfile(tmp_path / "Voltage_time_00004.00.00", dtype=np.float64)
    assert np.array_equal(raw, a.voltage())
    b = Monodomain(m, capi.TUSSCHER, capi.FP64, **kw)
    b.set_stimulus(M.corner_block(m, 3, 3), 0.0, 1.0, 1e5)
    b.read_restart(4.0, tmp_path)
    assert b.time()[1] == 200
    a.step(100)
    b.step(100)
    assert np.array_equal(a.voltage(), b.voltage())
    with open(tmp_path / "InterVariables_time_00004.00.00", "rb") as f:
        nv = np.frombuffer(f.read(4), dtype=np.int32)[0]
    assert nv == 19


def test_truncated_restart_is_an_error(gpu, tmp_path):
    m = _slab()
    a = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=D)
    a.write_restart(1.0, tmp_path)
    a.write_output(1.0, tmp_path)
    p = tmp_path / "InterVariables_time_00001.00.00"
    p.write_bytes(p.read_bytes()[:100])
    with pytest.raises(capi.EPError) as ei:
        a.read_restart(1.0, tmp_path)
    assert ei.value.code == -10


def test_cg_maxit_reports_failure(gpu):
    """Forced non-convergence (cg_maxit=1 with a tiny tolerance) is counted,
    not hidden."""
    m = _slab()
    g = Monodomain(m, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=D, cg_tol=1e-14,
                   cg_maxit=1)
    g.set_voltage(np.linspace(-85, 0, m.n))
    st = g.step(3)
    assert st["cg_failures"] == 6 and st["cg_max_iters"] == 1
