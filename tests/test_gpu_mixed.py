"""Mixed tissues on the GPU (ep_create_mixed): a slab of ten Tusscher tissue
with a Purkinje cable reaching into it, against the oracle's mixed split
step.

The reference gives every .purk node a Purkinje cell and every other node
the tissue model (CardiacBody::New, CardiacBody.cc:982-1101); the 2-node
cables join the tets in the operators (MixedMesh3D.cc:62-108,
CardiacBody.cc:100-187).  The oracle runs the same split step with its C
restatement of both cell models (pinned to the reference's own objects in
tests/test_oracle.py) or the reference objects themselves; a tight CG
tolerance on both sides takes the preconditioners out.  Bar: FP64 max
|V_gpu - V_cpu| <= 1e-6 max |V_cpu| at every checkpoint, the cable's
stimulus conducting into the slab.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M, voomep_io as IO
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu
CG_TOL = 1e-13


def _case(k=6, h=0.05):
    """A 7 x 6 x 3 slab and a k-node cable hanging from its corner node 0."""
    m = M.slab(7, 6, 3, 0.3, 0.25, 0.1)
    n0 = m.n
    extra = m.xyz[[0]] + np.stack([np.zeros(k), np.zeros(k), -h * np.arange(1, k + 1)], 1)
    xyz = np.vstack([m.xyz, extra])
    mesh = M.TetMesh(xyz, m.tets, m.fibers, {})
    bars = np.array([[0, n0]] + [[n0 + j, n0 + j + 1] for j in range(k - 1)], np.int32)
    purk = np.arange(n0, n0 + k)
    return mesh, bars, purk, n0


@pytest.mark.parametrize("cells", ["restatement", "reference"])
def test_mixed_tissue_fp64_against_the_oracle(gpu, cells):
    if cells == "reference" and O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    mesh, bars, purk, n0 = _case()
    n = mesh.n
    D = M.sigma_to_D(1.2, 0.2)
    cab = dict(bars=bars, Dp=(0.0016,) * 3, DpLeft=(0.0016,) * 3, radius=0.0275)
    dt = 0.01
    g = Monodomain(mesh, capi.TUSSCHER, capi.FP64, dt=dt, ionic_dt=dt, D=D, cg_tol=CG_TOL, cg_maxit=4000,
                   tt_jacobian=capi.TT_JAC_REFERENCE, cables=cab, purkinje=purk)
    assert g.nstate == 22
    far = np.array([n - 1, n - 2], np.int32)                 # the cable's free end
    amp = 250000.0
    g.set_stimulus(far, 0.0, 2.0, amp)
    V0 = g.voltage()
    assert np.allclose(V0[purk], O.initial_state(O.PURKINJE)[0])
    is_purk = np.zeros(n, np.uint8)
    is_purk[purk] = 1
    nt, npk = int((is_purk == 0).sum()), int(is_purk.sum())
    if cells == "reference":
        tissue, pk = O.RefCells(O.TUSSCHER, nt), O.RefCells(O.PURKINJE, npk)
    else:
        tissue, pk = O.Cells(O.TUSSCHER, nt), O.Cells(O.PURKINJE, npk)
    mc = O.MixedCells(tissue, pk, is_purk)
    csr = O.Csr(mesh.xyz, mesh.tets, mesh.fibers, D, 1.0, dt, cables=O.Cables(bars, radius=0.0275))
    s = O.Sim(csr, mc, dt, dt, cg_tol=CG_TOL, cg_maxit=4000, jacobi_steps=1)
    s.V[:] = V0
    worst = 0.0
    for chk in range(6):                                     # 6 x 1 ms
        for kk in range(100):
            step = chk * 100 + kk
            s.istim[:] = 0.0
            if step < 200:
                s.istim[far] = amp
            s.step()
        st = g.step(100)
        assert st["cg_failures"] == 0
        worst = max(worst, float(np.max(np.abs(g.voltage() - s.V)) / np.max(np.abs(s.V))))
    assert worst <= 1e-6, worst
    # the stimulus at the cable's end reached the slab through the junction
    ta = g.activation()[0]
    assert ta[n - 1] >= 0.0 and ta[0] > ta[n - 1]
    assert np.max(s.V[:n0]) > 0.0
    g.close()


def test_mixed_states_and_restart_files(gpu, tmp_path):
    """Rows of 22 values for Purkinje nodes and 19 (zero-padded) for tissue
    nodes; the restart file keeps each node's own nVar; a state written and
    read back continues bit for bit."""
    mesh, bars, purk, n0 = _case()
    n = mesh.n

    def mk():
        return Monodomain(mesh, capi.TUSSCHER, capi.FP32, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                          tt_jacobian=capi.TT_JAC_TRUE, cables=dict(bars=bars), purkinje=purk)
    g = mk()
    g.set_stimulus(np.array([n - 1], np.int32), 0.0, 2.0, 250000.0)
    g.step(150)
    S = g.states()
    assert S.shape == (n, 22)
    assert np.all(S[:n0, 19:] == 0.0) and np.any(S[purk, 21] != 0.0)
    g.write_restart(3.0, str(tmp_path))
    g.write_output(3.0, str(tmp_path))
    rows = IO.read_intervariables(IO.output_name(str(tmp_path), "InterVariables", 3.0))
    assert [len(r) for r in rows] == [19] * n0 + [22] * len(purk)
    assert np.array_equal(np.array(rows[n - 1]), S[n - 1])
    g.step(100)
    V_cont = g.voltage()
    h = mk()
    h.set_stimulus(np.array([n - 1], np.int32), 0.0, 2.0, 250000.0)
    h.read_restart(3.0, str(tmp_path))
    assert h.time()[1] == 150
    h.step(100)
    assert np.array_equal(h.voltage(), V_cont)
    S2 = h.states()
    h.set_states(S2)
    assert np.array_equal(h.states(), S2)
    g.close()
    h.close()


def test_mixed_tissue_ecg_includes_the_cables(gpu):
    """The in-run pseudo-ECG of a mixed tissue integrates over the cables as
    ComputeECG does on a MIX3D mesh (tissue D along the cable, radius 0.0275
    cm): equal to the oracle's weights, tets plus cables."""
    mesh, bars, purk, n0 = _case()
    D = M.sigma_to_D(1.2, 0.2)
    g = Monodomain(mesh, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=D, tt_jacobian=capi.TT_JAC_TRUE,
                   cables=dict(bars=bars, radius=0.05), purkinje=purk)
    el = np.array([[0.15, 0.12, 2.0], [0.0, 0.0, -0.5], [-3.0, 0.1, 0.0]])
    g.set_electrodes(el)
    rng = np.random.default_rng(8)
    V = -85.0 + 100.0 * (mesh.xyz[:, 2] < -0.1) + rng.normal(0.0, 1.0, mesh.n)
    g.set_voltage(V)
    e = g.compute_ecg()
    Wc = O.ecg_weights(mesh.xyz, mesh.tets, mesh.fibers, D, el, cables=O.Cables(bars, radius=0.0275))
    assert np.max(np.abs(e - Wc @ V)) <= 1e-9 * np.max(np.abs(Wc @ V))
    g.close()


def test_driver_runs_a_mix3d_case_like_the_oracle_driver(gpu, tmp_path):
    """An EPSimulator input over a MIX3D mesh (tets + cable, .purk) through
    the GPU driver and through the oracle's EPSimulator loop: the same
    Voltage_time_* frames (FP64, tight CG on both sides) and the same
    InterVariables layout."""
    from ucla_cmg_b200 import driver as D
    from oracle import driver_oracle as DO
    from tests.test_driver import _mix_case
    inp, n0, k = _mix_case(tmp_path)
    out_gpu, out_cpu = str(tmp_path / "gpu"), str(tmp_path / "cpu")
    cfg, nsteps = D.run(inp, capi.FP64, rest_voltage=True, verbose=False, tt_jacobian=capi.TT_JAC_REFERENCE,
                        cg_tol=CG_TOL)
    os.rename(os.path.join(cfg["input_dir"], cfg["output_dir"]), out_gpu)
    DO.run(inp, out_cpu, reference_cells=False, rest_voltage=True, cg_tol=CG_TOL, jacobi_steps=1)
    for t in (0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0):
        a = IO.read_voltage(IO.output_name(out_cpu, "Voltage", t))
        b = IO.read_voltage(IO.output_name(out_gpu, "Voltage", t))
        assert len(a) == len(b) == n0 + k
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(a)), t
    ra = IO.read_intervariables(IO.output_name(out_cpu, "InterVariables", 6.0))
    rb = IO.read_intervariables(IO.output_name(out_gpu, "InterVariables", 6.0))
    assert [len(r) for r in ra] == [len(r) for r in rb] == [19] * n0 + [22] * k
