"""FP64 parity on the GPU at the benchmark configurations' own sizes.

Each test runs a configuration's mesh, cell set-up and time step through
the C ABI in FP64 and the same run on the CPU oracle (the C restatement of
EP_CrankNicholson::Solve, EP_CrankNicholson.cc:78-156, with the cell update
of CardiacBody::getIonicCurrent, CardiacBody.cc:405-435), with a tight CG
tolerance on both sides so that the two Jacobi preconditioners drop out.
Bar: max |V_gpu - V_cpu| <= 1e-6 max |V_cpu| at every checkpoint.

* C0 as configured: the 51 x 51 x 11 slab (28,611 nodes), fibres rotating
  -60..+60 degrees, the 5 x 5 x 11 corner stimulus, dt = 0.02 ms, ten
  Tusscher with the true-Jacobian Newton (the reference's transposed one
  diverges at this step), 10 ms; plus the pseudo-ECG at the two electrodes.
* C0's mesh at dt = 0.01 ms with the reference's own ten Tusscher objects
  (compiled from its sources), which that step keeps stable.
* C1: the 201 x 201 x 21 slab (848,421 nodes), Mahajan, dt = 0.01 ms, the
  x <= 0.1 cm strip stimulated, 1 ms; V and all 26 states.
* C3: three of the 64 batch instances (their own sizes, parameter scalings
  and corner stimuli) in one batch handle, each against its own oracle run.
"""
import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, workloads as W
from ucla_cmg_b200.simulation import Batch, Monodomain

pytestmark = pytest.mark.gpu
TOL = 1e-6
CG_TOL = 1e-13


def _oracle(wl, cells, dt, idt):
    c = O.Csr(wl.mesh.xyz, wl.mesh.tets, wl.mesh.fibers, wl.D, 1.0, dt)
    s = O.Sim(c, cells, dt, idt, cg_tol=CG_TOL, cg_maxit=4000, jacobi_steps=1)
    return c, s


def _windows(ids, t_on, t_off, dt):
    on = (np.asarray(t_on) / dt).astype(np.int64)
    off = (np.asarray(t_off) / dt).astype(np.int64)
    return np.asarray(ids), on, off


def _advance(s, k0, k1, stim, amp):
    ids, on, off = stim
    for k in range(k0, k1):
        s.istim[:] = 0.0
        live = (on <= k) & (k < off)
        s.istim[ids[live]] = amp[live] if np.ndim(amp) else amp
        s.step()


def _worst(Vg, Vo):
    return float(np.max(np.abs(Vg - Vo)) / np.max(np.abs(Vo)))


def test_c0_as_configured(gpu):
    wl = W.slab_c0()
    assert wl.mesh.n == 28611 and len(wl.stim_ids) == 275
    O.set_threads(0)
    cells = O.Cells(O.TUSSCHER, wl.mesh.n, tt_jac_true=1, newton_cap=100)
    c, s = _oracle(wl, cells, wl.dt, wl.ionic_dt)
    s.V[:] = wl.V0
    g = wl.create(capi.FP64, cg_tol=CG_TOL, cg_maxit=4000)
    stim = _windows(wl.stim_ids, wl.stim_on, wl.stim_off, wl.dt)
    worst = 0.0
    for chk in range(4):                                   # 4 x 2.5 ms
        _advance(s, chk * 125, (chk + 1) * 125, stim, wl.stim_amp)
        st = g.step(125)
        assert st["cg_failures"] == 0 and st["newton_cap_hits"] == 0
        worst = max(worst, _worst(g.voltage(), s.V))
    assert np.max(s.V) > 0.0                               # the wave is running
    assert worst <= TOL, worst
    # the pseudo-ECG of the final field at the configuration's electrodes
    W_ecg = O.ecg_weights(wl.mesh.xyz, wl.mesh.tets, wl.mesh.fibers, wl.D, wl.electrodes)
    e_cpu = W_ecg @ s.V
    e_gpu = g.compute_ecg()
    assert np.max(np.abs(e_gpu - e_cpu)) <= TOL * np.max(np.abs(e_cpu))
    g.close()


def test_c0_mesh_reference_cell_objects(gpu):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    wl = W.slab_c0()
    dt = 0.01
    O.set_threads(0)
    cells = O.RefCells(O.TUSSCHER, wl.mesh.n)
    c, s = _oracle(wl, cells, dt, dt)
    s.V[:] = wl.V0
    g = Monodomain(wl.mesh, capi.TUSSCHER, capi.FP64, dt=dt, ionic_dt=dt, D=wl.D, cg_tol=CG_TOL,
                   cg_maxit=4000, tt_jacobian=capi.TT_JAC_REFERENCE)
    g.set_voltage(wl.V0)
    g.set_stimulus(wl.stim_ids, wl.stim_on, wl.stim_off, wl.stim_amp)
    stim = _windows(wl.stim_ids, wl.stim_on, wl.stim_off, dt)
    worst = 0.0
    for chk in range(3):                                   # 3 x 2 ms
        _advance(s, chk * 200, (chk + 1) * 200, stim, wl.stim_amp)
        g.step(200)
        worst = max(worst, _worst(g.voltage(), s.V))
    assert np.max(s.V) > 0.0
    assert worst <= TOL, worst
    g.close()


def test_c1_mahajan_full_size(gpu):
    wl = W.slab_c1()
    assert wl.mesh.n == 848421
    O.set_threads(0)
    cells = O.Cells(O.MAHAJAN, wl.mesh.n, types=wl.node_type)
    c, s = _oracle(wl, cells, wl.dt, wl.ionic_dt)
    V0 = cells.initial_voltage()
    s.V[:] = V0
    g = wl.create(capi.FP64, cg_tol=CG_TOL, cg_maxit=4000)
    assert np.allclose(g.model_voltage(), V0)
    g.set_voltage(V0)
    stim = _windows(wl.stim_ids, wl.stim_on, wl.stim_off, wl.dt)
    worst = 0.0
    for chk in range(2):                                   # 2 x 0.5 ms
        _advance(s, chk * 50, (chk + 1) * 50, stim, wl.stim_amp)
        st = g.step(50)
        assert st["cg_failures"] == 0
        worst = max(worst, _worst(g.voltage(), s.V))
    assert np.max(s.V[wl.stim_ids]) > -20.0                # the strip is depolarising
    assert worst <= TOL, worst
    S = g.states()
    assert np.allclose(S[:, 1:], cells.state[:, 1:], rtol=1e-6, atol=1e-9)
    g.close()


def test_c3_instances_against_the_oracle(gpu):
    wl = W.batch_c3()
    picks = [0, 1, 2]
    insts = [wl.instances[k] for k in picks]
    b = Batch(insts, capi.TUSSCHER, capi.FP64, dt=wl.dt, ionic_dt=wl.ionic_dt, cg_tol=CG_TOL, cg_maxit=4000,
              tt_jacobian=capi.TT_JAC_TRUE)
    b.set_voltage(wl.V0)
    # the picked instances' stimulus blocks, renumbered into the small batch
    full_off = np.concatenate([[0], np.cumsum([inst["mesh"].n for inst in wl.instances])])
    ids, off = [], 0
    for k in picks:
        sel = (wl.stim_ids >= full_off[k]) & (wl.stim_ids < full_off[k + 1])
        ids.append(wl.stim_ids[sel] - full_off[k] + off)
        off += wl.instances[k]["mesh"].n
    ids = np.concatenate(ids).astype(np.int32)
    b.set_stimulus(ids, 0.0, 1.0, wl.stim_amp[0])
    O.set_threads(0)
    sims = []
    for j, k in enumerate(picks):
        inst = wl.instances[k]
        m = inst["mesh"]
        cells = O.Cells(O.TUSSCHER, m.n, types=np.zeros(m.n, np.uint8), type_consts=inst["type_consts"],
                        tt_jac_true=1, newton_cap=100)
        cc = O.Csr(m.xyz, m.tets, m.fibers, inst["D"], 1.0, wl.dt)
        s = O.Sim(cc, cells, wl.dt, wl.ionic_dt, cg_tol=CG_TOL, cg_maxit=4000, jacobi_steps=1)
        s.V[:] = wl.V0
        loc = ids[(ids >= b.offsets[j]) & (ids < b.offsets[j + 1])] - b.offsets[j]
        sims.append((cc, cells, s, loc))
    worst = 0.0
    for chk in range(3):                                   # 3 x 2 ms
        for cc, cells, s, loc in sims:
            for k in range(chk * 100, (chk + 1) * 100):
                s.istim[:] = 0.0
                if k < 50:
                    s.istim[loc] = wl.stim_amp[0]
                s.step()
        b.step(100)
        for (cc, cells, s, loc), Vg in zip(sims, b.split(b.voltage())):
            worst = max(worst, _worst(Vg, s.V))
    assert all(np.max(s.V) > 0.0 for _, _, s, _ in sims)
    assert worst <= TOL, worst
    b.close()
