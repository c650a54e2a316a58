"""The CPU oracle pinned against the reference (CPU-only tests).

* the C restatement of the cell models vs the golden vectors made by the
  reference's own cell-model sources (tests/golden/make_golden.py) and vs
  those sources run live (oracle/_ref) where built;
* the FEM restatement vs the reference's quadrature/shape self-checks
  (TetQuadrature::check, Shape::checkC0Completeness) re-expressed as
  properties: M row sums = element volume / 4 with the truncated rule,
  K 1 = 0, symmetry, positivity;
* the ECG per-node weights vs the element-wise formula of ComputeECG.h;
* the stimulus schedule and step count of the EPSimulator main loop.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import mesh as M

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = {"tt": O.TUSSCHER, "mahajan": O.MAHAJAN, "mahajan_fail": O.MAHAJAN_FAIL,
         "lr": O.LUORUDY, "lrgate": O.LUORUDYWITHGATE, "purkinje": O.PURKINJE}
XI = {O.TUSSCHER: 2000.0, O.MAHAJAN: 1.55e-4 / 2.58e-8, O.MAHAJAN_FAIL: 1.55e-4 / 2.58e-8,
      O.LUORUDY: 2 * (11e-4 + 100e-4) / (11e-4 * 100e-4),
      O.LUORUDYWITHGATE: 2 * (11e-4 + 100e-4) / (11e-4 * 100e-4), O.PURKINJE: 2500.0}


@pytest.mark.parametrize("name", list(NAMES))
def test_kat_single_call(name):
    """One Compute_Ion call on 128-384 states: the restatement reproduces the
    reference's outputs (states and returned dV/dt) to rounding."""
    g = np.load(os.path.join(GOLD, f"kat_{name}.npz"))
    model = NAMES[name]
    types = g["types"] if model in (O.MAHAJAN, O.MAHAJAN_FAIL) else None
    c = O.Cells(model, len(g["V"]), types=types)
    c.state[:] = g["states_in"]
    dv = c.compute_ion(g["V"], g["istim"], float(g["dt"]))
    scale = np.maximum(np.abs(g["dvdt"]), 1.0)
    assert np.max(np.abs(dv - g["dvdt"]) / scale) < 1e-9
    so, sr = c.state, g["states_out"]
    mask = np.ones(sr.shape[1], bool)
    if model in (O.LUORUDY, O.LUORUDYWITHGATE):
        mask[7] = False                  # _in[7] = V is not advanced by the model
    rel = np.abs(so - sr)[:, mask] / np.maximum(np.abs(sr[:, mask]), 1e-12)
    assert np.max(rel) < 1e-9


@pytest.mark.parametrize("name", list(NAMES))
def test_trajectory(name):
    """A full single-cell action potential (400-500 ms) under the split
    update matches the reference's trajectory."""
    g = np.load(os.path.join(GOLD, f"cell_{name}.npz"))
    model = NAMES[name]
    dt = float(g["dt"])
    t_stim = float(g["t_stim"])
    types = g["types"] if len(g["types"]) else None
    n = len(types) if types is not None else 1
    c = O.Cells(model, n, types=types)
    st = c.state
    V = (np.full(n, -84.0) if model in (O.LUORUDY, O.LUORUDYWITHGATE) else st[:, 0].copy())
    nsteps = int(round(g["t"][-1] / dt)) + int(round(1.0 / dt))
    every = int(round(1.0 / dt))
    Vs = []
    for k in range(nsteps):
        ist = np.full(n, 50.0 * XI[model] if t_stim <= k * dt < t_stim + 1.0 else 0.0)
        if k % every == 0:
            Vs.append(V.copy())
        V = V + dt * c.compute_ion(V, ist, dt)
    Vs = np.array(Vs)
    assert Vs.shape == g["V"].shape
    assert np.max(np.abs(Vs - g["V"])) < 1e-6          # mV
    assert np.max(np.abs(V - g["V_end"])) < 1e-6


def test_live_reference_matches():
    """Where oracle/_ref is built: restatement == reference objects, step by
    step, for TT (both Newton layouts tried on the restatement side)."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    n = 4
    ref = O.RefCells(O.TUSSCHER, n)
    port = O.Cells(O.TUSSCHER, n)
    V = np.array([-85.423, -80.0, -60.0, -20.0])
    for k in range(200):
        ist = np.where(np.arange(n) == 0, 1e5 if k < 50 else 0.0, 0.0)
        a = ref.compute_ion(V, ist, 0.01)
        b = port.compute_ion(V, ist, 0.01)
        assert np.max(np.abs(a - b)) <= 1e-9 * max(1.0, np.max(np.abs(a)))
        V = V + 0.01 * a
    assert np.allclose(ref.state, port.state, rtol=1e-10, atol=1e-14)


def test_live_reference_matches_purkinje():
    """Where oracle/_ref is built: the Purkinje restatement equals the
    reference's Purkinje objects bit for bit through an action potential,
    both branches of its adaptive forward Euler (|dV/dt| > 1.5 takes ten
    dt/10 steps) included."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    n = 3
    ref = O.RefCells(O.PURKINJE, n)
    port = O.Cells(O.PURKINJE, n)
    V = np.array([-88.34, -70.0, -30.0])
    fast = 0
    for k in range(2000):
        ist = np.where(np.arange(n) == 0, 50.0 * 2500.0 if 100 <= k < 150 else 0.0, 0.0)
        a = ref.compute_ion(V, ist, 0.02)
        b = port.compute_ion(V, ist, 0.02)
        assert np.array_equal(a, b)
        fast += int(np.sum(np.abs(a) > 1.5))
        V = V + 0.02 * a
    assert fast > 0
    assert np.array_equal(ref.state, port.state)


def test_tt_reference_jacobian_diverges_at_dt_002():
    """Parity hazard: with the reference's Jacobian layout (J^T through the
    column-major dgesv_) the TT Newton solve blows up at dt = 0.02 ms within
    the first action potential; with J itself it does not."""
    outs = {}
    for jac in (0, 1):
        c = O.Cells(O.TUSSCHER, 1, tt_jac_true=jac, newton_cap=200)
        V = np.array([-85.423])
        finite = True
        for k in range(500):                       # 10 ms
            ist = np.array([1e5 if k < 50 else 0.0])
            V = V + 0.02 * c.compute_ion(V, ist, 0.02)
            if not np.all(np.isfinite(V)) or abs(V[0]) > 500:
                finite = False
                break
        outs[jac] = finite
    assert outs[1] is True
    assert outs[0] is False


def test_mahajan_abs_modes_differ_only_in_trigger():
    c0 = O.Cells(O.MAHAJAN, 1, types=np.array([0], np.uint8), mh_abs_mode=0)
    c1 = O.Cells(O.MAHAJAN, 1, types=np.array([0], np.uint8), mh_abs_mode=1)
    V = c0.initial_voltage()
    a = c0.compute_ion(V, np.zeros(1), 0.02)
    b = c1.compute_ion(V, np.zeros(1), 0.02)
    assert abs(a[0]) < 20 and np.allclose(a, b)


# ------------------------------------------------------------------ FEM
@pytest.fixture(scope="module")
def small_slab():
    return M.slab(9, 7, 4, 0.8, 0.6, 0.3)


def test_mass_and_stiffness_properties(small_slab):
    m = small_slab
    D = M.sigma_to_D(1.2, 0.2)
    c = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, 0.02)
    assert not c.degenerate
    K, Mm = c.scipy("K"), c.scipy("M")
    one = np.ones(c.n)
    assert np.max(np.abs(K @ one)) < 1e-14 * np.max(np.abs(K.data))
    assert abs((K - K.T)).max() < 1e-14 * np.max(np.abs(K.data))
    assert abs((Mm - Mm.T)).max() == 0.0
    # lumped capacitance = row sums of M (Cm = 1); total = volume
    vol = m.volumes().sum()
    assert np.isclose(c.arr("CL").sum(), vol, rtol=1e-12)
    assert np.allclose(np.asarray(Mm.sum(axis=1)).ravel(), c.arr("CL"), rtol=1e-12)
    # 4-point rule with the truncated coordinates: M_e(a,b) = wJ sum_q N_qa N_qb
    qa, qb = 0.58541020, 0.13819660
    N = np.array([[1 - qa - 2 * qb, qa, qb, qb], [1 - qa - 2 * qb, qb, qa, qb],
                  [1 - qa - 2 * qb, qb, qb, qa], [1 - 3 * qb, qb, qb, qb]])
    Me = N.T @ N / 4.0
    assert abs(Me.sum() - 1.0) < 1e-12                  # partition of unity
    # A = M + dt/4 K, B = M - dt/4 K
    A, B = c.scipy("A"), c.scipy("B")
    assert abs(A + B - 2 * Mm).max() < 1e-14
    assert abs(A - B - 0.01 * K).max() < 1e-15
    # positive definite A: smallest eigenvalue > 0
    w = np.linalg.eigvalsh(A.toarray())
    assert w.min() > 0


def test_quadrature_exactness():
    """TetQuadrature::check analogue: the order-2 rule integrates quadratics
    on the reference tet to the truncation level of its coordinates."""
    qa, qb = 0.58541020, 0.13819660
    pts = np.array([[qa, qb, qb], [qb, qa, qb], [qb, qb, qa], [qb, qb, qb]])
    w = np.full(4, 1.0 / 24.0)
    # exact integrals over the unit tet: 1 -> 1/6, x -> 1/24, x^2 -> 1/60, xy -> 1/120
    assert abs(w.sum() - 1 / 6) < 1e-15
    assert abs((w * pts[:, 0]).sum() - 1 / 24) < 1e-8
    assert abs((w * pts[:, 0] ** 2).sum() - 1 / 60) < 1e-8
    assert abs((w * pts[:, 0] * pts[:, 1]).sum() - 1 / 120) < 1e-8


def test_pcg_solves(small_slab):
    m = small_slab
    c = O.Csr(m.xyz, m.tets, m.fibers, M.sigma_to_D(1.2, 0.2), 1.0, 0.5)
    rng = np.random.default_rng(0)
    x_true = rng.normal(size=c.n)
    A = c.scipy("A")
    b = A @ x_true
    for k in (1, 3):
        x, it, rr = c.pcg(b, np.zeros(c.n), tol=1e-12, maxit=500, jacobi_steps=k)
        assert it > 0 and rr <= 1e-12
        assert np.max(np.abs(x - x_true)) < 1e-9


def test_ecg_weights_match_elementwise(small_slab):
    m = small_slab
    D = np.array([1e-3, 5e-4, 2.5e-4])
    el = np.array([[2.5, 0.3, 0.15], [-1.5, 0.3, 0.15], [0.4, 0.3, 3.0]])
    rng = np.random.default_rng(3)
    W = O.ecg_weights(m.xyz, m.tets, m.fibers, D, el)
    for _ in range(3):
        V = rng.normal(size=m.n) * 30 - 50
        e1 = O.ecg_elementwise(m.xyz, m.tets, m.fibers, D, el, V)
        e2 = W @ V
        assert np.allclose(e1, e2, rtol=1e-10, atol=1e-14 * np.abs(e1).max())
    # a uniform field has no gradient and no ECG
    assert np.max(np.abs(W @ np.ones(m.n))) < 1e-14 * np.abs(W).sum()


def test_stimulus_schedule_single_pointer():
    """EPSimulator.cc:483-570: stimuli are consumed in list order with one
    pending start and one pending stop pointer; a stimulus listed after a
    later one is skipped."""
    s0, s1 = O.stim_schedule([0.0, 400.0], [5.0, 405.0], 0.1, 6000)
    assert list(s0) == [0, 4000] and list(s1) == [50, 4050]
    s0, s1 = O.stim_schedule([10.0, 5.0], [11.0, 6.0], 0.1, 500)
    assert list(s0) == [100, -1]


def test_num_steps_accumulation():
    """while (simtime < T) simtime += dt counts float accumulation."""
    assert O.num_steps(0.1, 1.0) in (10, 11)
    assert O.num_steps(0.5, 2.0) == 4


def test_substep_schedule():
    """EP_CrankNicholson.cc:114-143 ionic sub-steps, double arithmetic."""
    m = M.slab(3, 3, 3, 0.1, 0.1, 0.1)
    c = O.Csr(m.xyz, m.tets, None, (1e-3, 1e-3, 1e-3), 1.0, 0.1)
    cells = O.Cells(O.TUSSCHER, m.n)
    s = O.Sim(c, cells, 0.1, 0.02)
    sub = s.sub_dt
    assert abs(sum(sub) - 0.1) < 1e-15 and len(sub) in (5, 6)
    s2 = O.Sim(c, cells, 0.02, 0.05)
    assert s2.sub_dt == [0.02]


def _cable(k=5, h=0.1, axis=0):
    xyz = np.zeros((k + 1, 3))
    xyz[:, axis] = np.arange(k + 1) * h
    bars = np.stack([np.arange(k), np.arange(1, k + 1)], 1)
    return xyz, bars


def test_cable_elements_match_the_closed_form():
    """A straight Purkinje cable of 2-node elements (MixedMesh3D beam branch,
    two Gauss points): K = 2 Dp pi r^2 C_m / h * tridiag(-1, 2, -1), M row sums
    = C_L / C_m, K 1 = 0, symmetric, and the total mass is 2 pi r^2 L -- twice
    the cylinder's volume, because the reference scales Gauss weights that sum
    to 2 by the element length (parity hazard, kept)."""
    k, h, r, Dp, Cm = 6, 0.05, 0.0275, 0.0016, 1.3
    xyz, bars = _cable(k, h, axis=1)
    c = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=O.Cables(bars, Dp=(Dp,) * 3, radius=r), Cm=Cm, dt=0.1)
    K = c.scipy("K").toarray()
    M = c.scipy("M").toarray()
    ref = 2 * Dp * np.pi * r * r * Cm / h * (2 * np.eye(k + 1) - np.eye(k + 1, k=1) - np.eye(k + 1, k=-1))
    ref[0, 0] = ref[-1, -1] = 2 * Dp * np.pi * r * r * Cm / h
    assert np.allclose(K, ref, rtol=1e-12, atol=1e-18)
    assert np.allclose(K, K.T, rtol=0, atol=1e-18)
    assert np.max(np.abs(K.sum(1))) < 1e-15
    assert np.isclose(M.sum(), 2 * np.pi * r * r * k * h, rtol=1e-12)
    assert np.allclose(M.sum(1) * Cm, c.arr("CL"), rtol=1e-12)
    # A = Cm M + dt/4 K, B = Cm M - dt/4 K on the same pattern
    assert np.allclose(c.scipy("A").toarray(), Cm * M + 0.1 / 4 * K, rtol=1e-12, atol=1e-18)


def test_mixed_mesh_is_tets_plus_cables(small_slab):
    """Tets and cables sharing nodes: the mixed operators are the sum of the
    tet-only and the cable-only operators; the LV flag selects DpLeft."""
    m = small_slab
    n0 = m.n
    # a cable from three surface nodes of the slab out to two extra nodes
    extra = m.xyz[[0]] + np.array([[0.0, 0.0, -0.05], [0.0, 0.0, -0.1]])
    xyz = np.vstack([m.xyz, extra])
    bars = np.array([[1, 0], [0, n0], [n0, n0 + 1]])
    D = (1.2e-3, 2e-4, 2e-4)
    lv = np.array([0, 1, 1], np.uint8)
    cb = O.Cables(bars, Dp=(0.0016,) * 3, DpLeft=(0.003,) * 3, lv=lv, radius=0.02)
    mix = O.Csr(xyz, m.tets, m.fibers, D, 1.0, 0.1, cables=cb)
    tet = O.Csr(xyz, m.tets, m.fibers, D, 1.0, 0.1)
    only = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=cb, D=D, Cm=1.0, dt=0.1)
    for name in ("K", "M", "A", "B"):
        diff = mix.scipy(name) - tet.scipy(name) - only.scipy(name)
        assert abs(diff).max() <= 1e-15 * max(1.0, abs(mix.scipy(name)).max())
    assert np.allclose(mix.arr("CL"), tet.arr("CL") + only.arr("CL"), rtol=1e-13)
    # the LV bars conduct with DpLeft: stiffness scales with D along the bar
    lvK = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=O.Cables(bars, Dp=(0.0016,) * 3, DpLeft=(0.0016,) * 3,
                                                             lv=lv, radius=0.02), D=D, Cm=1.0, dt=0.1)
    k1 = only.scipy("K").toarray()[n0, n0 + 1]
    k2 = lvK.scipy("K").toarray()[n0, n0 + 1]
    assert np.isclose(k1 / k2, 0.003 / 0.0016, rtol=1e-12)


def test_cable_orientation_override_sticks_like_the_reference():
    """A node listed in the .angle file replaces the direction and length of
    the cable that starts there; in the reference the flag is never reset, so
    every later cable takes the last override (sticky) -- the non-sticky
    option applies it to its own cable only."""
    xyz, bars = _cable(4, 0.1)
    orient = {1: (1.0, 0.0, 0.0, 0.2)}          # bar 1 starts at node 1: length 0.2
    Ks = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=O.Cables(bars, orient=orient, sticky=True, n=len(xyz)),
               Cm=1.0, dt=0.1).scipy("K").toarray()
    Kn = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=O.Cables(bars, orient=orient, sticky=False, n=len(xyz)),
               Cm=1.0, dt=0.1).scipy("K").toarray()
    Kp = O.Csr(xyz, np.zeros((0, 4), np.int32), cables=O.Cables(bars), Cm=1.0, dt=0.1).scipy("K").toarray()
    assert np.isclose(Kp[0, 1], Ks[0, 1]) and np.isclose(Kp[0, 1], Kn[0, 1])     # bar 0: before the override
    assert np.isclose(Ks[1, 2], Kp[1, 2] / 2) and np.isclose(Kn[1, 2], Kp[1, 2] / 2)   # bar 1: length 0.2
    assert np.isclose(Ks[3, 4], Kp[3, 4] / 2)                                    # bar 3: sticky
    assert np.isclose(Kn[3, 4], Kp[3, 4])                                        # bar 3: its own geometry


def _cable_slab(k=10, h=0.05):
    m = M.slab(9, 7, 4, 0.8, 0.6, 0.3)
    n0 = m.n
    extra = m.xyz[[0]] + np.stack([np.zeros(k), np.zeros(k), -h * np.arange(1, k + 1)], 1)
    xyz = np.vstack([m.xyz, extra])
    bars = np.array([[0, n0]] + [[n0 + j, n0 + j + 1] for j in range(k - 1)])
    is_purk = np.zeros(len(xyz), np.uint8)
    is_purk[n0:] = 1
    return m, xyz, bars, is_purk


def test_mixed_populations_without_purkinje_nodes_equal_the_tissue_alone(small_slab):
    m = small_slab
    D = M.sigma_to_D(1.2, 0.2)
    c = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, 0.02)
    a_cells = O.Cells(O.TUSSCHER, m.n, tt_jac_true=1)
    b_cells = O.Cells(O.TUSSCHER, m.n, tt_jac_true=1)
    mix = O.MixedCells(b_cells, O.Cells(O.PURKINJE, 0), np.zeros(m.n, np.uint8))
    sa = O.Sim(c, a_cells, 0.02, 0.02, jacobi_steps=1)
    sb = O.Sim(c, mix, 0.02, 0.02, jacobi_steps=1)
    blk = M.corner_block(m, 3, 3)
    for s in (sa, sb):
        s.V[:] = -85.423
    for step in range(150):
        for s in (sa, sb):
            s.istim[:] = 0.0
            if step < 50:
                s.istim[blk] = 50.0 * 2000.0
            s.step(1)
    assert np.max(sa.V) > 0.0
    assert np.array_equal(sa.V, sb.V)


def test_mixed_restatement_equals_the_reference_objects():
    """Tissue (TT) plus a Purkinje cable whose far end is stimulated: the
    split step with the restated populations follows the one with the
    reference's own cell objects in both populations."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    m, xyz, bars, is_purk = _cable_slab()
    n0, n = m.n, len(xyz)
    D = M.sigma_to_D(1.2, 0.2)
    dt = 0.01                                    # the reference TT Newton layout needs dt <= 0.01
    c = O.Csr(xyz, m.tets, m.fibers, D, 1.0, dt, cables=O.Cables(bars, radius=0.0275))
    sims = []
    for ref in (False, True):
        tis = O.RefCells(O.TUSSCHER, n0) if ref else O.Cells(O.TUSSCHER, n0)
        pk = O.RefCells(O.PURKINJE, n - n0) if ref else O.Cells(O.PURKINJE, n - n0)
        mix = O.MixedCells(tis, pk, is_purk)
        s = O.Sim(c, mix, dt, dt, jacobi_steps=1, cg_tol=1e-12)
        s.V[:n0] = -85.423
        s.V[n0:] = -88.34
        sims.append((s, mix))
    for step in range(400):
        for s, _ in sims:
            s.istim[:] = 0.0
            if step < 200:
                s.istim[n - 3:] = 2 * 50.0 * 2500.0
            s.step(1)
    Va, Vb = sims[0][0].V, sims[1][0].V
    assert np.max(Va[n0:]) > 0.0                # the cable fired
    assert np.max(np.abs(Va - Vb)) < 1e-6 * np.max(np.abs(Vb))


def test_purkinje_cable_drives_the_tissue():
    """The stimulated far end of a 10-element cable (0.5 cm, r = 0.0275 cm)
    sends a wave down the Purkinje cells (~1 m/s) into the tissue at the
    junction node, which then activates part of the slab."""
    m, xyz, bars, is_purk = _cable_slab()
    n0, n = m.n, len(xyz)
    c = O.Csr(xyz, m.tets, m.fibers, M.sigma_to_D(1.2, 0.2), 1.0, 0.02, cables=O.Cables(bars, radius=0.0275))
    mix = O.MixedCells(O.Cells(O.TUSSCHER, n0, tt_jac_true=1), O.Cells(O.PURKINJE, n - n0), is_purk)
    s = O.Sim(c, mix, 0.02, 0.02, jacobi_steps=1, cg_tol=1e-10)
    s.V[:n0] = -85.423
    s.V[n0:] = -88.34
    tact = np.full(n, -1.0)
    for step in range(700):
        s.istim[:] = 0.0
        if step < 100:
            s.istim[n - 3:] = 2 * 50.0 * 2500.0
        s.step(1)
        new = (tact < 0) & (s.V > -40.0)
        tact[new] = (step + 1) * 0.02
    cable = tact[n0:]
    assert np.all(cable > 0) and np.all(np.diff(cable[:8]) < 0)     # activation travels toward the junction
    speed = 7 * 0.05 / (cable[0] - cable[7])                           # cm/ms
    assert 0.05 < speed < 0.5
    assert tact[0] > cable[0] and np.sum(tact[:n0] > 0) > 5


def test_tissue_restatement_matches_the_reference_cells_golden():
    """A 13x11x5 slab for 10 ms under the split step: the restated TT cells
    reproduce the V fields made with the reference's own TT objects
    (tests/golden/tissue_tt_slab.npz) at t = 2, 5 and 10 ms."""
    g = np.load(os.path.join(GOLD, "tissue_tt_slab.npz"))
    L = g["L"]
    m = M.slab(int(g["nx"]), int(g["ny"]), int(g["nz"]), float(L[0]), float(L[1]), float(L[2]))
    dt = float(g["dt"])
    c = O.Csr(m.xyz, m.tets, m.fibers, M.sigma_to_D(1.2, 0.2), 1.0, dt)
    s = O.Sim(c, O.Cells(O.TUSSCHER, m.n), dt, dt, cg_tol=1e-12, cg_maxit=2000, jacobi_steps=1)
    s.V[:] = -85.423
    blk = g["stim_nodes"]
    out = []
    for k in range(int(round(g["t"][-1] / dt))):
        s.istim[:] = 0.0
        if k * dt < 1.0:
            s.istim[blk] = 50.0 * 2000.0
        s.step(1)
        if np.any(np.abs((k + 1) * dt - g["t"]) < 1e-9):
            out.append(s.V.copy())
    out = np.array(out)
    assert np.max(g["V"]) > 0.0
    assert np.max(np.abs(out - g["V"])) < 1e-6 * np.max(np.abs(g["V"]))
