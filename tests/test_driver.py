"""The EPSimulator-compatible driver: input parsing, the reference's
stimulus schedule and region types, and the mesh file formats (CPU)."""
import os
import numpy as np

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200 import driver as D
from ucla_cmg_b200 import voomep_io as IO


def test_parse_input(tmp_path):
    f = tmp_path / "case.input"
    f.write_text("""# comment line
MODEL  Mesh/slab
OutputDir out/
CellModel Tusscher
dt 0.02
IonicDt 0.01
SimulationTime 12.5   # any '#' in a line drops the whole line (the reference's test)
SimulationTime 10
frequency 0.5
TissueDiffusion 1e-3 2e-4 2e-4
Smoothing
Stimulus Nodal set.txt 0. 1.0
Stimulus Circ 0.1 0.2 0.0 0.05 5.0 6.0 30000
Stimulus Zonal y 0.1 7 8
Stimulus Plane 0 0 0 1 0 0 9 10 100
MechDt 999
TwoDRadius 0.03
PurkinjeDiffusion 0.004 0.004 0.004
LVPurkinjeDiffusion 0.008 0.008 0.008
""")
    c = D.parse_input(str(f))
    assert c["model"] == "Mesh/slab" and c["output_dir"] == "out/" and c["cell_model"] == "Tusscher"
    assert c["dt"] == 0.02 and c["ionic_dt"] == 0.01 and c["simulation_time"] == 10.0
    assert c["frequency"] == 0.5 and c["D"] == [1e-3, 2e-4, 2e-4] and c["smoothing"] == 0.1
    assert c["write_restart"] == 99999.0 and c["read_restart"] is None
    s = c["stimuli"]
    assert [x["type"] for x in s] == [0, 1, 2, 3]
    assert s[0]["i_stim"] == 50000.0 and s[1]["i_stim"] == 30000.0 and s[3]["i_stim"] == 100.0
    assert s[1]["radius"] == 0.05 and s[1]["center"] == [0.1, 0.2, 0.0]
    assert s[2]["axis"] == 1 and s[2]["limit"] == 0.1
    assert s[3]["normal"] == [1.0, 0.0, 0.0] and s[3]["t_start"] == 9.0
    assert "MECHDT" in c["ignored"]
    assert c["radius"] == 0.03 and c["Dp"] == [0.004] * 3 and c["DpLeft"] == [0.008] * 3
    f.write_text("MODEL m\n")
    d = D.parse_input(str(f))
    assert d["radius"] == 0.0275 and d["Dp"] == [0.0032] * 3        # EPSimulator.cc:89, 102-103


def test_stimulus_pointer_schedule():
    st = [dict(t_start=0.0, t_stop=1.0), dict(t_start=5.0, t_stop=6.0)]
    ev = D.stimulus_events(st, 0.1, 100)
    assert ev == [(0, 0, True), (10, 0, False), (50, 1, True), (60, 1, False)]
    # out of order: the second start precedes the first stop; the reference's
    # start pointer has moved past it when the count gets there, so it never fires
    st = [dict(t_start=5.0, t_stop=6.0), dict(t_start=1.0, t_stop=2.0)]
    ev = D.stimulus_events(st, 0.1, 100)
    assert (10, 1, True) not in ev and (50, 0, True) in ev


def test_stimulus_regions_and_windows():
    xyz = np.array([[0.0, 0, 0], [0.05, 0, 0], [0.2, 0, 0], [0.5, 0, 0]])
    circ = dict(type=1, center=[0.0, 0.0, 0.0], radius=0.1, i_stim=7.0, t_start=0.0, t_stop=1.0)
    zonal = dict(type=2, axis=0, limit=0.3, i_stim=3.0, t_start=2.0, t_stop=3.0)
    plane = dict(type=3, center=[0.3, 0, 0], normal=[-1.0, 0, 0], i_stim=5.0, t_start=4.0, t_stop=5.0)
    istim = np.full(4, 9.0)
    D.apply_region(istim, circ, True, xyz, None, ".")
    assert list(istim) == [7.0, 7.0, 0.0, 0.0]            # CIRC switches the others off
    D.apply_region(istim, zonal, True, xyz, None, ".")
    assert list(istim) == [3.0, 3.0, 3.0, 0.0]
    # PLANE: nodes with (x - c).n < 0, here x > 0.3; node 4 (1-based) is a
    # Purkinje node and keeps its value; every other node is switched off
    D.apply_region(istim, plane, True, xyz, np.array([4]), ".")
    assert list(istim) == [0.0, 0.0, 0.0, 0.0]
    ids, on, off, amp = D.stimulus_windows([circ, zonal, plane], 0.5, 20, xyz, None, ".")
    w = set(zip(ids.tolist(), on.tolist(), off.tolist(), amp.tolist()))
    assert w == {(0, 0, 2, 7.0), (1, 0, 2, 7.0), (0, 4, 6, 3.0), (1, 4, 6, 3.0), (2, 4, 6, 3.0),
                 (3, 8, 10, 5.0)}


def test_zonal_stop_falls_through_to_plane_stop():
    """The reference's ZONAL stop has no ``break`` and also runs the PLANE
    stop with current 0 (EPSimulator.cc:557-563, CardiacBody.cc:265-287): a
    NODAL stimulus still running elsewhere is switched off with it, Purkinje
    nodes excepted.  Default = the reference; opt-out = the ``break``."""
    xyz = np.array([[0.0, 0, 0], [0.05, 0, 0], [0.2, 0, 0], [0.5, 0, 0]])
    zonal = dict(type=2, axis=0, limit=0.1, i_stim=3.0, t_start=0.0, t_stop=1.0)
    istim = np.array([3.0, 3.0, 8.0, 8.0])                 # nodes 3, 4 (1-based) under another stimulus
    a = istim.copy()
    D.apply_region(a, zonal, False, xyz, np.array([4]), ".")
    assert list(a) == [0.0, 0.0, 0.0, 8.0]                 # node 4 is a Purkinje node
    b = istim.copy()
    D.apply_region(b, zonal, False, xyz, np.array([4]), ".", zonal_fallthrough=False)
    assert list(b) == [0.0, 0.0, 8.0, 8.0]
    # in a schedule (dt 0.5): a zonal stimulus 0.0-1.0, then a plane one
    # 0.5-5.0 over the nodes x > 0.3; the zonal stop at step 2 also ends the
    # plane window there
    zonal = dict(type=2, axis=0, limit=0.1, i_stim=3.0, t_start=0.0, t_stop=1.0)
    plane = dict(type=3, center=[0.3, 0, 0], normal=[-1.0, 0, 0], i_stim=5.0, t_start=0.5, t_stop=5.0)
    assert D.stimulus_events([zonal, plane], 0.5, 20) == [(0, 0, True), (1, 1, True), (2, 0, False),
                                                         (10, 1, False)]
    w = set(zip(*[x.tolist() for x in D.stimulus_windows([zonal, plane], 0.5, 20, xyz, None, ".")]))
    assert w == {(0, 0, 1, 3.0), (1, 0, 1, 3.0), (3, 1, 2, 5.0)}
    w = set(zip(*[x.tolist() for x in D.stimulus_windows([zonal, plane], 0.5, 20, xyz, None, ".",
                                                         zonal_fallthrough=False)]))
    assert (3, 1, 10, 5.0) in w


def test_mesh_files_round_trip(tmp_path):
    m = M.slab(5, 4, 3, 0.4, 0.3, 0.2)
    t = (np.arange(m.n) % 3).astype(np.uint8)
    base = str(tmp_path / "slab")
    IO.write_mesh(base, m, t)
    m2, t2, purk, other = IO.read_mesh(base)
    assert other == 0 and purk is None
    assert np.array_equal(m2.tets, m.tets)
    assert np.allclose(m2.xyz, m.xyz, rtol=0, atol=0)
    assert np.array_equal(m2.fibers, m.fibers)
    assert np.array_equal(t2, t)


def test_mesh_reader_skips_cables(tmp_path):
    base = str(tmp_path / "mix")
    (tmp_path / "mix.node").write_text("5 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n5 2 2 2\n")
    (tmp_path / "mix.ele").write_text("2 4 0\n1 4 1 2 3 4\n2 2 4 5\n")
    (tmp_path / "mix.purk").write_text("2\n4 5\n")
    m, t, purk, other = IO.read_mesh(base)
    assert m.m == 1 and other == 1 and list(purk) == [4, 5]


def test_mixed_mesh_cables_read_and_assembled(tmp_path):
    """A MIX3D mesh (tets + 2-node cables, .cell with LV Purkinje type 11,
    .fibers for every element, .angle override): the cable reader feeds the
    library's host assembly, which equals the oracle's on the same data."""
    from oracle import oracle as O
    from ucla_cmg_b200 import simulation as S
    m = M.slab(5, 4, 3, 0.4, 0.3, 0.2)
    n0 = m.n
    extra = m.xyz[[0]] + np.array([[0.0, 0.0, -0.05], [0.0, 0.0, -0.1]])
    xyz = np.vstack([m.xyz, extra])
    bars = np.array([[0, n0], [n0, n0 + 1], [1, 0]])
    base = str(tmp_path / "mix")
    with open(base + ".node", "w") as f:
        f.write(f"{len(xyz)} 3 0 0\n")
        for i, p in enumerate(xyz):
            f.write(f"{i + 1} {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
    # elements interleaved as a MIX3D .ele may hold them
    rng = np.random.default_rng(0)
    bfib = np.array([np.linalg.qr(rng.normal(size=(3, 3)))[0].T.reshape(-1) for _ in bars])
    elems, fibs = [], []
    for e, tet in enumerate(m.tets):
        elems.append([4] + list(tet + 1)); fibs.append(m.fibers[e])
        if e < len(bars):
            elems.append([2] + list(bars[e] + 1)); fibs.append(bfib[e])
    with open(base + ".ele", "w") as f:
        f.write(f"{len(elems)} 0 0\n")
        for e, el in enumerate(elems):
            f.write(" ".join(str(v) for v in [e + 1] + el) + "\n")
    np.savetxt(base + ".fibers", np.array(fibs))
    cell = np.zeros(len(xyz), np.uint8); cell[[n0 + 1]] = 11
    with open(base + ".cell", "w") as f:
        for i in range(len(xyz)):
            f.write(f"{i + 1} {cell[i]}\n")
    with open(base + ".angle", "w") as f:
        f.write(f"{n0 + 1} 0 0 -1 0.06\n")
    mesh, t, purk, other = IO.read_mesh(base)
    cab = IO.read_cables(base, t)
    # the driver's view: LV cables take PURKINJEDIFFUSION as in the reference
    cfg = {"input_dir": str(tmp_path), "model": "mix", "radius": 0.0275, "Dp": [0.002] * 3,
           "DpLeft": [0.009] * 3, "quad_order": 2}
    setup = D.cable_setup(cfg, t)
    assert np.array_equal(setup["bars"], bars) and setup["DpLeft"] == setup["Dp"] == (0.002,) * 3
    assert other == len(bars) and np.array_equal(cab["bars"], bars)
    assert np.allclose(cab["fibers"], bfib) and list(cab["lv"]) == [0, 1, 0]
    assert cab["angle"] == {n0: (0.0, 0.0, -1.0, 0.06)}
    kw = dict(Dp=(0.0016, 0.0008, 0.0004), DpLeft=(0.003, 0.001, 0.0005), radius=0.0275)
    Dt = M.sigma_to_D(1.2, 0.2)
    A, B, CL = S.assemble_operators(mesh, Dt, 0.1, bars=cab["bars"], bar_fibers=cab["fibers"], lv=cab["lv"],
                                    angle=cab["angle"], **kw)
    o = O.Csr(mesh.xyz, mesh.tets, mesh.fibers, Dt, 1.0, 0.1,
              cables=O.Cables(cab["bars"], fibers=cab["fibers"], lv=cab["lv"], orient=cab["angle"], n=mesh.n, **kw))
    assert abs(A - o.scipy("A")).max() <= 1e-15 * abs(A).max()
    assert np.allclose(CL, o.arr("CL"), rtol=1e-15, atol=0)


def test_schedule_matches_oracle_restatement():
    """The driver's two-pointer schedule against the oracle's C restatement
    of the same EPSimulator logic, on sorted and unsorted lists."""
    from oracle import oracle as O
    rng = np.random.default_rng(1)
    for trial in range(20):
        k = int(rng.integers(1, 6))
        t0 = np.round(rng.uniform(0, 20, k), 2)
        if trial % 2 == 0:
            t0 = np.sort(t0)
        t1 = t0 + np.round(rng.uniform(0.5, 3, k), 2)
        st = [dict(t_start=a, t_stop=b) for a, b in zip(t0, t1)]
        ev = D.stimulus_events(st, 0.1, 300)
        on, off = O.stim_schedule(t0, t1, 0.1, 300)
        assert sorted((s, i) for s, i, f in ev if f) == sorted((int(s), i) for i, s in enumerate(on) if s >= 0)
        assert sorted((s, i) for s, i, f in ev if not f) == sorted((int(s), i) for i, s in enumerate(off) if s >= 0)


def test_output_files_round_trip(tmp_path):
    """The reference's output formats: V as raw FP64, InterVariables as per
    node (int nVar, nVar doubles) -- nVar may differ between nodes (tissue
    model and Purkinje cells of a mixed tissue); truncation is an error."""
    rng = np.random.default_rng(2)
    assert IO.output_name(str(tmp_path), "Voltage", 12.5).endswith("Voltage_time_00012.50.00")
    V = rng.normal(size=17)
    V.tofile(IO.output_name(str(tmp_path), "Voltage", 1.0))
    assert np.array_equal(IO.read_voltage(IO.output_name(str(tmp_path), "Voltage", 1.0)), V)
    uni = rng.normal(size=(5, 19))
    p = IO.output_name(str(tmp_path), "InterVariables", 1.0)
    IO.write_intervariables(p, uni)
    assert np.array_equal(IO.read_intervariables(p), uni)
    mixed = [rng.normal(size=19), rng.normal(size=22), rng.normal(size=19)]
    IO.write_intervariables(p, mixed)
    got = IO.read_intervariables(p)
    assert [len(v) for v in got] == [19, 22, 19] and all(np.array_equal(a, b) for a, b in zip(got, mixed))
    with open(p, "r+b") as f:
        f.truncate(4 + 8 * 19 + 4 + 8 * 10)
    import pytest
    with pytest.raises(ValueError):
        IO.read_intervariables(p)


def _mix_case(tmp_path, cell_model="Tusscher"):
    """A slab with a 6-element Purkinje cable hanging from node 1, .purk
    listing the cable nodes, a nodal stimulus at the cable's far end."""
    m = M.slab(5, 4, 3, 0.4, 0.3, 0.2)
    n0, k, h = m.n, 6, 0.05
    extra = m.xyz[[0]] + np.stack([np.zeros(k), np.zeros(k), -h * np.arange(1, k + 1)], 1)
    xyz = np.vstack([m.xyz, extra])
    bars = [[0, n0]] + [[n0 + j, n0 + j + 1] for j in range(k - 1)]
    base = tmp_path / "mix"
    with open(str(base) + ".node", "w") as f:
        f.write(f"{len(xyz)} 3 0 0\n")
        for i, p in enumerate(xyz):
            f.write(f"{i + 1} {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
    elems = [[4] + list(t + 1) for t in m.tets] + [[2, a + 1, b + 1] for a, b in bars]
    with open(str(base) + ".ele", "w") as f:
        f.write(f"{len(elems)} 0 0\n")
        for e, el in enumerate(elems):
            f.write(" ".join(str(v) for v in [e + 1] + el) + "\n")
    (tmp_path / "mix.purk").write_text(f"{k}\n" + " ".join(str(n0 + j + 1) for j in range(k)) + "\n")
    (tmp_path / "stim.txt").write_text(f"{n0 + k}\n{n0 + k - 1}\n")
    (tmp_path / "case.input").write_text(f"""MODEL mix
OutputDir out/
CellModel {cell_model}
DT 0.01
IonicDT 0.01
SimulationTime 6
Frequency 1
WriteRestart 3
TissueDiffusion 1e-3 2e-4 2e-4
Stimulus Nodal stim.txt 0 2 250000
""")
    return str(tmp_path / "case.input"), n0, k


def test_oracle_driver_runs_a_mixed_case(tmp_path):
    """The oracle's EPSimulator loop on a MIX3D case: output frames at t = 0
    and every ms, restart files at 3 and 6 ms with 19 states on tissue nodes
    and 22 on Purkinje nodes, the cable fires from its stimulated end; the
    reference's own cell objects and the restatement give the same fields."""
    from oracle import oracle as O
    if O.ref_lib() is None:
        import pytest
        pytest.skip("oracle/_ref not built")
    from oracle import driver_oracle as DO
    inp, n0, k = _mix_case(tmp_path)
    out_ref, out_port = str(tmp_path / "ref"), str(tmp_path / "port")
    cfg, nsteps, is_purk = DO.run(inp, out_ref, reference_cells=True, rest_voltage=True)
    DO.run(inp, out_port, reference_cells=False, rest_voltage=True)
    assert nsteps == 601 and int(is_purk.sum()) == k             # simtime += dt accumulates one more step
    frames = [IO.read_voltage(IO.output_name(out_ref, "Voltage", t)) for t in (0.0, 1.0, 2.0, 3.0)]
    assert all(len(f) == n0 + k for f in frames)
    assert max(f[n0:].max() for f in frames) > 0.0               # the cable fired
    st = IO.read_intervariables(IO.output_name(out_ref, "InterVariables", 3.0))
    assert [len(v) for v in st[:n0]] == [19] * n0 and [len(v) for v in st[n0:]] == [22] * k
    for t in (1.0, 2.0, 3.0):
        a = IO.read_voltage(IO.output_name(out_ref, "Voltage", t))
        b = IO.read_voltage(IO.output_name(out_port, "Voltage", t))
        assert np.max(np.abs(a - b)) < 1e-6 * np.max(np.abs(a))


def test_oracle_driver_read_restart(tmp_path):
    """READRESTART in the oracle's loop: V and the per-node states (19 and
    22 values) come from the restart files, the loop starts at simtime = t,
    count = long(t/dt), and the frames after it equal those of the run that
    never stopped."""
    import shutil
    from oracle import driver_oracle as DO
    inp, n0, k = _mix_case(tmp_path)
    full, cont = str(tmp_path / "full"), str(tmp_path / "cont")
    DO.run(inp, full, reference_cells=False, rest_voltage=True)
    os.makedirs(cont)
    for kind in ("Voltage", "InterVariables"):
        shutil.copy(IO.output_name(full, kind, 3.0), IO.output_name(cont, kind, 3.0))
    txt = open(inp).read() + "ReadRestart 3\n"
    inp2 = str(tmp_path / "restart.input")
    open(inp2, "w").write(txt)
    cfg, nsteps, _ = DO.run(inp2, cont, reference_cells=False, rest_voltage=True)
    assert cfg["read_restart"] == 3.0 and nsteps == 601
    assert not os.path.exists(IO.output_name(cont, "Voltage", 0.0))
    for t in (4.0, 5.0, 6.0):
        a = IO.read_voltage(IO.output_name(full, "Voltage", t))
        b = IO.read_voltage(IO.output_name(cont, "Voltage", t))
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
