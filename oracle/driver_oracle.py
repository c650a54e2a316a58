"""EPSimulator's time loop on the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Runs an EPSimulator input file with the oracle's split step (the C
restatement of EP_CrankNicholson over the FEM operators) and the
reference's own cell objects (or their restatement), using the same input
parser, stimulus schedule and mesh readers as the library's driver.  MIX3D
meshes get their 2-node Purkinje cables in the operators and the Purkinje
cell on the .purk nodes, the tissue model elsewhere (CardiacBody::New,
voomEP/src/Body/CardiacBody.cc:982-1101): the reference's behaviour for
mixed tissues, which the GPU path is to be checked against.  Writes
Voltage_time_* and InterVariables_time_* as EPSolver does
(voomEP/src/Solvers/EPSolver.cc:116-211; outputs at t = 0 and every
int(FREQUENCY/DT) steps, restart files every long(WRITERESTART/DT) steps,
time accumulated as simtime += dt, EPSimulator.cc:572-596).
"""
import os

import numpy as np

from . import oracle as O
from ucla_cmg_b200 import driver as D
from ucla_cmg_b200 import voomep_io as IO

MODELS = {"LUORUDY": O.LUORUDY, "LUORUDYWITHGATE": O.LUORUDYWITHGATE, "TUSSCHER": O.TUSSCHER,
          "MAHAJAN": O.MAHAJAN, "MAHAJAN_FAIL": O.MAHAJAN_FAIL}


def _istim_at(k, n, ids, on, off, amp):
    """Per-node current at step k from the stimulus windows: the window that
    started last among those covering k (as the device does)."""
    ist = np.zeros(n)
    best = np.full(n, -1, dtype=np.int64)
    live = (on <= k) & (k < off)
    for i, o, a in zip(ids[live], on[live], amp[live]):
        if o > best[i]:
            best[i] = o
            ist[i] = a
    return ist


def run(input_file, out_dir=None, reference_cells=True, rest_voltage=False, cg_tol=1e-7, jacobi_steps=3):
    """Run the case; returns (cfg, number of steps, is_purk)."""
    cfg = D.parse_input(input_file)
    base = cfg["input_dir"]
    model = MODELS[cfg["cell_model"].upper()]
    mesh, node_type, purk, other = IO.read_mesh(os.path.join(base, cfg["model"]))
    n = mesh.n
    cab = D.cable_setup(cfg, node_type) if other else None
    is_purk = np.zeros(n, np.uint8)
    if purk is not None and cab is not None:
        is_purk[purk - 1] = 1
    dt = cfg["dt"]
    cables = None
    if cab is not None:
        cables = O.Cables(cab["bars"], Dp=cab["Dp"], DpLeft=cab["DpLeft"], radius=cab["radius"],
                          fibers=cab["bar_fibers"], lv=cab["lv"], quad_order=cab["quad_order"],
                          orient=cab["angle"] or None, n=n,
                          bar_orient_node=cab["bar_angle_node"] if cab["angle"] else None)
    csr = O.Csr(mesh.xyz, mesh.tets, mesh.fibers, cfg["D"], 1.0, dt, smoothing_alpha=cfg["smoothing"] or 0.0,
                cables=cables)
    tis_nodes = np.where(is_purk == 0)[0]
    pk_nodes = np.where(is_purk == 1)[0]
    types = None
    if node_type is not None and model in (O.MAHAJAN, O.MAHAJAN_FAIL):
        types = np.ascontiguousarray(node_type[tis_nodes])
    if reference_cells:
        tissue = O.RefCells(model, len(tis_nodes), types)
        pk = O.RefCells(O.PURKINJE, len(pk_nodes)) if len(pk_nodes) else None
    else:
        tissue = O.Cells(model, len(tis_nodes), types=types)
        pk = O.Cells(O.PURKINJE, len(pk_nodes)) if len(pk_nodes) else None
    cells = O.MixedCells(tissue, pk, is_purk) if pk is not None else tissue
    sim = O.Sim(csr, cells, dt, cfg["ionic_dt"], cg_tol=cg_tol, cg_maxit=1000, jacobi_steps=jacobi_steps)
    # InitializeVoltage with IonicModel::getVoltage (EPSimulator.cc:463): 0 for
    # TT and LR (hazard H1), State[0] for Mahajan and the Purkinje cell
    V = sim.V
    st = tissue.state
    if rest_voltage or model in (O.MAHAJAN, O.MAHAJAN_FAIL):
        V[tis_nodes] = st[:, 7] if model in (O.LUORUDY, O.LUORUDYWITHGATE) else st[:, 0]
    else:
        V[tis_nodes] = 0.0
    if pk is not None:
        V[pk_nodes] = pk.state[:, 0]
    out = out_dir or os.path.join(base, cfg["output_dir"])
    os.makedirs(out, exist_ok=True)
    # READRESTART: V and the cell states from the restart files, the loop
    # starting at simtime = t, count = long(t/dt) (EPSimulator.cc:495-500,
    # EPSolver::readRestart, EPSolver.cc:179-211)
    simtime, count = 0.0, 0
    if cfg["read_restart"] is not None:
        simtime = cfg["read_restart"]
        count = int(simtime / dt)
        V[:] = IO.read_voltage(IO.output_name(out, "Voltage", simtime))
        rows = IO.read_intervariables(IO.output_name(out, "InterVariables", simtime))
        if len(rows) != n:
            raise ValueError(f"restart file has {len(rows)} nodes, the mesh {n}")
        _set_states(tissue, [rows[i] for i in tis_nodes])
        if pk is not None:
            _set_states(pk, [rows[i] for i in pk_nodes])
    times, t = [], simtime
    while t < cfg["simulation_time"]:
        t += dt
        times.append(t)
    nsteps = count + len(times)
    ids, on, off, amp = D.stimulus_windows(cfg["stimuli"], dt, nsteps, mesh.xyz, purk, base)
    steps_per_frame = int(cfg["frequency"] / dt)
    restart_every = int(cfg["write_restart"] / dt)

    def write_states(tt):
        rows = [None] * n
        for k, i in enumerate(tis_nodes):
            rows[i] = tissue.state[k]
        if pk is not None:
            for k, i in enumerate(pk_nodes):
                rows[i] = pk.state[k]
        IO.write_intervariables(IO.output_name(out, "InterVariables", tt), rows)

    if cfg["read_restart"] is None:
        np.asarray(sim.V, dtype=np.float64).tofile(IO.output_name(out, "Voltage", 0.0))
    for k in range(count, nsteps):
        sim.istim[:] = _istim_at(k, n, ids, on, off, amp)
        sim.step(1)
        c = k + 1
        tk = times[k - count]
        if c % steps_per_frame == 0:
            np.asarray(sim.V, dtype=np.float64).tofile(IO.output_name(out, "Voltage", tk))
        if restart_every > 0 and c % restart_every == 0:
            write_states(tk)
    return cfg, nsteps, is_purk


def _set_states(cells, rows):
    """Per-node state rows into a population (restatement or reference objects)."""
    a = np.array(rows, dtype=np.float64).reshape(len(rows), -1)
    if a.shape[1] != cells.nstate:
        raise ValueError(f"restart rows have {a.shape[1]} values, the cell model {cells.nstate}")
    if isinstance(cells, O.RefCells):
        cells.state = a
    else:
        cells.state[:] = a
