"""The voomEP EP driver on the GPU path: reads an EPSimulator input file
(voomEP/src/Applications/CardiacEP/EPSimulator.cc:143-264), the mesh files
of its MODEL, and runs the time loop of EPSimulator.cc:483-596 through the C
ABI, writing the reference's Voltage_time_* and InterVariables_time_* files.

    python -m ucla_cmg_b200.driver input.txt [--precision fp64|fp32|surrogate]
                                             [--rest-voltage] [--device N]

Same as the reference:

* input syntax: whitespace-separated ``KEY value...`` lines, keys case
  insensitive, and any line holding ``#``, ``$`` or ``*`` anywhere is skipped
  (boost ``find_first`` in a boolean context, EPSimulator.cc:144-145);
  defaults of EPSimulator.cc:80-113 (dt = IONICDT = 0.1 ms, 300 ms, output
  every 1 ms, D = (1e-3, 5e-4, 2.5e-4), MAHAJAN);
* the stimulus schedule: the reference's two pointers over the STIMULUS list
  (a stimulus starts when the step count equals ``long(t_start/dt)`` of the
  start pointer's entry, stops likewise; entries out of order never fire) and
  the four region types of CardiacBody::setStimulusCurrent
  (CardiacBody.cc:243-324): NODAL (1-based node-set file), CIRC (|x - c| <= r;
  every other non-Purkinje node is switched off), ZONAL (coordinate <= limit
  along X/Y/Z), PLANE ((x - c) . n < 0; every other non-Purkinje node is
  switched off).  The resulting per-node on/off windows are handed to the
  device once (ep_set_stimulus);
* initial voltage from the cell models (CardiacBody::getInitialVoltage:
  State[0] for Mahajan, 0 mV for ten Tusscher and Luo-Rudy, hazard H1);
  ``--rest-voltage`` starts every model from its resting State[0] instead;
* INITIALSTATES: the ``CELL`` block's values become every node's state;
* ten Tusscher's Newton uses the true Jacobian by default: the reference's
  transposed one (Tusscher.cc:173,181) diverges at dt >= 0.02 ms, with the
  reference's own objects; ``--tt-reference-jacobian`` selects it;
* CN solver with CG tolerance 1e-7 and 1000 iterations (EP_CrankNicholson.cc:
  104, 150); SMOOTHING alpha; output at t = 0 (unless READRESTART) and every
  ``int(FREQUENCY/DT)`` steps; restart files every ``long(WRITERESTART/DT)``
  steps; simulated time accumulated as ``simtime += dt``.

A MIX3D mesh with 2-node cables runs as a mixed tissue (ep_create_mixed):
the cables join the tets in the operators, the .purk nodes carry the
Purkinje cell and the other nodes the tissue model, the PURKINJE block of
INITIALSTATES goes to the Purkinje nodes, and restart files keep each node's
own nVar.  The Purkinje keys (TWODRADIUS, PURKINJEDIFFUSION,
LVPURKINJEDIFFUSION, with the reference's defaults 0.0275 cm and 0.0032
cm^2/ms, EPSimulator.cc:89, 102-103) are read with the cables' LV flags and
.angle overrides (``voomep_io.read_cables``, which resolves the overrides
over the whole .ele order as MixedMesh3D::Compute does); as in the
reference, the LV cables get PURKINJEDIFFUSION, not LVPURKINJEDIFFUSION
(``setPurkinjeDiffusionInLV(Dp)``, EPSimulator.cc:420-421).

Not on this path (accepted and ignored, with a note): the mechanics keys,
QUADORDER other than 2, CONSISTENCYCHECK.

The ZONAL stop of the reference falls through into the PLANE stop (a missing
``break``, EPSimulator.cc:557-563), which calls the plane overload of
setStimulusCurrent with its default current 0 (CardiacBody.cc:265-287): every
non-Purkinje node is switched off, whatever the plane.  That is reproduced by
default (``zonal_fallthrough=True``); ``--no-zonal-fallthrough`` switches off
only the ZONAL region, as the ``break`` would.
"""
import argparse
import os

import numpy as np

from . import capi
from .simulation import Monodomain
from .voomep_io import read_mesh

CELL_MODELS = {"LUORUDY": capi.LUORUDY, "LUORUDYWITHGATE": capi.LUORUDYWITHGATE,
               "TUSSCHER": capi.TUSSCHER, "MAHAJAN": capi.MAHAJAN, "MAHAJAN_FAIL": capi.MAHAJAN_FAIL}
STIM_TYPES = {"NODAL": 0, "CIRC": 1, "ZONAL": 2, "PLANE": 3}


def parse_input(path):
    """Settings of an EPSimulator input file (reference defaults filled in)."""
    cfg = dict(model=None, output_dir="Output/", cell_model="MAHAJAN", mesh_type="MIX3D", quad_order=2,
               ionic_dt=0.1, dt=0.1, read_restart=None, write_restart=99999.0, simulation_time=300.0,
               frequency=1.0, D=[0.001, 0.0005, 0.00025], smoothing=None, initial_states=None,
               stimuli=[], ignored=[], radius=0.0275, Dp=[0.0032] * 3, DpLeft=[0.0032] * 3)
    base = os.path.dirname(os.path.abspath(path))
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or "#" in line or "$" in line or "*" in line:
                continue
            s = line.split()
            key = s[0].upper()
            if key == "MODEL":
                cfg["model"] = s[1]
            elif key == "OUTPUTDIR":
                cfg["output_dir"] = s[1]
            elif key == "CELLMODEL":
                cfg["cell_model"] = s[1]
            elif key == "MESHTYPE":
                cfg["mesh_type"] = s[1]
            elif key == "QUADORDER":
                cfg["quad_order"] = int(s[1])
            elif key == "IONICDT":
                cfg["ionic_dt"] = float(s[1])
            elif key == "DT":
                cfg["dt"] = float(s[1])
            elif key == "READRESTART":
                cfg["read_restart"] = float(s[1])
            elif key == "WRITERESTART":
                cfg["write_restart"] = float(s[1])
            elif key == "SIMULATIONTIME":
                cfg["simulation_time"] = float(s[1])
            elif key == "FREQUENCY":
                cfg["frequency"] = float(s[1])
            elif key == "TISSUEDIFFUSION":
                cfg["D"] = [float(v) for v in s[1:4]]
            elif key == "TWODRADIUS":
                cfg["radius"] = float(s[1])
            elif key == "PURKINJEDIFFUSION":
                cfg["Dp"] = [float(v) for v in s[1:4]]
            elif key == "LVPURKINJEDIFFUSION":
                cfg["DpLeft"] = [float(v) for v in s[1:4]]
            elif key == "SMOOTHING":
                cfg["smoothing"] = float(s[1]) if len(s) == 2 else 0.1
            elif key == "INITIALSTATES":
                cfg["initial_states"] = s[1]
            elif key == "STIMULUS":
                cfg["stimuli"].append(_parse_stimulus(s))
            else:
                cfg["ignored"].append(key)
    cfg["input_dir"] = base
    return cfg


def _parse_stimulus(s):
    kind = s[1].upper()
    if kind not in STIM_TYPES:
        raise ValueError(f"unknown stimulus type {s[1]}")
    st = dict(type=STIM_TYPES[kind], i_stim=50000.0)
    if kind == "NODAL":
        st.update(node_file=s[2], t_start=float(s[3]), t_stop=float(s[4]))
        if len(s) == 6:
            st["i_stim"] = float(s[5])
    elif kind == "CIRC":
        st.update(center=[float(v) for v in s[2:5]], radius=float(s[5]), t_start=float(s[6]),
                  t_stop=float(s[7]))
        if len(s) == 9:
            st["i_stim"] = float(s[8])
    elif kind == "ZONAL":
        st.update(axis={"X": 0, "Y": 1, "Z": 2}.get(s[2].upper(), 0), limit=float(s[3]),
                  t_start=float(s[4]), t_stop=float(s[5]))
        if len(s) == 7:
            st["i_stim"] = float(s[6])
    else:
        st.update(center=[float(v) for v in s[2:5]], normal=[float(v) for v in s[5:8]],
                  t_start=float(s[8]), t_stop=float(s[9]))
        if len(s) == 11:
            st["i_stim"] = float(s[10])
    return st


def stimulus_events(stimuli, dt, nsteps):
    """The reference's two-pointer schedule (EPSimulator.cc:472-570): a list
    of (step, stimulus index, on) in firing order."""
    ev = []
    if not stimuli:
        return ev
    start_ctr = stop_ctr = 0
    pulse_start = int(stimuli[0]["t_start"] / dt)
    pulse_stop = int(stimuli[0]["t_stop"] / dt)
    for count in range(nsteps):
        if count == pulse_start:
            ev.append((count, start_ctr, True))
            start_ctr = min(start_ctr + 1, len(stimuli) - 1)
            pulse_start = int(stimuli[start_ctr]["t_start"] / dt)
        if count == pulse_stop:
            ev.append((count, stop_ctr, False))
            stop_ctr = min(stop_ctr + 1, len(stimuli) - 1)
            pulse_stop = int(stimuli[stop_ctr]["t_stop"] / dt)
    return ev


def apply_region(istim, st, on, xyz, purkinje, base_dir, zonal_fallthrough=True):
    """CardiacBody::setStimulusCurrent for one stimulus (CardiacBody.cc:
    243-324), in place on the per-node current array.  A ZONAL stop with
    ``zonal_fallthrough`` also runs the PLANE stop the reference falls
    through to (EPSimulator.cc:557-563): current 0 on every non-Purkinje
    node."""
    amp = st["i_stim"] if on else 0.0
    n = len(istim)
    t = st["type"]
    if t == 0:
        ids = np.loadtxt(os.path.join(base_dir, st["node_file"]), dtype=np.int64, ndmin=1) - 1
        istim[ids] = amp
        return
    not_purk = np.ones(n, bool)
    if purkinje is not None:
        not_purk[purkinje - 1] = False
    if t == 1:
        inside = np.linalg.norm(xyz - np.asarray(st["center"]), axis=1) <= st["radius"]
        istim[not_purk] = np.where(inside[not_purk], amp, 0.0)
    elif t == 2:
        istim[xyz[:, st["axis"]] <= st["limit"]] = amp
        if not on and zonal_fallthrough:
            istim[not_purk] = 0.0
    else:
        nrm = np.asarray(st["normal"], dtype=np.float64)
        nrm = nrm / np.linalg.norm(nrm)
        below = (xyz - np.asarray(st["center"])) @ nrm < 0.0
        istim[not_purk] = np.where(below[not_purk], amp, 0.0)


def stimulus_windows(stimuli, dt, nsteps, xyz, purkinje, base_dir, zonal_fallthrough=True):
    """Per-node windows (node, first step, end step, amplitude) equivalent to
    the reference's schedule over nsteps steps."""
    n = len(xyz)
    istim = np.zeros(n)
    since = np.zeros(n, dtype=np.int64)
    out_ids, out_on, out_off, out_amp = [], [], [], []
    events = stimulus_events(stimuli, dt, nsteps)
    for step, k, on in events + [(nsteps, None, None)]:
        new = istim.copy()
        if k is not None:
            apply_region(new, stimuli[k], on, xyz, purkinje, base_dir, zonal_fallthrough)
        changed = np.where(new != istim)[0]
        ended = changed[istim[changed] != 0.0]
        if k is None:
            ended = np.where(istim != 0.0)[0]
        for i in ended:
            if step > since[i]:
                out_ids.append(i); out_on.append(since[i]); out_off.append(step); out_amp.append(istim[i])
        since[changed] = step
        istim = new
    return (np.array(out_ids, dtype=np.int32), np.array(out_on, dtype=np.int64),
            np.array(out_off, dtype=np.int64), np.array(out_amp))


def read_initial_states(path):
    cell, purk, flag = [], [], ""
    with open(path) as f:
        for line in f:
            u = line.strip().upper()
            if not u:
                flag = ""
                continue
            if "PURKINJE" in u:
                flag = "PURKINJE"
                continue
            if "CELL" in u:
                flag = "CELL"
                continue
            if flag == "CELL":
                cell.append(float(u))
            elif flag == "PURKINJE":
                purk.append(float(u))
    return np.array(cell), np.array(purk)


def cable_setup(cfg, node_type):
    """The 2-node cables of the input's MIX3D mesh as the reference would
    assemble them: dict for ``simulation.assemble_operators`` (bars, fibres,
    LV flags, .angle overrides, radius, and Dp for both RV and LV cables,
    EPSimulator.cc:420-421), or None when the mesh has none."""
    from .voomep_io import read_cables
    cab = read_cables(os.path.join(cfg["input_dir"], cfg["model"]), node_type)
    if not len(cab["bars"]):
        return None
    return dict(bars=cab["bars"], bar_fibers=cab["fibers"], lv=cab["lv"], angle=cab["angle"],
                bar_angle_node=cab["angle_node"],
                radius=cfg["radius"], Dp=tuple(cfg["Dp"]), DpLeft=tuple(cfg["Dp"]), quad_order=cfg["quad_order"])


def run(input_file, precision=capi.FP64, rest_voltage=False, device=0, surrogate_path=None, verbose=True,
        tt_jacobian=capi.TT_JAC_TRUE, zonal_fallthrough=True, cg_tol=1e-7):
    cfg = parse_input(input_file)
    base_dir = cfg["input_dir"]
    model = CELL_MODELS[cfg["cell_model"].upper()]
    mesh, node_type, purk, other = read_mesh(os.path.join(base_dir, cfg["model"]))
    # a MIX3D mesh with cables: a mixed tissue, the Purkinje cell on the
    # .purk nodes (CardiacBody::New, CardiacBody.cc:982-1101)
    cab = cable_setup(cfg, node_type) if other else None
    purk0 = None
    if cab is not None or (purk is not None and other):
        purk0 = (np.asarray(purk, dtype=np.int64) - 1) if purk is not None else np.zeros(0, np.int64)
        if verbose:
            nb = 0 if cab is None else len(cab["bars"])
            print(f"** mixed tissue: {nb} Purkinje cables (radius {cfg['radius']} cm, D_p {cfg['Dp'][0]}), "
                  f"{len(purk0)} Purkinje cells")
    nstate = capi.model_nstate(model)
    init, pk_init = None, None
    if cfg["initial_states"]:
        cell, pkb = read_initial_states(os.path.join(base_dir, cfg["initial_states"]))
        if len(cell) != nstate:
            raise ValueError(f"INITIALSTATES CELL block has {len(cell)} values, the model {nstate}")
        init = np.tile(cell, (mesh.n, 1))
        if purk0 is not None and len(pkb):
            if len(pkb) != capi.model_nstate(capi.PURKINJE):
                raise ValueError(f"INITIALSTATES PURKINJE block has {len(pkb)} values, the cell 22")
            pk_init = pkb
    n_types = None
    if node_type is not None and model in (capi.MAHAJAN, capi.MAHAJAN_FAIL):
        n_types = 9
        if purk0 is not None:
            # Purkinje nodes carry types 11/12; their tissue rows are unused
            node_type = np.where(node_type > 8, 0, node_type)
    elif model not in (capi.MAHAJAN, capi.MAHAJAN_FAIL):
        node_type = None                        # one parameter set (TT, LR)
    dt = cfg["dt"]
    mixed = {} if purk0 is None else dict(cables=cab, purkinje=purk0)
    g = Monodomain(mesh, model, precision, dt=dt, ionic_dt=cfg["ionic_dt"], D=cfg["D"], cg_tol=cg_tol,
                   cg_maxit=1000, node_type=node_type, n_types=n_types, initial_states=init,
                   smoothing_alpha=cfg["smoothing"] or 0.0, tt_jacobian=tt_jacobian, device=device, **mixed)
    if precision == capi.SURROGATE:
        from .surrogate import Surrogate, DEFAULT_PATH
        Surrogate.load(surrogate_path or DEFAULT_PATH).deploy(g)
    if pk_init is not None:
        S = g.states()
        S[purk0, :len(pk_init)] = pk_init
        g.set_states(S)
    lr = model in (capi.LUORUDY, capi.LUORUDYWITHGATE)
    if rest_voltage:
        S = g.states()
        V0 = S[:, 7 if lr else 0].copy()
        if purk0 is not None:
            V0[purk0] = S[purk0, 0]             # the Purkinje cell keeps V in slot 0
        g.set_voltage(V0)
    else:
        V0 = g.model_voltage()
        if pk_init is not None:
            V0[purk0] = pk_init[0]              # Purkinje::getVoltage: State[0]
        g.set_voltage(V0)
    out = os.path.join(base_dir, cfg["output_dir"])
    os.makedirs(out, exist_ok=True)
    # the loop's step count and simulated time, accumulated as the reference does
    times = []
    simtime = 0.0
    count = 0
    if cfg["read_restart"] is not None:
        simtime = cfg["read_restart"]
        count = int(simtime / dt)
    t = simtime
    while t < cfg["simulation_time"]:
        t += dt
        times.append(t)
    nsteps = count + len(times)
    ids, on, off, amp = stimulus_windows(cfg["stimuli"], dt, nsteps, mesh.xyz, purk, base_dir, zonal_fallthrough)
    # windows as times that round back to the same step under long(t/dt)
    g.set_stimulus(ids, (on + 0.5) * dt, (off + 0.5) * dt, amp)
    if cfg["read_restart"] is not None:
        g.read_restart(simtime, out)
    else:
        g.write_output(0.0, out)
    steps_per_frame = int(cfg["frequency"] / dt)
    if steps_per_frame <= 0:
        raise ValueError("FREQUENCY below DT: no output step (the reference divides by zero here)")
    restart_every = int(cfg["write_restart"] / dt)
    k = 0
    while k < len(times):
        # advance to the next output or restart step in one call
        nxt = k
        while True:
            c = count + nxt + 1
            nxt += 1
            if nxt >= len(times) or c % steps_per_frame == 0 or (restart_every > 0 and c % restart_every == 0):
                break
        g.step(nxt - k)
        c = count + nxt
        simt = times[nxt - 1]
        if c % steps_per_frame == 0:
            g.write_output(simt, out)
        if restart_every > 0 and c % restart_every == 0:
            g.write_restart(simt, out)
        k = nxt
    g.close()
    return cfg, nsteps


def main():
    ap = argparse.ArgumentParser(description="EPSimulator input file on the GPU path")
    ap.add_argument("input")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "surrogate"])
    ap.add_argument("--rest-voltage", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--tt-reference-jacobian", action="store_true",
                    help="ten Tusscher Newton with the reference's transposed Jacobian (diverges at dt >= 0.02 ms)")
    ap.add_argument("--no-zonal-fallthrough", action="store_true",
                    help="a ZONAL stop switches off its own region only (the reference also switches "
                         "off every other non-Purkinje node, EPSimulator.cc:557-563)")
    a = ap.parse_args()
    prec = {"fp64": capi.FP64, "fp32": capi.FP32, "surrogate": capi.SURROGATE}[a.precision]
    cfg, nsteps = run(a.input, prec, a.rest_voltage, a.device,
                      tt_jacobian=capi.TT_JAC_REFERENCE if a.tt_reference_jacobian else capi.TT_JAC_TRUE,
                      zonal_fallthrough=not a.no_zonal_fallthrough)
    print(f"** {nsteps} steps done; output in {cfg['output_dir']}")


if __name__ == "__main__":
    main()
