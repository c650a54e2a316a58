"""Host-side mirror of the reference's EP solver interface over the C ABI.

Reference interface (paths inside wsklug/UCLA_CMG, voomEP/src/...):

* ``CardiacBody`` (Body/CardiacBody.h) -- cell model per node, diffusion
  tensor, stimulus currents;
* ``EPSolver`` / ``EP_CrankNicholson`` (Solvers/EPSolver.h,
  EP_CrankNicholson.cc) -- ``InitializeVoltage``, ``setIonicTimeStep``,
  ``setSolveTime``, ``Solve``, ``WriteOutput``, ``writeRestart``,
  ``readRestart``;
* ``EPSimulator`` main loop (Applications/CardiacEP/EPSimulator.cc:483-596).

:class:`Monodomain` owns one device-resident tissue instance
(``ep_create``); the method names of the reference are kept as aliases.  The
steps that ``setIonicTimeStep`` and ``setSolveTime`` set are constructor
arguments here (``ionic_dt``, ``dt``): the CN operators are assembled for
them once.
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import check, ptr


def _instance_descs(mesh, model, D, Cm, node_type, type_consts, n_types, gks_scale, user_xi,
                    newton_cap, tt_jacobian, mh_abs_mode, initial_states):
    """MeshDesc and ModelDesc of one instance, and the arrays they point to."""
    keep = {}
    keep["xyz"] = np.ascontiguousarray(mesh.xyz, dtype=np.float64)
    keep["tets"] = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    keep["fib"] = None if mesh.fibers is None else np.ascontiguousarray(mesh.fibers, dtype=np.float64)
    md = capi.MeshDesc()
    md.n_nodes = mesh.n
    md.xyz = ptr(keep["xyz"])
    md.n_tets = mesh.m
    md.tets = ptr(keep["tets"], C.POINTER(C.c_int32))
    md.one_based = 0
    md.fibers = ptr(keep["fib"])
    for k in range(3):
        md.D[k] = float(D[k])
    md.Cm = float(Cm)
    mo = capi.ModelDesc()
    mo.model = model
    keep["types"] = None if node_type is None else np.ascontiguousarray(node_type, dtype=np.uint8)
    keep["tc"] = None if type_consts is None else np.ascontiguousarray(type_consts, dtype=np.float64)
    if n_types is None:
        if keep["tc"] is not None:
            n_types = keep["tc"].shape[0]
        elif keep["types"] is not None and len(keep["types"]):
            n_types = int(keep["types"].max()) + 1
        else:
            n_types = 1
    mo.n_types = int(n_types)
    mo.type_consts = ptr(keep["tc"])
    mo.node_type = ptr(keep["types"], C.POINTER(C.c_uint8))
    keep["gks"] = None if gks_scale is None else np.ascontiguousarray(gks_scale, dtype=np.float64)
    mo.node_gks_scale = ptr(keep["gks"])
    mo.user_xi = float(user_xi)
    mo.newton_cap = int(newton_cap)
    mo.tt_jacobian = int(tt_jacobian)
    mo.mh_abs_mode = int(mh_abs_mode)
    keep["init"] = None if initial_states is None else np.ascontiguousarray(initial_states, dtype=np.float64)
    mo.initial_states = ptr(keep["init"])
    return md, mo, keep


def _solver_desc(dt, ionic_dt, cg_tol, cg_maxit, smoothing_alpha, precision, newton_tol, ecg_every,
                 act_threshold, scheme=capi.SCHEME_CN, diffusion_dt=0.0):
    sd = capi.SolverDesc()
    sd.dt, sd.ionic_dt = float(dt), float(ionic_dt)
    sd.cg_tol, sd.cg_maxit = float(cg_tol), int(cg_maxit)
    sd.smoothing_alpha = float(smoothing_alpha)
    sd.precision = int(precision)
    sd.newton_tol = float(newton_tol)
    sd.ecg_every = int(ecg_every)
    sd.act_threshold = float(act_threshold)
    sd.scheme = int(scheme)
    sd.diffusion_dt = float(diffusion_dt)
    return sd


class Monodomain:
    """One tissue instance on one GPU (FP64 or FP32 arithmetic).

    mesh: :class:`ucla_cmg_b200.mesh.TetMesh` (zero-based tets)
    model: capi.TUSSCHER / MAHAJAN / MAHAJAN_FAIL / LUORUDY / LUORUDYWITHGATE
    D: (D_f, D_s, D_n) in cm^2/ms; Cm in uF/cm^2
    """

    def __init__(self, mesh, model=capi.TUSSCHER, precision=capi.FP64, dt=0.02, ionic_dt=0.02,
                 D=(1e-3, 5e-4, 2.5e-4), Cm=1.0, cg_tol=1e-7, cg_maxit=1000, node_type=None,
                 type_consts=None, n_types=None, gks_scale=None, user_xi=0.0, newton_cap=0,
                 tt_jacobian=capi.TT_JAC_REFERENCE, mh_abs_mode=0, initial_states=None,
                 smoothing_alpha=0.0, newton_tol=0.0, ecg_every=0, act_threshold=-40.0, device=0,
                 scheme=capi.SCHEME_CN, diffusion_dt=0.0, cables=None, purkinje=None):
        """scheme: capi.SCHEME_CN (EP_CrankNicholson, the reference driver's),
        SCHEME_BE (EP_BackwardEuler) or SCHEME_EXPLICIT (EP_ExplicitSolver,
        diffusion sub-step diffusion_dt, 0: 0.05 ms).  cg_tol 0 takes the
        scheme's own (1e-7 CN, 1e-10 BE).

        Mixed tissues (ep_create_mixed): ``cables``, a dict of the keywords
        of :func:`assemble_operators` for 2-node cables (bars, bar_fibers,
        lv, Dp, DpLeft, radius, quad_order, angle, angle_sticky,
        bar_angle_node), and ``purkinje``, the zero-based nodes carrying the
        Purkinje cell; the states then come in rows of max(nstate, 22)."""
        L = capi.lib()
        self.mesh = mesh
        self.model = model
        self.precision = precision
        self.dt = float(dt)
        self.n = mesh.n
        md, mo, self._keep = _instance_descs(mesh, model, D, Cm, node_type, type_consts, n_types, gks_scale,
                                             user_xi, newton_cap, tt_jacobian, mh_abs_mode, initial_states)
        sd = _solver_desc(dt, ionic_dt, cg_tol, cg_maxit, smoothing_alpha, precision, newton_tol, ecg_every,
                          act_threshold, scheme, diffusion_dt)
        h = C.c_void_p()
        if cables is None and purkinje is None:
            check(L.ep_create(C.byref(md), C.byref(mo), C.byref(sd), int(device), C.byref(h)))
        else:
            cd = _cables_desc(self._keep, **cables) if cables is not None else None
            self._keep["purk"] = np.ascontiguousarray(purkinje if purkinje is not None else [], dtype=np.int32)
            check(L.ep_create_mixed(C.byref(md), C.byref(cd) if cd is not None else None, len(self._keep["purk"]),
                                    ptr(self._keep["purk"], C.POINTER(C.c_int32)), C.byref(mo), C.byref(sd),
                                    int(device), C.byref(h)))
        self._h = h
        self.nstate = L.ep_num_states(h)
        self.last_stats = None

    # ---- launch shape ----
    def launch_config(self):
        c = capi.LaunchConfig()
        check(capi.lib().ep_get_launch_config(self._h, C.byref(c)))
        return c.as_dict()

    def set_launch_config(self, cg_block=None, cg_per_sm=None, ionic_block=None, graph_steps=None,
                          ionic_min_ctas=None, cg_batch=None, cg_variant=None, cg_predict=None,
                          cg_prefetch=None, sg_variant=None):
        cur = self.launch_config()
        c = capi.LaunchConfig()
        c.cg_block = cur["cg_block"] if cg_block is None else int(cg_block)
        c.cg_per_sm = cur["cg_per_sm"] if cg_per_sm is None else int(cg_per_sm)
        c.ionic_block = cur["ionic_block"] if ionic_block is None else int(ionic_block)
        c.graph_steps = cur["graph_steps"] if graph_steps is None else int(graph_steps)
        c.ionic_min_ctas = cur["ionic_min_ctas"] if ionic_min_ctas is None else int(ionic_min_ctas)
        c.cg_batch = cur["cg_batch"] if cg_batch is None else int(cg_batch)
        c.cg_variant = cur["cg_variant"] if cg_variant is None else int(cg_variant)
        c.cg_predict = cur["cg_predict"] if cg_predict is None else int(cg_predict)
        c.cg_prefetch = cur["cg_prefetch"] if cg_prefetch is None else int(cg_prefetch)
        c.sg_variant = cur["sg_variant"] if sg_variant is None else int(sg_variant)
        check(capi.lib().ep_set_launch_config(self._h, C.byref(c)))

    def autotune(self, trial_steps=20):
        """Pick the launch shape by timing (ep_autotune); returns
        (config dict, ms/step chosen, ms/step at the start, configurations tried)."""
        c = capi.LaunchConfig()
        best, start = C.c_double(), C.c_double()
        tried = C.c_int32()
        check(capi.lib().ep_autotune(self._h, int(trial_steps), C.byref(c), C.byref(best), C.byref(start),
                                     C.byref(tried)))
        return c.as_dict(), best.value, start.value, tried.value

    # ---- life cycle ----
    def close(self):
        if getattr(self, "_h", None):
            capi.lib().ep_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state ----
    def set_voltage(self, V):
        V = np.ascontiguousarray(np.broadcast_to(np.asarray(V, dtype=np.float64), (self.n,)))
        check(capi.lib().ep_set_voltage(self._h, ptr(V)))

    InitializeVoltage = set_voltage

    def voltage(self):
        out = np.empty(self.n)
        check(capi.lib().ep_get_voltage(self._h, ptr(out)))
        return out

    def model_voltage(self):
        out = np.empty(self.n)
        check(capi.lib().ep_get_model_voltage(self._h, ptr(out)))
        return out

    def states(self):
        out = np.empty((self.n, self.nstate))
        check(capi.lib().ep_get_states(self._h, ptr(out)))
        return out

    def set_states(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(self.n, self.nstate)
        check(capi.lib().ep_set_states(self._h, ptr(s)))

    # ---- stimulus, electrodes ----
    def set_stimulus(self, node_ids, t_on, t_off, amp):
        """Per-entry nodal windows [t_on, t_off) in ms, amplitude uA/cm^3."""
        ids = np.ascontiguousarray(node_ids, dtype=np.int32)
        k = len(ids)
        t0 = np.ascontiguousarray(np.broadcast_to(np.asarray(t_on, dtype=np.float64), (k,)))
        t1 = np.ascontiguousarray(np.broadcast_to(np.asarray(t_off, dtype=np.float64), (k,)))
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(amp, dtype=np.float64), (k,)))
        check(capi.lib().ep_set_stimulus(self._h, k, ptr(ids, C.POINTER(C.c_int32)), ptr(t0),
                                         ptr(t1), ptr(a)))

    def set_electrodes(self, xyz, D_ecg=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._ne = len(xyz)
        D = None if D_ecg is None else np.ascontiguousarray(D_ecg, dtype=np.float64)
        check(capi.lib().ep_set_electrodes(self._h, len(xyz), ptr(xyz), ptr(D)))

    def compute_ecg(self):
        out = np.empty(self._ne)
        check(capi.lib().ep_compute_ecg(self._h, ptr(out)))
        return out

    def ecg(self):
        n = C.c_int32(0)
        check(capi.lib().ep_get_ecg(self._h, None, 0, C.byref(n), None))
        out = np.empty((n.value, self._ne))
        t = np.empty(n.value)
        if n.value:
            check(capi.lib().ep_get_ecg(self._h, ptr(out), n.value, C.byref(n), ptr(t)))
        return t, out

    # ---- time stepping ----
    def step(self, n_steps=1):
        """Advance n_steps; returns the step statistics.  On an error status
        (EP_ERR_NAN, EP_ERR_TIMEOUT, ...) raises EPError, with the call's
        statistics still in ``last_stats``."""
        st = capi.StepStats()
        rc = capi.lib().ep_step(self._h, int(n_steps), C.byref(st))
        self.last_stats = st.as_dict()
        check(rc)
        return self.last_stats

    def set_wait_limits(self, grid_polls=0, mbar_polls=0):
        """Poll limits of the in-kernel waits (0: the built-in ones)."""
        check(capi.lib().ep_set_wait_limits(self._h, int(grid_polls), int(mbar_polls)))

    def test_hold_barrier(self, extra_arrivals):
        """Test hook: the CG barrier waits for arrivals that never come."""
        check(capi.lib().ep_test_hold_barrier(self._h, int(extra_arrivals)))

    def diffusion_half_step(self):
        """One CN half diffusion step on the current V; returns (CG
        iterations, final ||r||/||r0||)."""
        it = C.c_int32(0)
        rr = C.c_double(0)
        check(capi.lib().ep_diffusion_half_step(self._h, C.byref(it), C.byref(rr)))
        return it.value, rr.value

    def set_profiling(self, on=True):
        check(capi.lib().ep_set_profiling(self._h, int(bool(on))))

    def Solve(self):
        """EP_CrankNicholson::Solve: one global step."""
        return self.step(1)

    def time(self):
        t = C.c_double(0)
        s = C.c_int64(0)
        check(capi.lib().ep_get_time(self._h, C.byref(t), C.byref(s)))
        return t.value, s.value

    def activation(self):
        ta = np.empty(self.n)
        apd = np.empty(self.n)
        check(capi.lib().ep_get_activation(self._h, ptr(ta), ptr(apd)))
        return ta, apd

    # ---- reference file formats ----
    def write_output(self, t, directory):
        check(capi.lib().ep_write_output(self._h, float(t), str(directory).encode()))

    WriteOutput = write_output

    def write_restart(self, t, directory):
        check(capi.lib().ep_write_restart(self._h, float(t), str(directory).encode()))

    writeRestart = write_restart

    def read_restart(self, t, directory):
        check(capi.lib().ep_read_restart(self._h, float(t), str(directory).encode()))

    readRestart = read_restart


class Batch(Monodomain):
    """Independent tissue instances advanced together (ep_batch_create).

    instances: list of dicts with the per-instance keywords of
    :class:`Monodomain` (mesh, and optionally D, node_type, type_consts,
    n_types, gks_scale, initial_states); the cell model, C_m and the solver
    settings are shared.  Every per-node array of the API is the instances'
    nodes concatenated in order: ``offsets[k]`` is where instance k starts.
    """

    def __init__(self, instances, model=capi.TUSSCHER, precision=capi.FP32, dt=0.02, ionic_dt=0.02,
                 Cm=1.0, cg_tol=1e-7, cg_maxit=1000, user_xi=0.0, newton_cap=0,
                 tt_jacobian=capi.TT_JAC_REFERENCE, mh_abs_mode=0, smoothing_alpha=0.0, newton_tol=0.0,
                 act_threshold=-40.0, device=0):
        L = capi.lib()
        self.model = model
        self.precision = precision
        self.dt = float(dt)
        self.meshes = [inst["mesh"] for inst in instances]
        k = len(instances)
        mds = (capi.MeshDesc * k)()
        mos = (capi.ModelDesc * k)()
        self._keep = []
        for i, inst in enumerate(instances):
            md, mo, keep = _instance_descs(inst["mesh"], model, inst.get("D", (1e-3, 5e-4, 2.5e-4)), Cm,
                                           inst.get("node_type"), inst.get("type_consts"), inst.get("n_types"),
                                           inst.get("gks_scale"), user_xi, newton_cap, tt_jacobian, mh_abs_mode,
                                           inst.get("initial_states"))
            mds[i] = md
            mos[i] = mo
            self._keep.append(keep)
        sd = _solver_desc(dt, ionic_dt, cg_tol, cg_maxit, smoothing_alpha, precision, newton_tol, 0,
                          act_threshold)
        h = C.c_void_p()
        check(L.ep_batch_create(k, mds, mos, C.byref(sd), int(device), C.byref(h)))
        self._h = h
        self.nstate = L.ep_num_states(h)
        self.n = L.ep_num_nodes(h)
        self.last_stats = None
        self.n_inst = k
        off = np.zeros(k + 1, np.int32)
        cta = np.zeros(k + 1, np.int32)
        check(L.ep_batch_layout(h, None, ptr(off, C.POINTER(C.c_int32)), ptr(cta, C.POINTER(C.c_int32))))
        self.offsets = off
        self.cta_offsets = cta

    def split(self, a):
        """Per-instance views of a concatenated per-node array."""
        return [a[self.offsets[k]:self.offsets[k + 1]] for k in range(self.n_inst)]

    def cg_last(self):
        it = np.zeros(self.n_inst, np.int32)
        rr = np.zeros(self.n_inst)
        check(capi.lib().ep_batch_cg_last(self._h, ptr(it, C.POINTER(C.c_int32)), ptr(rr)))
        return it, rr


def batch_plan(inst_row, grid):
    """The CTA-group split of the persistent CG launch (ep_batch_plan)."""
    row = np.ascontiguousarray(inst_row, dtype=np.int32)
    out = np.zeros(len(row), np.int32)
    check(capi.lib().ep_batch_plan(len(row) - 1, ptr(row, C.POINTER(C.c_int32)), int(grid),
                                   ptr(out, C.POINTER(C.c_int32))))
    return out


def _cables_desc(keep, bars, Dp=(0.0016,) * 3, DpLeft=None, radius=0.0275, bar_fibers=None, lv=None,
                 quad_order=2, angle=None, angle_sticky=True, bar_angle_node=None):
    """capi.CablesDesc of 2-node cables (zero-based), the arrays kept in ``keep``."""
    keep["bars"] = np.ascontiguousarray(bars, dtype=np.int32).reshape(-1, 2)
    keep["bfib"] = None if bar_fibers is None else np.ascontiguousarray(bar_fibers, dtype=np.float64)
    keep["lv"] = None if lv is None else np.ascontiguousarray(lv, dtype=np.uint8)
    cd = capi.CablesDesc()
    cd.n_bars = len(keep["bars"])
    cd.bars = ptr(keep["bars"], C.POINTER(C.c_int32))
    cd.one_based = 0
    cd.fibers = ptr(keep["bfib"])
    cd.lv = ptr(keep["lv"], C.POINTER(C.c_uint8))
    for k in range(3):
        cd.Dp[k] = float(Dp[k])
        cd.DpLeft[k] = float((DpLeft if DpLeft is not None else Dp)[k])
    cd.radius = float(radius)
    cd.quad_order = int(quad_order)
    cd.angle_sticky = int(bool(angle_sticky))
    if angle:
        keep["an"] = np.array(sorted(angle), dtype=np.int32)
        keep["ad"] = np.array([angle[k] for k in sorted(angle)], dtype=np.float64).reshape(-1, 4)
        cd.n_angle = len(keep["an"])
        cd.angle_nodes = ptr(keep["an"], C.POINTER(C.c_int32))
        cd.angle = ptr(keep["ad"])
        if bar_angle_node is not None:
            row = {int(v): k for k, v in enumerate(keep["an"])}
            keep["ba"] = np.array([row[int(v)] if v >= 0 else -1 for v in bar_angle_node], dtype=np.int32)
            cd.bar_angle = ptr(keep["ba"], C.POINTER(C.c_int32))
    return cd


def assemble_operators(mesh, D, dt, Cm=1.0, scheme=capi.SCHEME_CN, smoothing_alpha=0.0, bars=None,
                       Dp=(0.0016,) * 3, DpLeft=None, radius=0.0275, bar_fibers=None, lv=None, quad_order=2,
                       angle=None, angle_sticky=True, bar_angle_node=None):
    """The FP64 operators ep_create builds, assembled on the host only
    (ep_assemble_operators; no GPU): scipy CSR matrices A and B and the
    lumped capacitance C_L.  ``bars`` (nb x 2, zero-based) adds 2-node
    Purkinje cables after the tets; ``angle`` maps a zero-based node to
    (dx, dy, dz, length) as in a .angle file; ``bar_angle_node`` (per cable,
    the node whose row overrides it or -1, from
    :func:`ucla_cmg_b200.voomep_io.bar_angle_nodes` over the .ele order)
    replaces the bars-only sticky rule."""
    import scipy.sparse as sp
    md, _, keep = _instance_descs(mesh, capi.TUSSCHER, D, Cm, None, None, None, None, 0.0, 0, 0, 0, None)
    sd = _solver_desc(dt, dt, 1e-7, 1000, smoothing_alpha, capi.FP64, 0.0, 0, -40.0, scheme)
    cd = None
    if bars is not None:
        cd = _cables_desc(keep, bars, Dp, DpLeft, radius, bar_fibers, lv, quad_order, angle, angle_sticky,
                          bar_angle_node)
    nnz = C.c_int64(0)
    L = capi.lib()
    cdp = C.byref(cd) if cd is not None else None
    check(L.ep_assemble_operators(C.byref(md), cdp, C.byref(sd), C.byref(nnz), None, None, None, None, None))
    n = mesh.n
    rowptr = np.zeros(n + 1, np.int32)
    col = np.zeros(nnz.value, np.int32)
    A, B, CL = np.zeros(nnz.value), np.zeros(nnz.value), np.zeros(n)
    ip = C.POINTER(C.c_int32)
    check(L.ep_assemble_operators(C.byref(md), cdp, C.byref(sd), C.byref(nnz), ptr(rowptr, ip), ptr(col, ip),
                                  ptr(A), ptr(B), ptr(CL)))
    return (sp.csr_matrix((A, col, rowptr), shape=(n, n)), sp.csr_matrix((B, col, rowptr), shape=(n, n)), CL)


def ionic_step(model, V, istim, states, dt, Cm=1.0, precision=capi.FP64, node_type=None,
               type_consts=None, gks_scale=None, user_xi=0.0, newton_cap=0,
               tt_jacobian=capi.TT_JAC_REFERENCE, mh_abs_mode=0):
    """Batched IonicModel::Compute_Ion: returns dV/dt, updates ``states``
    (n x nstate, node-major, FP64) in place."""
    n = len(V)
    V = np.ascontiguousarray(V, dtype=np.float64)
    istim = np.ascontiguousarray(np.broadcast_to(np.asarray(istim, dtype=np.float64), (n,)))
    assert states.dtype == np.float64 and states.flags.c_contiguous
    mo = capi.ModelDesc()
    mo.model = model
    types = None if node_type is None else np.ascontiguousarray(node_type, dtype=np.uint8)
    tc = None if type_consts is None else np.ascontiguousarray(type_consts, dtype=np.float64)
    mo.n_types = tc.shape[0] if tc is not None else (int(types.max()) + 1 if types is not None else 1)
    mo.type_consts = ptr(tc)
    mo.node_type = ptr(types, C.POINTER(C.c_uint8))
    g = None if gks_scale is None else np.ascontiguousarray(gks_scale, dtype=np.float64)
    mo.node_gks_scale = ptr(g)
    mo.user_xi = float(user_xi)
    mo.newton_cap = int(newton_cap)
    mo.tt_jacobian = int(tt_jacobian)
    mo.mh_abs_mode = int(mh_abs_mode)
    out = np.empty(n)
    check(capi.lib().ep_ionic_step(C.byref(mo), int(precision), n, float(dt), float(Cm), ptr(V),
                                   ptr(istim), ptr(states), ptr(out)))
    return out
