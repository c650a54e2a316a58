"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries sit behind it:

* ``libep_oracle.so`` -- the plain-C FP64 restatement of the voomEP
  monodomain path (``ep_oracle.c``);
* ``_ref/libvoomep_ref.so`` -- the reference's own cell-model sources
  (voomEP/src/IonicModel/{Tusscher,Mahajan,Mahajan_fail,LR,Purkinje}.cc) compiled
  unmodified, used to pin the restatement and as the CPU reference arm.

* ``_ref/libvoomep_fem.so`` -- the reference's own mesh reader
  (voomEP/src/Mesh/Mesh.cc), tet and cable geometry (TetMesh.cc,
  MixedMesh3D.cc), element assembly (Body/CardiacBody.cc) and pseudo-ECG
  (Applications/CardiacEP/ComputeECG.h), compiled unmodified against
  stand-in headers; it pins the restatement's operators and ECG.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the product package never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

TUSSCHER, MAHAJAN, MAHAJAN_FAIL, LUORUDY, LUORUDYWITHGATE = 2, 3, 4, 0, 1
PURKINJE = 5          # the cell model of .purk nodes (not in CellModelType)
NSTATE = {TUSSCHER: 19, MAHAJAN: 26, MAHAJAN_FAIL: 26, LUORUDY: 8, LUORUDYWITHGATE: 8, PURKINJE: 22}

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def _p(a, t=dp):
    return a.ctypes.data_as(t) if a is not None else None


class _Csr(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("rowptr", ip), ("col", ip),
                ("A", dp), ("B", dp), ("M", dp), ("K", dp), ("CL", dp)]


class _Cables(C.Structure):
    _fields_ = [("nb", C.c_int), ("bars", ip), ("fibers", dp), ("lv", C.POINTER(C.c_uint8)),
                ("Dp", C.c_double * 3), ("DpLeft", C.c_double * 3), ("radius", C.c_double),
                ("quad_order", C.c_int), ("orient_has", C.POINTER(C.c_uint8)), ("orient", dp),
                ("orient_sticky", C.c_int), ("bar_orient_node", ip)]


class _Cells(C.Structure):
    _fields_ = [("model", C.c_int), ("n", C.c_int), ("nstate", C.c_int), ("nconst", C.c_int),
                ("state", dp), ("consts", dp), ("ntypes", C.c_int),
                ("type", C.POINTER(C.c_uint8)), ("gks_scale", dp), ("alg12", dp),
                ("lr_table", dp), ("Xi", C.c_double), ("user_Xi", C.c_double),
                ("user_xi", C.c_int), ("newton_cap", C.c_int), ("tt_jac_true", C.c_int),
                ("mh_abs_mode", C.c_int),
                ("newton_total", C.c_longlong), ("newton_max", C.c_longlong),
                ("substep_count", C.c_longlong)]


class _Sim(C.Structure):
    _fields_ = [("csr", C.POINTER(_Csr)), ("n", C.c_int), ("dt", C.c_double),
                ("ionic_dt", C.c_double), ("Cm", C.c_double), ("cg_tol", C.c_double),
                ("cg_maxit", C.c_int), ("jacobi_steps", C.c_int),
                ("V", dp), ("istim", dp), ("dvdt", dp), ("b", dp), ("ici", dp),
                ("ionic", C.c_void_p), ("ionic_ctx", C.c_void_p),
                ("nsub", C.c_int), ("sub_dt", C.c_double * 64),
                ("cg_iters_total", C.c_longlong), ("cg_fail", C.c_int), ("step", C.c_long),
                ("scheme", C.c_int), ("ionic_node", C.c_void_p), ("A_be", dp), ("B_be", dp),
                ("nex", C.c_int), ("ex_h", C.c_double * 4096)]


def build():
    """Compile the oracle (and, where the reference sources exist, _ref)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "libep_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.epo_cells_create.restype = C.POINTER(_Cells)
        L.epo_cells_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        L.epo_cells_destroy.argtypes = [C.c_void_p]
        L.epo_cells_compute_ion.argtypes = [C.c_void_p, C.c_double, C.c_double, dp, dp, dp]
        L.epo_cells_initial_voltage.argtypes = [C.c_void_p, dp]
        L.epo_assemble.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.c_double, C.c_double,
                                   C.c_double, C.POINTER(_Csr)]
        L.epo_assemble_mixed.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.POINTER(_Cables),
                                         C.c_double, C.c_double, C.c_double, C.POINTER(_Csr)]
        L.epo_csr_free.argtypes = [C.POINTER(_Csr)]
        L.epo_spmv.argtypes = [C.POINTER(_Csr), dp, dp, dp]
        L.epo_pcg.argtypes = [C.POINTER(_Csr), dp, dp, dp, C.c_double, C.c_int, C.c_int, dp]
        L.epo_ecg_elementwise.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.c_int, dp, dp, dp]
        L.epo_ecg_weights.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.c_int, dp, dp]
        L.epo_ecg_weights_cables.argtypes = [C.c_int, dp, C.POINTER(_Cables), dp, C.c_int, dp, dp]
        L.epo_sim_init.argtypes = [C.POINTER(_Sim), C.POINTER(_Csr), C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                   C.c_void_p]
        L.epo_sim_free.argtypes = [C.POINTER(_Sim)]
        L.epo_sim_step.argtypes = [C.POINTER(_Sim)]
        L.epo_sim_set_scheme.argtypes = [C.POINTER(_Sim), C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.epo_stim_schedule.argtypes = [C.c_int, dp, dp, C.c_double, C.c_long,
                                        C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.epo_num_steps.restype = C.c_long
        L.epo_num_steps.argtypes = [C.c_double, C.c_double]
        L.epo_set_threads.argtypes = [C.c_int]
        L.epo_get_threads.restype = C.c_int
        L.epo_tt_constants.argtypes = [dp]
        L.epo_mh_constants.argtypes = [dp, C.c_int, C.c_int]
        L.epo_tt_initial_state.argtypes = [dp]
        L.epo_mh_initial_state.argtypes = [dp, C.c_int]
        L.epo_lr_initial_state.argtypes = [dp]
        L.epo_pk_constants.argtypes = [dp]
        L.epo_mixed_init.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.epo_mixed_free.argtypes = [C.c_void_p]
        L.epo_pk_initial_state.argtypes = [dp]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference cell models compiled unmodified (None if not built)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libvoomep_ref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_cells_create.restype = C.c_void_p
        L.ref_cells_create.argtypes = [C.c_int, C.c_int, C.c_void_p]
        L.ref_cells_destroy.argtypes = [C.c_void_p]
        L.ref_cells_nstate.argtypes = [C.c_void_p]
        L.ref_cells_compute_ion.argtypes = [C.c_void_p, C.c_double, C.c_double, dp, dp, dp]
        L.ref_cells_get_states.argtypes = [C.c_void_p, dp]
        L.ref_cells_set_states.argtypes = [C.c_void_p, dp]
        L.ref_cells_get_voltage.argtypes = [C.c_void_p, dp]
        L.ref_cells_set_user_xi.argtypes = [C.c_void_p, C.c_double]
        L.epo_assemble.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.c_double, C.c_double,
                                   C.c_double, C.POINTER(_Csr)]
        L.epo_assemble_mixed.argtypes = [C.c_int, dp, C.c_int, ip, dp, dp, C.POINTER(_Cables),
                                         C.c_double, C.c_double, C.c_double, C.POINTER(_Csr)]
        L.epo_csr_free.argtypes = [C.POINTER(_Csr)]
        L.epo_sim_init.argtypes = [C.POINTER(_Sim), C.POINTER(_Csr), C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                   C.c_void_p]
        L.epo_sim_step.argtypes = [C.POINTER(_Sim)]
        L.epo_sim_set_scheme.argtypes = [C.POINTER(_Sim), C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.epo_sim_free.argtypes = [C.POINTER(_Sim)]
        L.epo_set_threads.argtypes = [C.c_int]
        _REF = L
    return _REF


_FEM = None


def ref_fem_lib():
    """The reference's FEM sources compiled unmodified (None if not built)."""
    global _FEM
    if _FEM is None:
        path = os.path.join(HERE, "_ref", "libvoomep_fem.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.fem_mesh_new.restype = C.c_void_p
        L.fem_mesh_new.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double]
        L.fem_mesh_compute.argtypes = [C.c_void_p]
        L.fem_mesh_free.argtypes = [C.c_void_p]
        for f in ("fem_mesh_num_points", "fem_mesh_num_elements", "fem_mesh_num_local_nodes"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.fem_mesh_points.argtypes = [C.c_void_p, ip, dp, dp, dp]
        L.fem_body_new.restype = C.c_void_p
        L.fem_body_new.argtypes = [C.c_void_p, C.c_int, dp, C.c_double, dp, dp]
        L.fem_body_free.argtypes = [C.c_void_p]
        L.fem_body_diffusion.restype = C.c_long
        L.fem_body_diffusion.argtypes = [C.c_void_p, C.c_double, ip, ip, dp]
        L.fem_body_capacitance.restype = C.c_long
        L.fem_body_capacitance.argtypes = [C.c_void_p, C.c_int, ip, ip, dp]
        L.fem_body_lumped.argtypes = [C.c_void_p, dp]
        L.fem_ecg.argtypes = [C.c_void_p, dp, C.c_int, dp, dp, dp]
        _FEM = L
    return _FEM


def write_reference_case(base, xyz, elements, fibers=None, purk=None, cell=None, angle=None):
    """Mesh files as the reference's Mesh::New reads them (Mesh.cc:142-483):
    <base>.node (``n 3 0 0``, then ``id x y z``), <base>.ele (``m 0 0``, then
    ``id k n1..nk``, 1-based), <base>.fibers (9 numbers per element), the
    one-rank partition files <base>.metis.npart.1 / .metis.epart.1 (read
    even for one rank), and optionally .purk, .cell and .angle.
    ``elements``: list of zero-based node-id sequences (4 for a tet, 2 for a
    cable); ``purk``: zero-based node ids; ``cell``: per-node type;
    ``angle``: {zero-based node: (dx, dy, dz, length)}."""
    n = len(xyz)
    with open(base + ".node", "w") as f:
        f.write(f"{n} 3 0 0\n")
        for i, p in enumerate(xyz):
            f.write(f"{i + 1} {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
    with open(base + ".ele", "w") as f:
        f.write(f"{len(elements)} 0 0\n")
        for e, el in enumerate(elements):
            f.write(" ".join(str(v) for v in [e + 1, len(el)] + [int(x) + 1 for x in el]) + "\n")
    if fibers is not None:
        np.savetxt(base + ".fibers", np.asarray(fibers).reshape(len(elements), 9), fmt="%.17g")
    with open(base + ".metis.npart.1", "w") as f:
        f.write("0\n" * n)
    with open(base + ".metis.epart.1", "w") as f:
        f.write("0\n" * len(elements))
    if purk is not None:
        with open(base + ".purk", "w") as f:
            f.write(f"{len(purk)}\n" + "\n".join(str(int(i) + 1) for i in purk) + "\n")
    if cell is not None:
        with open(base + ".cell", "w") as f:
            for i, t in enumerate(cell):
                f.write(f"{i + 1} {int(t)}\n")
    if angle:
        with open(base + ".angle", "w") as f:
            for k, v in sorted(angle.items()):
                f.write(f"{k + 1} {v[0]:.17g} {v[1]:.17g} {v[2]:.17g} {v[3]:.17g}\n")


class RefFemMesh:
    """Mesh::New + setRadius of the reference on files written by
    :func:`write_reference_case` (one rank).  ``compute=True`` runs
    Mesh::Compute at once, as ComputeECG does; a mesh handed to
    :class:`RefFemBody` is computed by the CardiacBody constructor instead."""

    def __init__(self, base, quad_order=2, mixed=False, radius=0.0275, compute=False):
        L = ref_fem_lib()
        if L is None:
            raise RuntimeError("oracle/_ref/libvoomep_fem.so is not built")
        self.h = L.fem_mesh_new(base.encode(), int(quad_order), int(bool(mixed)), float(radius))
        self.n = L.fem_mesh_num_local_nodes(self.h)
        self.n_elements = L.fem_mesh_num_elements(self.h)
        if compute:
            L.fem_mesh_compute(self.h)

    def points(self):
        """Per quadrature point: node count k, N[4], dN/dx[4, 3], w*J."""
        L = ref_fem_lib()
        q = L.fem_mesh_num_points(self.h)
        k = np.zeros(q, np.int32)
        N = np.zeros((q, 4))
        dN = np.zeros((q, 4, 3))
        w = np.zeros(q)
        L.fem_mesh_points(self.h, _p(k, ip), _p(N), _p(dN), _p(w))
        return k, N, dN, w

    def ecg(self, D, electrodes, V):
        """ComputeECG.h's chain for the nodal voltage V (global order)."""
        el = np.ascontiguousarray(electrodes, dtype=np.float64).reshape(-1, 3)
        D = np.ascontiguousarray(D, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros(len(el))
        ref_fem_lib().fem_ecg(self.h, _p(D), len(el), _p(el), _p(V), _p(out))
        return out

    def __del__(self):
        try:
            ref_fem_lib().fem_mesh_free(self.h)
        except Exception:
            pass


class RefFemBody:
    """CardiacBody::New(mesh, model) + Compute of the reference; matrices as
    scipy CSR (the inserted triplets summed)."""

    def __init__(self, mesh, model, D, Cm=1.0, Dp=None, DpLeft=None):
        L = ref_fem_lib()
        self.mesh = mesh
        D = np.ascontiguousarray(D, dtype=np.float64)
        Dp = None if Dp is None else np.ascontiguousarray(Dp, dtype=np.float64)
        DpL = None if DpLeft is None else np.ascontiguousarray(DpLeft, dtype=np.float64)
        self.h = L.fem_body_new(mesh.h, int(model), _p(D), float(Cm), _p(Dp), _p(DpL))

    def _triplets(self, fn, arg):
        import scipy.sparse as sp
        L = ref_fem_lib()
        m = getattr(L, fn)(self.h, arg, None, None, None)
        r = np.zeros(m, np.int32)
        c = np.zeros(m, np.int32)
        v = np.zeros(m)
        getattr(L, fn)(self.h, arg, _p(r, ip), _p(c, ip), _p(v))
        n = self.mesh.n
        return sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsr()

    def diffusion(self, scale=1.0):
        """getDiffusionMatrix(M, scale): scale x K (K includes C_m)."""
        return self._triplets("fem_body_diffusion", float(scale))

    def capacitance(self, is_cap=True):
        """getCapacitanceMatrix(M, isCap): C_m M (or M)."""
        return self._triplets("fem_body_capacitance", int(bool(is_cap)))

    def lumped(self):
        out = np.zeros(self.mesh.n)
        ref_fem_lib().fem_body_lumped(self.h, _p(out))
        return out

    def __del__(self):
        try:
            ref_fem_lib().fem_body_free(self.h)
        except Exception:
            pass


def set_threads(n):
    lib().epo_set_threads(int(n))
    r = ref_lib()
    if r is not None:
        r.epo_set_threads(int(n))


def tt_constants():
    c = np.zeros(54)
    lib().epo_tt_constants(_p(c))
    return c


def mh_constants(pos, failing=False):
    c = np.zeros(35)
    lib().epo_mh_constants(_p(c), int(pos), int(bool(failing)))
    return c


def pk_constants():
    c = np.zeros(63)
    lib().epo_pk_constants(_p(c))
    return c


def initial_state(model, pos=0):
    L = lib()
    if model == TUSSCHER:
        s = np.zeros(19); L.epo_tt_initial_state(_p(s))
    elif model == PURKINJE:
        s = np.zeros(22); L.epo_pk_initial_state(_p(s))
    elif model in (MAHAJAN, MAHAJAN_FAIL):
        s = np.zeros(26); L.epo_mh_initial_state(_p(s), int(pos))
    else:
        s = np.zeros(8); L.epo_lr_initial_state(_p(s))
    return s


class Cells:
    """Oracle population: one state row per node (node-major, FP64)."""

    def __init__(self, model, n, types=None, type_consts=None, gks_scale=None,
                 newton_cap=0, mh_abs_mode=0, user_xi=None, tt_jac_true=0):
        L = lib()
        self.model, self.n = model, n
        self._types = None if types is None else np.ascontiguousarray(types, dtype=np.uint8)
        self._tc = None
        ntypes = 0
        if type_consts is not None:
            self._tc = np.ascontiguousarray(type_consts, dtype=np.float64)
            ntypes = self._tc.shape[0]
        elif self._types is not None:
            ntypes = int(self._types.max()) + 1 if n else 1
            if model == TUSSCHER:
                ntypes = 1
        self.h = L.epo_cells_create(model, n, _p(self._types, C.c_void_p) if self._types is not None else None,
                                    ntypes, _p(self._tc, C.c_void_p) if self._tc is not None else None)
        c = self.h.contents
        c.newton_cap = int(newton_cap)
        c.tt_jac_true = int(tt_jac_true)
        c.mh_abs_mode = int(mh_abs_mode)
        if user_xi is not None:
            c.user_Xi = float(user_xi); c.user_xi = 1
        self.nstate = c.nstate
        if gks_scale is not None:
            # malloc'd by libc so that epo_cells_destroy can free it
            libc = C.CDLL(None)
            libc.malloc.restype = C.c_void_p
            buf = libc.malloc(C.c_size_t(8 * n))
            arr = np.ctypeslib.as_array(C.cast(buf, dp), shape=(n,))
            arr[:] = gks_scale
            c.gks_scale = C.cast(buf, dp)

    @property
    def state(self):
        c = self.h.contents
        return np.ctypeslib.as_array(c.state, shape=(self.n, self.nstate))

    @property
    def newton_stats(self):
        c = self.h.contents
        return c.newton_total, c.newton_max

    def compute_ion(self, V, istim, dt, Cm=1.0):
        V = np.ascontiguousarray(V, dtype=np.float64)
        istim = np.ascontiguousarray(istim, dtype=np.float64)
        out = np.empty(self.n)
        lib().epo_cells_compute_ion(self.h, Cm, dt, _p(V), _p(istim), _p(out))
        return out

    def initial_voltage(self):
        V = np.empty(self.n)
        lib().epo_cells_initial_voltage(self.h, _p(V))
        return V

    def __del__(self):
        try:
            lib().epo_cells_destroy(self.h)
        except Exception:
            pass


class RefCells:
    """The reference's unmodified cell objects (one heap object per node)."""

    def __init__(self, model, n, types=None):
        L = ref_lib()
        if L is None:
            raise RuntimeError("oracle/_ref/libvoomep_ref.so is not built")
        self._types = None if types is None else np.ascontiguousarray(types, dtype=np.uint8)
        self.h = L.ref_cells_create(model, n, _p(self._types, C.c_void_p) if self._types is not None else None)
        self.n, self.model = n, model
        self.nstate = L.ref_cells_nstate(self.h)

    def compute_ion(self, V, istim, dt, Cm=1.0):
        V = np.ascontiguousarray(V, dtype=np.float64)
        istim = np.ascontiguousarray(istim, dtype=np.float64)
        out = np.empty(self.n)
        ref_lib().ref_cells_compute_ion(self.h, Cm, dt, _p(V), _p(istim), _p(out))
        return out

    @property
    def state(self):
        out = np.empty((self.n, self.nstate))
        ref_lib().ref_cells_get_states(self.h, _p(out))
        return out

    @state.setter
    def state(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        ref_lib().ref_cells_set_states(self.h, _p(s))

    def get_voltage(self):
        out = np.empty(self.n)
        ref_lib().ref_cells_get_voltage(self.h, _p(out))
        return out

    def __del__(self):
        try:
            ref_lib().ref_cells_destroy(self.h)
        except Exception:
            pass


class Cables:
    """2-node Purkinje cables of a mixed mesh for ``Csr`` (see epo_cables):
    bars (nb x 2, zero-based), optional per-bar fibres and LV flags, the
    Purkinje diffusion, the cable radius and the .angle overrides."""

    def __init__(self, bars, Dp=(0.0016,) * 3, DpLeft=None, radius=0.0275, fibers=None, lv=None,
                 quad_order=2, orient=None, sticky=True, n=None, bar_orient_node=None):
        """bar_orient_node: per cable the node whose ``orient`` row overrides
        it (-1: none), resolved over the whole element order (see
        :func:`bar_angle_nodes`); given, it replaces the sticky rule."""
        self.bars = np.ascontiguousarray(bars, dtype=np.int32).reshape(-1, 2)
        self.fibers = None if fibers is None else np.ascontiguousarray(fibers, dtype=np.float64)
        self.lv = None if lv is None else np.ascontiguousarray(lv, dtype=np.uint8)
        self.c = _Cables()
        self.c.nb = len(self.bars)
        self.c.bars = _p(self.bars, ip)
        self.c.fibers = _p(self.fibers)
        self.c.lv = _p(self.lv, C.POINTER(C.c_uint8)) if self.lv is not None else None
        for k in range(3):
            self.c.Dp[k] = Dp[k]
            self.c.DpLeft[k] = (DpLeft if DpLeft is not None else Dp)[k]
        self.c.radius = radius
        self.c.quad_order = quad_order
        self.c.orient_sticky = int(bool(sticky))
        self.has = self.orient = self.bon = None
        if orient:                       # {node (zero-based): (dx, dy, dz, length)}
            self.has = np.zeros(n, np.uint8)
            self.orient = np.zeros((n, 4))
            for k, v in orient.items():
                self.has[k] = 1
                self.orient[k] = v
            self.c.orient_has = _p(self.has, C.POINTER(C.c_uint8))
            self.c.orient = _p(self.orient)
        if bar_orient_node is not None:
            self.bon = np.ascontiguousarray(bar_orient_node, dtype=np.int32)
            if self.orient is None:
                self.orient = np.zeros((n, 4))
                self.c.orient = _p(self.orient)
            self.c.bar_orient_node = _p(self.bon, ip)


def bar_angle_nodes(elements, angle, sticky=True):
    """Per 2-node element of ``elements`` (zero-based node lists in .ele
    order), the node whose .angle row overrides it, or -1: the rule of
    MixedMesh3D::Compute (MixedMesh3D.cc:30-34, 78-87), where every element
    whose first node is listed -- tets included -- switches the override on
    (sticky: it stays on, with the latest row, for every later cable) and
    ``sticky=False`` applies a row to the cable that starts at its node only."""
    out, cur = [], -1
    for el in elements:
        if el[0] in angle:
            cur = el[0]
        if len(el) == 2:
            if sticky:
                out.append(cur)
            else:
                out.append(el[0] if el[0] in angle else -1)
    return np.array(out, dtype=np.int32)


class Csr:
    """Assembled CN system (oracle); ``cables`` adds the 2-node Purkinje
    elements of a mixed mesh after the tets."""

    def __init__(self, xyz, tets, fibers=None, D=(1e-3, 1e-3, 1e-3), Cm=1.0, dt=0.02,
                 smoothing_alpha=0.0, L=None, cables=None):
        self._L = L or lib()
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.tets = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
        self.fibers = None if fibers is None else np.ascontiguousarray(fibers, dtype=np.float64)
        self.D = np.ascontiguousarray(D, dtype=np.float64)
        self.c = _Csr()
        self.cables = cables
        if cables is None:
            rc = self._L.epo_assemble(len(self.xyz), _p(self.xyz), len(self.tets), _p(self.tets, ip),
                                      _p(self.fibers), _p(self.D), Cm, dt, smoothing_alpha,
                                      C.byref(self.c))
        else:
            rc = self._L.epo_assemble_mixed(len(self.xyz), _p(self.xyz), len(self.tets), _p(self.tets, ip),
                                            _p(self.fibers), _p(self.D), C.byref(cables.c), Cm, dt,
                                            smoothing_alpha, C.byref(self.c))
        self.degenerate = rc != 0
        self.n, self.nnz = self.c.n, self.c.nnz

    def arr(self, name):
        size = self.n + 1 if name == "rowptr" else (self.n if name == "CL" else self.nnz)
        return np.ctypeslib.as_array(getattr(self.c, name), shape=(size,)).copy()

    def scipy(self, name):
        import scipy.sparse as sp
        return sp.csr_matrix((self.arr(name), self.arr("col"), self.arr("rowptr")),
                             shape=(self.n, self.n))

    def pcg(self, b, x0, tol=1e-7, maxit=1000, jacobi_steps=3):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64)
        rr = C.c_double(0)
        it = lib().epo_pcg(C.byref(self.c), self.c.A, _p(b), _p(x), tol, maxit, jacobi_steps,
                           C.byref(rr))
        return x, it, rr.value

    def __del__(self):
        try:
            self._L.epo_csr_free(C.byref(self.c))
        except Exception:
            pass


def ecg_elementwise(xyz, tets, fibers, D, electrodes, V):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    fib = None if fibers is None else np.ascontiguousarray(fibers, dtype=np.float64)
    D = np.ascontiguousarray(D, dtype=np.float64)
    el = np.ascontiguousarray(electrodes, dtype=np.float64)
    V = np.ascontiguousarray(V, dtype=np.float64)
    out = np.zeros(len(el))
    lib().epo_ecg_elementwise(len(xyz), _p(xyz), len(tets), _p(tets, ip), _p(fib), _p(D),
                              len(el), _p(el), _p(V), _p(out))
    return out


def ecg_weights(xyz, tets, fibers, D, electrodes, cables=None):
    """Per-node ECG weights W (ECG = W V); ``cables`` (a :class:`Cables`,
    its radius as ComputeECG sets it, 0.0275) adds the 2-node elements of a
    MIX3D mesh with the tissue D."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
    fib = None if fibers is None else np.ascontiguousarray(fibers, dtype=np.float64)
    D = np.ascontiguousarray(D, dtype=np.float64)
    el = np.ascontiguousarray(electrodes, dtype=np.float64).reshape(-1, 3)
    W = np.zeros((len(el), len(xyz)))
    lib().epo_ecg_weights(len(xyz), _p(xyz), len(tets), _p(tets, ip), _p(fib), _p(D),
                          len(el), _p(el), _p(W))
    if cables is not None:
        rc = lib().epo_ecg_weights_cables(len(xyz), _p(xyz), C.byref(cables.c), _p(D), len(el), _p(el), _p(W))
        if rc:
            raise ValueError("unsupported cable quadrature order")
    return W


def stim_schedule(t_start, t_stop, dt, nsteps):
    t0 = np.ascontiguousarray(t_start, dtype=np.float64)
    t1 = np.ascontiguousarray(t_stop, dtype=np.float64)
    s0 = (C.c_long * len(t0))()
    s1 = (C.c_long * len(t0))()
    lib().epo_stim_schedule(len(t0), _p(t0), _p(t1), dt, nsteps, s0, s1)
    return np.array(list(s0)), np.array(list(s1))


def num_steps(dt, T):
    return lib().epo_num_steps(dt, T)


class _Mixed(C.Structure):
    _fields_ = [("n", C.c_int), ("nt", C.c_int), ("np", C.c_int), ("tmap", ip), ("pmap", ip),
                ("tfn", C.c_void_p), ("pfn", C.c_void_p), ("tctx", C.c_void_p), ("pctx", C.c_void_p),
                ("buf", dp)]


def _cb(cells):
    """(callback, context) of a population for the split step."""
    if isinstance(cells, RefCells):
        return C.cast(ref_lib().ref_cells_ionic_cb, C.c_void_p), C.c_void_p(cells.h)
    return C.cast(lib().epo_cells_ionic_cb, C.c_void_p), C.cast(cells.h, C.c_void_p)


class MixedCells:
    """A tissue model on every node but the Purkinje nodes (is_purk), which
    carry the Purkinje cell (CardiacBody::New): two compact populations in
    increasing node order, each a Cells or a RefCells."""

    def __init__(self, tissue, purk, is_purk):
        self.tissue, self.purk = tissue, purk
        self.is_purk = np.ascontiguousarray(is_purk, dtype=np.uint8)
        self.n = len(self.is_purk)
        assert tissue.n == int((self.is_purk == 0).sum()) and purk.n == int(self.is_purk.sum())
        self.m = _Mixed()
        tf, tc = _cb(tissue)
        pf, pc = _cb(purk)
        self._mp = C.cast(C.pointer(self.m), C.c_void_p)
        lib().epo_mixed_init(self._mp, self.n, self.is_purk.ctypes.data_as(C.c_void_p), tf, tc, pf, pc)

    def __del__(self):
        try:
            lib().epo_mixed_free(self._mp)
        except Exception:
            pass


class Sim:
    """The split time step (EP_CrankNicholson::Solve) on the oracle.

    ``cells`` is a :class:`Cells` (restatement) or :class:`RefCells` (the
    reference objects); the FEM/PCG part is the C restatement either way.
    """

    def __init__(self, csr, cells, dt, ionic_dt, Cm=1.0, cg_tol=1e-7, cg_maxit=1000,
                 jacobi_steps=3):
        self.csr, self.cells = csr, cells
        self.s = _Sim()
        if isinstance(cells, MixedCells):
            L = lib()
            fn = C.cast(L.epo_mixed_ionic_cb, C.c_void_p)
            ctx = C.cast(C.pointer(cells.m), C.c_void_p)
            self._L = L
        elif isinstance(cells, RefCells):
            L = ref_lib()
            fn = C.cast(L.ref_cells_ionic_cb, C.c_void_p)
            ctx = C.c_void_p(cells.h)
            self._L = L
        else:
            L = lib()
            fn = C.cast(L.epo_cells_ionic_cb, C.c_void_p)
            ctx = C.cast(cells.h, C.c_void_p)
            self._L = L
        self._L.epo_sim_init(C.byref(self.s), C.byref(csr.c), dt, ionic_dt, Cm, cg_tol,
                             cg_maxit, jacobi_steps, fn, ctx)
        self.n = csr.n

    def set_scheme(self, scheme, dt_diff=0.05):
        """EPO_SCHEME_BE (1) or EPO_SCHEME_EXPLICIT (2); the cells then move by
        the reference's per-node ionic strides."""
        if isinstance(self.cells, RefCells):
            fn = C.cast(ref_lib().ref_cells_ionic_node_cb, C.c_void_p)
            ctx = C.c_void_p(self.cells.h)
        else:
            fn = C.cast(lib().epo_cells_ionic_node_cb, C.c_void_p)
            ctx = C.cast(self.cells.h, C.c_void_p)
        self._L.epo_sim_set_scheme(C.byref(self.s), int(scheme), float(dt_diff), fn, ctx)

    @property
    def V(self):
        return np.ctypeslib.as_array(self.s.V, shape=(self.n,))

    @property
    def istim(self):
        return np.ctypeslib.as_array(self.s.istim, shape=(self.n,))

    @property
    def sub_dt(self):
        return [self.s.sub_dt[i] for i in range(self.s.nsub)]

    def step(self, k=1):
        for _ in range(k):
            self._L.epo_sim_step(C.byref(self.s))

    def __del__(self):
        try:
            self._L.epo_sim_free(C.byref(self.s))
        except Exception:
            pass
