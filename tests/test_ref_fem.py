"""The FEM and pseudo-ECG rows pinned to the reference's own code.

The reference's mesh reader (Mesh::New), tet and cable geometry
(TetMesh::Compute, MixedMesh3D::Compute), element assembly
(CardiacBody::Compute, getDiffusionMatrix, getCapacitanceMatrix,
computeLumpedCapacitance) and pseudo-ECG (ComputeECG.h) are compiled
unmodified into oracle/_ref/libvoomep_fem.so against stand-in headers for
tvmet, Blitz++, Epetra and MPI.  Here they read mesh files in the
reference's formats and their results are compared with

* the oracle's C restatement (oracle/ep_oracle.c), and
* the library's own host assembly (ep_assemble_operators, the operators
  ep_create uploads), which needs no GPU.

The CN operators follow EP_CrankNicholson::Initialize (EP_CrankNicholson.cc:
15-29): A = getDiffusionMatrix(dt/4) + getCapacitanceMatrix(), B the same
with -dt/4.  Tolerances are rounding-level (the reference and the
restatement add the element contributions in different orders)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M, simulation as S

pytestmark = pytest.mark.skipif(O.ref_fem_lib() is None, reason="oracle/_ref/libvoomep_fem.so not built")

RTOL = 1e-13


def _rel(a, b):
    a, b = a.tocsr(), b.tocsr()
    return abs(a - b).max() / abs(b).max()


def _ref(tmp_path, name, xyz, elements, fibers, **kw):
    base = os.path.join(str(tmp_path), name)
    O.write_reference_case(base, xyz, elements, fibers, **kw)
    return base


def _check_tets(tmp_path, name, mesh, D, Cm, dt, fibers=True):
    fib = mesh.fibers if fibers else None
    base = _ref(tmp_path, name, mesh.xyz, mesh.tets, fib)
    rm = O.RefFemMesh(base)
    assert rm.n == mesh.n and rm.n_elements == mesh.m
    rb = O.RefFemBody(rm, O.TUSSCHER, D, Cm)
    K, Mc, CL = rb.diffusion(1.0), rb.capacitance(True), rb.lumped()
    A = rb.diffusion(dt / 4.0) + rb.capacitance(True)
    B = rb.diffusion(-dt / 4.0) + rb.capacitance(True)
    o = O.Csr(mesh.xyz, mesh.tets, fib, D, Cm, dt)
    # the restatement
    assert _rel(o.scipy("K"), K) <= RTOL
    assert _rel(o.scipy("M") * Cm, Mc) <= RTOL
    assert np.max(np.abs(o.arr("CL") - CL)) <= RTOL * np.max(CL)
    assert _rel(o.scipy("A"), A) <= RTOL and _rel(o.scipy("B"), B) <= RTOL
    # the library's host assembly (what ep_create uploads)
    mm = M.TetMesh(mesh.xyz, mesh.tets, fib, {})
    Al, Bl, CLl = S.assemble_operators(mm, D, dt, Cm=Cm)
    assert _rel(Al, A) <= RTOL and _rel(Bl, B) <= RTOL
    assert np.max(np.abs(CLl - CL)) <= RTOL * np.max(CL)
    return rm


def test_slab_operators_equal_the_reference(tmp_path):
    """A Kuhn-split slab with the fibre rotation of the slab workloads."""
    m = M.slab(9, 7, 5, 0.8, 0.6, 0.4)
    _check_tets(tmp_path, "slab", m, M.sigma_to_D(1.2, 0.2), 1.0, 0.02)


def test_shell_operators_equal_the_reference(tmp_path):
    """Curved prism-split tets with helical fibres (the shell workload's
    element shapes), C_m != 1, the shell's step."""
    m = M.shell(h=0.5, n_rho=3)
    _check_tets(tmp_path, "shell", m, M.sigma_to_D(1.2, 0.2), 1.3, 0.1)


def test_isotropic_operators_equal_the_reference(tmp_path):
    """No .fibers file: the reference uses D[0] times the identity
    (CardiacBody.cc:115-168)."""
    m = M.slab(6, 5, 4, 0.5, 0.4, 0.3)
    _check_tets(tmp_path, "iso", m, (1e-3, 5e-4, 2.5e-4), 1.0, 0.05, fibers=False)


@pytest.mark.parametrize("name", ["slab", "shell"])
def test_ecg_equals_the_reference(tmp_path, name):
    """ComputeECG.h's chain (diffusion tensor, grad(1/r), grad V per
    quadrature point, quadrature sum) against the restatement element by
    element and through its per-node weights, for a voltage field with a
    wavefront, including an electrode close to the mesh."""
    m = M.slab(9, 7, 5, 0.8, 0.6, 0.4) if name == "slab" else M.shell(h=0.5, n_rho=3)
    D = (1e-3, 5e-4, 2.5e-4)
    base = _ref(tmp_path, name, m.xyz, m.tets, m.fibers)
    rm = O.RefFemMesh(base, compute=True)
    rng = np.random.default_rng(4)
    c = m.xyz.mean(axis=0)
    el = np.vstack([M.fibonacci_sphere(6, 15.0, c), c + [0.0, 0.0, 2.0], m.xyz[0] + [0.0, 0.0, -0.05]])
    V = np.where(m.xyz[:, 0] < c[0], 20.0, -85.0) + rng.normal(0.0, 1.0, m.n)
    e_ref = rm.ecg(D, el, V)
    e_el = O.ecg_elementwise(m.xyz, m.tets, m.fibers, D, el, V)
    e_w = O.ecg_weights(m.xyz, m.tets, m.fibers, D, el) @ V
    scale = np.max(np.abs(e_ref))
    assert np.max(np.abs(e_el - e_ref)) <= 1e-12 * scale
    assert np.max(np.abs(e_w - e_ref)) <= 1e-12 * scale


def _mixed_case(tmp_path, sticky_angle):
    """A slab plus a Purkinje cable: bars joining slab nodes, and bars that
    leave the slab to nodes of no tet; .purk lists the cable nodes, .cell
    marks some of them RV (12; the others stay LV, 11), .angle overrides
    the direction and length of the cable that starts at one node."""
    slab = M.slab(6, 5, 4, 0.5, 0.4, 0.3)
    n0 = slab.n
    extra = slab.xyz[[0]] + np.array([[0.0, 0.0, -0.05], [0.0, 0.0, -0.1], [0.03, 0.0, -0.12]])
    xyz = np.vstack([slab.xyz, extra])
    bars = np.array([[1, 0], [0, n0], [n0, n0 + 1], [n0 + 1, n0 + 2], [6, 7]])
    elements = [list(t) for t in slab.tets[:40]] + [list(b) for b in bars[:3]] + \
               [list(t) for t in slab.tets[40:]] + [list(b) for b in bars[3:]]
    rng = np.random.default_rng(3)
    fib = np.zeros((len(elements), 9))
    tet_fib = iter(slab.fibers)
    bar_fib = []
    for e, el in enumerate(elements):
        if len(el) == 4:
            fib[e] = next(tet_fib)
        else:
            q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            fib[e] = q.T.reshape(-1)
            bar_fib.append(fib[e])
    purk = np.array([0, 1, 6, 7, n0, n0 + 1, n0 + 2])
    node_type = np.zeros(len(xyz), np.int64)
    node_type[purk] = 11
    node_type[[6, 7]] = 12
    angle = {n0: (0.0, 0.0, -1.0, 0.07)} if sticky_angle is not None else None
    base = _ref(tmp_path, "mix", xyz, elements, fib, purk=purk, cell=node_type, angle=angle)
    bars_in_order = np.array([el for el in elements if len(el) == 2])
    lv = ((node_type[bars_in_order[:, 0]] == 11) | (node_type[bars_in_order[:, 1]] == 11)).astype(np.uint8)
    return base, xyz, slab, bars_in_order, np.array(bar_fib), lv, angle


@pytest.mark.parametrize("with_angle", [False, True])
def test_mixed_mesh_operators_equal_the_reference(tmp_path, with_angle):
    """MIX3D: tets and 2-node cables in one .ele file.  The cables get
    DpLeft where either node is LV (tissue type 11) and Dp elsewhere
    (CardiacBody.cc:100-135), the bar quadrature of MixedMesh3D::Compute
    with its doubled weights (MixedMesh3D.cc:107) and the .angle override
    that stays on once met (MixedMesh3D.cc:14-34)."""
    base, xyz, slab, bars, bar_fib, lv, angle = _mixed_case(tmp_path, True if with_angle else None)
    D = M.sigma_to_D(1.2, 0.2)
    Dp, DpLeft, radius, dt = (0.0016, 0.0008, 0.0004), (0.003, 0.001, 0.0005), 0.0275, 0.1
    rm = O.RefFemMesh(base, mixed=True, radius=radius)
    rb = O.RefFemBody(rm, O.TUSSCHER, D, 1.0, Dp=Dp, DpLeft=DpLeft)
    A = rb.diffusion(dt / 4.0) + rb.capacitance(True)
    B = rb.diffusion(-dt / 4.0) + rb.capacitance(True)
    CL = rb.lumped()
    kw = dict(Dp=Dp, DpLeft=DpLeft, radius=radius)
    cb = O.Cables(bars, fibers=bar_fib, lv=lv, orient=angle, sticky=True, n=len(xyz), **kw)
    o = O.Csr(xyz, slab.tets, slab.fibers, D, 1.0, dt, cables=cb)
    assert _rel(o.scipy("A"), A) <= RTOL and _rel(o.scipy("B"), B) <= RTOL
    assert np.max(np.abs(o.arr("CL") - CL)) <= RTOL * np.max(CL)
    mm = M.TetMesh(xyz, slab.tets, slab.fibers, {})
    Al, Bl, CLl = S.assemble_operators(mm, D, dt, bars=bars, lv=lv, bar_fibers=bar_fib, angle=angle or {},
                                       angle_sticky=True, **kw)
    assert _rel(Al, A) <= RTOL and _rel(Bl, B) <= RTOL
    assert np.max(np.abs(CLl - CL)) <= RTOL * np.max(CL)
    assert CL[-1] > 0.0                                   # the cable-only nodes carry mass


def test_reference_reads_the_files_the_library_writes(tmp_path):
    """The library's mesh writer (voomep_io.write_mesh) produces files the
    reference's Mesh::New reads into the same operators."""
    from ucla_cmg_b200 import voomep_io as IO
    m = M.slab(5, 4, 3, 0.4, 0.3, 0.2)
    base = os.path.join(str(tmp_path), "w")
    IO.write_mesh(base, m)
    with open(base + ".metis.npart.1", "w") as f:
        f.write("0\n" * m.n)
    with open(base + ".metis.epart.1", "w") as f:
        f.write("0\n" * m.m)
    rm = O.RefFemMesh(base)
    rb = O.RefFemBody(rm, O.TUSSCHER, (1e-3, 2e-4, 2e-4), 1.0)
    o = O.Csr(m.xyz, m.tets, m.fibers, (1e-3, 2e-4, 2e-4), 1.0, 0.1)
    assert _rel(o.scipy("K"), rb.diffusion(1.0)) <= RTOL


@pytest.mark.parametrize("sticky_from", ["tet", "cable"])
def test_angle_override_switched_on_by_any_element(tmp_path, sticky_from):
    """MixedMesh3D::Compute tests the first node of EVERY element against the
    .angle list (MixedMesh3D.cc:30-34): a tet whose first node is listed
    switches the override on for the cables after it, though no cable starts
    there.  The library's MIX3D reader resolves the override per cable over
    the .ele order (voomep_io.read_cables), and the restatement and the host
    assembly then equal the reference's operators."""
    from ucla_cmg_b200 import voomep_io as IO
    slab = M.slab(6, 5, 4, 0.5, 0.4, 0.3)
    n0 = slab.n
    extra = slab.xyz[[0]] + np.array([[0.0, 0.0, -0.05], [0.0, 0.0, -0.1], [0.02, 0.0, -0.14]])
    xyz = np.vstack([slab.xyz, extra])
    bars = [[n0, n0 + 1], [n0 + 1, n0 + 2]]
    t0 = int(slab.tets[7][0])
    listed = t0 if sticky_from == "tet" else n0 + 1
    elements = [list(t) for t in slab.tets[:20]] + [bars[0]] + [list(t) for t in slab.tets[20:]] + [bars[1]]
    angle = {listed: (0.0, 0.6, -0.8, 0.07)}
    purk = np.array([n0, n0 + 1, n0 + 2])
    node_type = np.zeros(len(xyz), np.int64)
    node_type[purk] = 11
    base = _ref(tmp_path, "mixa", xyz, elements, None, purk=purk, cell=node_type, angle=angle)
    D, Dp, radius, dt = (1e-3,) * 3, (0.0016,) * 3, 0.0275, 0.1
    rm = O.RefFemMesh(base, mixed=True, radius=radius)
    rb = O.RefFemBody(rm, O.TUSSCHER, D, 1.0, Dp=Dp, DpLeft=Dp)
    A = rb.diffusion(dt / 4.0) + rb.capacitance(True)
    cab = IO.read_cables(base, node_type)
    expect = [listed, listed] if sticky_from == "tet" else [-1, listed]
    assert cab["angle_node"].tolist() == expect
    cb = O.Cables(cab["bars"], Dp=Dp, DpLeft=Dp, radius=radius, lv=cab["lv"], orient=cab["angle"], n=len(xyz),
                  bar_orient_node=cab["angle_node"])
    o = O.Csr(xyz, slab.tets, None, D, 1.0, dt, cables=cb)
    assert _rel(o.scipy("A"), A) <= RTOL
    mm = M.TetMesh(xyz, slab.tets, None, {})
    Al, _, _ = S.assemble_operators(mm, D, dt, bars=cab["bars"], lv=cab["lv"], angle=cab["angle"], Dp=Dp,
                                    DpLeft=Dp, radius=radius, bar_angle_node=cab["angle_node"])
    assert _rel(Al, A) <= RTOL
    if sticky_from == "tet":
        # the bars-only rule (no cable starts at a listed node) misses it
        Ab, _, _ = S.assemble_operators(mm, D, dt, bars=cab["bars"], lv=cab["lv"], angle=cab["angle"], Dp=Dp,
                                        DpLeft=Dp, radius=radius)
        assert _rel(Ab, A) > 1e-6


@pytest.mark.parametrize("with_fibres", [False, True])
def test_mixed_mesh_ecg_equals_the_reference(tmp_path, with_fibres):
    """ComputeECG on a MIX3D mesh integrates over the cables too, with the
    tissue D along each cable's fibre frame (computeDiffusionTensor applies
    Diff to every element) and the radius ComputeECG fixes at 0.0275 cm; the
    .angle override sets the cables' derivative and weight.  The
    restatement's per-node weights (tets + cables) against the reference's
    chain on a field with a front."""
    from ucla_cmg_b200 import voomep_io as IO
    base, xyz, slab, bars, bar_fib, lv, angle = _mixed_case(tmp_path, True)
    if not with_fibres:
        os.remove(base + ".fibers")
    D = (1e-3, 5e-4, 2.5e-4)
    rm = O.RefFemMesh(base, mixed=True, radius=0.0275, compute=True)
    rng = np.random.default_rng(6)
    c = xyz.mean(axis=0)
    el = np.vstack([M.fibonacci_sphere(5, 12.0, c), xyz[-1] + [0.02, 0.0, -0.03]])
    V = np.where(xyz[:, 2] < c[2], 15.0, -80.0) + rng.normal(0.0, 2.0, len(xyz))
    e_ref = rm.ecg(D, el, V)
    cab = IO.read_cables(base, np.zeros(len(xyz), np.int64))
    cb = O.Cables(cab["bars"], fibers=cab["fibers"], radius=0.0275, orient=cab["angle"], n=len(xyz),
                  bar_orient_node=cab["angle_node"])
    W = O.ecg_weights(xyz, slab.tets, slab.fibers if with_fibres else None, D, el, cables=cb)
    assert np.max(np.abs(W @ V - e_ref)) <= 1e-12 * np.max(np.abs(e_ref))
    # without the cables' share the sums differ: the cables carry signal
    W0 = O.ecg_weights(xyz, slab.tets, slab.fibers if with_fibres else None, D, el)
    assert np.max(np.abs(W0 @ V - e_ref)) > 1e-9 * np.max(np.abs(e_ref))
