"""The library's host-side FP64 assembly (ep_assemble_operators, the code
ep_create runs before it uploads the operators) against the oracle's
restatement of TetMesh::Compute / MixedMesh3D::Compute / CardiacBody::Compute
/ EP_CrankNicholson::Initialize.  No GPU: the entry point never touches the
device."""
import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M, simulation as S


@pytest.fixture(scope="module")
def slab():
    return M.slab(9, 7, 4, 0.8, 0.6, 0.3)


def _close(a, b, rtol=0.0):
    a, b = a.tocsr(), b.tocsr()
    return abs(a - b).max() <= rtol * max(1.0, abs(b).max())


def test_tets_crank_nicolson_equal_the_oracle(slab):
    D = M.sigma_to_D(1.2, 0.2)
    for Cm, dt in ((1.0, 0.1), (1.7, 0.02)):
        A, B, CL = S.assemble_operators(slab, D, dt, Cm=Cm)
        o = O.Csr(slab.xyz, slab.tets, slab.fibers, D, Cm, dt)
        assert _close(A, o.scipy("A")) and _close(B, o.scipy("B"))
        assert np.array_equal(CL, o.arr("CL"))


def test_other_schemes_from_the_same_element_matrices(slab):
    """Backward Euler: A = C_L + dt/2 K, B = diag C_L; explicit: A = -K."""
    D = M.sigma_to_D(1.2, 0.2)
    dt = 0.05
    o = O.Csr(slab.xyz, slab.tets, slab.fibers, D, 1.0, dt)
    K, CL = o.scipy("K"), o.arr("CL")
    import scipy.sparse as sp
    A, B, _ = S.assemble_operators(slab, D, dt, scheme=capi.SCHEME_BE)
    assert _close(A, sp.diags(CL) + dt / 2 * K, rtol=1e-13)
    assert np.allclose(B.diagonal(), CL, rtol=1e-15)
    assert abs(B - sp.diags(B.diagonal())).max() == 0.0
    A, _, _ = S.assemble_operators(slab, D, dt, scheme=capi.SCHEME_EXPLICIT)
    assert _close(A, -K, rtol=1e-14)


def _mixed(slab):
    """The slab plus a Purkinje cable: two bars on slab nodes, two reaching
    out to nodes that belong to no tet."""
    n0 = slab.n
    extra = slab.xyz[[0]] + np.array([[0.0, 0.0, -0.05], [0.0, 0.0, -0.1]])
    mesh = M.TetMesh(np.vstack([slab.xyz, extra]), slab.tets, slab.fibers, {})
    bars = np.array([[1, 0], [0, 9], [0, n0], [n0, n0 + 1]])
    rng = np.random.default_rng(3)
    fib = np.zeros((len(bars), 9))
    for e in range(len(bars)):          # an orthonormal frame per bar
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        fib[e] = q.T.reshape(-1)
    return mesh, bars, fib


@pytest.mark.parametrize("with_fibres", [False, True])
def test_mixed_mesh_with_cables_equals_the_oracle(slab, with_fibres):
    mesh, bars, fib = _mixed(slab)
    D = M.sigma_to_D(1.2, 0.2)
    lv = np.array([0, 1, 0, 1], np.uint8)
    kw = dict(Dp=(0.0016, 0.0008, 0.0004), DpLeft=(0.003, 0.001, 0.0005), radius=0.02)
    A, B, CL = S.assemble_operators(mesh, D, 0.1, bars=bars, lv=lv, bar_fibers=fib if with_fibres else None, **kw)
    cb = O.Cables(bars, lv=lv, fibers=fib if with_fibres else None, **kw)
    o = O.Csr(mesh.xyz, mesh.tets, mesh.fibers, D, 1.0, 0.1, cables=cb)
    assert _close(A, o.scipy("A"), rtol=1e-15) and _close(B, o.scipy("B"), rtol=1e-15)
    assert np.allclose(CL, o.arr("CL"), rtol=1e-15, atol=0)
    assert CL[-1] > 0 and A[mesh.n - 1, mesh.n - 2] != 0.0        # the cable-only nodes are coupled


@pytest.mark.parametrize("sticky", [True, False])
def test_angle_override_equals_the_oracle(slab, sticky):
    mesh, bars, _ = _mixed(slab)
    angle = {0: (0.0, 0.0, -1.0, 0.07)}
    A, _, _ = S.assemble_operators(mesh, (1e-3,) * 3, 0.1, bars=bars, angle=angle, angle_sticky=sticky)
    cb = O.Cables(bars, orient=angle, sticky=sticky, n=mesh.n)
    o = O.Csr(mesh.xyz, mesh.tets, None, (1e-3,) * 3, 1.0, 0.1, cables=cb)
    assert _close(A, o.scipy("A"), rtol=1e-15)


def test_bad_input_is_an_error_not_a_crash(slab):
    mesh, bars, _ = _mixed(slab)
    with pytest.raises(capi.EPError):
        S.assemble_operators(mesh, (1e-3,) * 3, 0.1, bars=np.array([[0, mesh.n]]))
    with pytest.raises(capi.EPError):                       # zero-length cable
        S.assemble_operators(mesh, (1e-3,) * 3, 0.1, bars=np.array([[3, 3]]))
    with pytest.raises(capi.EPError):
        S.assemble_operators(mesh, (1e-3,) * 3, 0.1, bars=bars, quad_order=5)
