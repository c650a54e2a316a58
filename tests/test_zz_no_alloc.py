"""The allocation-free half diffusion step (ep_cn_half_step_noalloc).

It serves callers that own all device memory and may not allocate (a solver
embedded in another code's memory pool, a time loop that must not call
cudaMalloc after start-up, a C/Fortran host handing over its own buffers).
Here the test plays such a caller: it builds the SELL-32 operators of a shell
from the CPU oracle's assembly, places them in device memory it owns (torch
tensors), and calls the entry point through the C ABI twice in a row.  Each
result must match the handle-based entry point (ep_diffusion_half_step on the
same mesh) within the tolerance the other CG tests use.

The file is named so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi, mesh as M, workloads as W
from ucla_cmg_b200.simulation import Monodomain


def _sell(csr, S=32):
    """SELL-32 packing of the oracle CSR (A and B share the columns): row r
    sits in slice r // 32, lane r % 32, its j-th entry at slice_ptr + 32 j +
    lane; padding entries point at the row itself with value 0."""
    rp, col = csr.arr("rowptr"), csr.arr("col")
    A, B = csr.arr("A"), csr.arr("B")
    n = csr.n
    ns = (n + S - 1) // S
    lens = np.diff(rp)
    lp = np.zeros(ns * S, np.int64)
    lp[:n] = lens
    width = lp.reshape(ns, S).max(axis=1)
    sp = np.concatenate([[0], np.cumsum(width * S)]).astype(np.int64)
    pos = np.arange(sp[-1])
    sl = np.repeat(np.arange(ns), width * S)
    row = sl * S + (pos - sp[sl]) % S
    c = np.minimum(row, n - 1).astype(np.int32)
    a = np.zeros(sp[-1])
    b = np.zeros(sp[-1])
    r = np.repeat(np.arange(n), lens)
    k = sp[r // S] + (np.arange(len(col)) - rp[r]) * S + r % S
    c[k] = col
    a[k] = A
    b[k] = B
    dinv = 1.0 / csr.scipy("A").diagonal()
    return ns, sp.astype(np.int32), c, a, b, dinv


@pytest.fixture(scope="module")
def case():
    wl = W.shell_c2(h=0.2)
    m = wl.mesh
    rng = np.random.default_rng(11)
    V = -85.0 + 120.0 * (m.xyz[:, 2] < -3.0) + rng.normal(0, 1.0, m.n)
    csr = O.Csr(m.xyz, m.tets, m.fibers, wl.D, 1.0, wl.dt)
    return wl, V, _sell(csr)


@pytest.fixture(scope="module")
def case_max():
    """A 64 x 64 x 64 slab: 262,144 rows, the entry point's limit, so every
    FP64 vector, the partial slots and the tail of the array are in use."""
    m = M.slab(64, 64, 64, 1.26, 1.26, 1.26)
    D = M.sigma_to_D(1.2, 0.2)
    assert m.n == 262144
    rng = np.random.default_rng(12)
    V = -85.0 + 120.0 * (m.xyz[:, 0] < 0.3) + rng.normal(0, 1.0, m.n)
    csr = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, 0.1)
    wl = W.Workload("slab_max", m, capi.TUSSCHER, 0.1, 0.02, 0.0, D, None, None, None, None, None, None)
    return wl, V, _sell(csr)


def test_sell_packing_reproduces_the_csr_product():
    """The packer itself, on the CPU: SELL-32 A x equals the CSR A x."""
    m = M.slab(7, 5, 4, 0.3, 0.2, 0.15)
    csr = O.Csr(m.xyz, m.tets, m.fibers, (1e-3, 2e-4, 2e-4), 1.0, 0.1)
    ns, sp, c, a, b, dinv = _sell(csr)
    x = np.random.default_rng(0).normal(size=m.n)
    y = np.zeros(ns * 32)
    for s in range(ns):
        w = (sp[s + 1] - sp[s]) // 32
        for j in range(w):
            idx = sp[s] + 32 * j + np.arange(32)
            y[s * 32:(s + 1) * 32] += a[idx] * x[c[idx]]
    assert np.allclose(y[:m.n], csr.scipy("A") @ x, rtol=1e-14, atol=1e-14)
    assert np.allclose(dinv * csr.scipy("A").diagonal(), 1.0)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("which", ["shell", "max_rows"])
@pytest.mark.gpu
def test_noalloc_matches_handle_path(gpu, case, case_max, which, prec):
    import torch
    wl, V, (ns, sp, c, a, b, dinv) = case if which == "shell" else case_max
    n = wl.mesh.n
    # the existing entry point on the same mesh
    g = Monodomain(wl.mesh, capi.TUSSCHER, prec, dt=wl.dt, ionic_dt=wl.ionic_dt, D=wl.D, cg_tol=1e-7)
    g.set_voltage(V)
    it_ref, _ = g.diffusion_half_step()
    x_ref = g.voltage()
    g.close()
    # the caller's own device buffers
    dt = torch.float64 if prec == capi.FP64 else torch.float32
    dev = torch.device("cuda", 0)
    t_sp = torch.from_numpy(sp).to(dev)
    t_c = torch.from_numpy(c).to(dev)
    t_a = torch.from_numpy(a).to(dev, dt)
    t_b = torch.from_numpy(b).to(dev, dt)
    t_d = torch.from_numpy(dinv).to(dev, dt)
    L = capi.lib()
    outs = []
    for call in range(2):
        x = torch.from_numpy(V).to(dev, dt).contiguous()
        torch.cuda.synchronize()
        it = C.c_int32(0)
        rr = C.c_double(0)
        rc = L.ep_cn_half_step_noalloc(prec, n, ns, t_sp.data_ptr(), t_c.data_ptr(), t_a.data_ptr(),
                                       t_b.data_ptr(), t_d.data_ptr(), x.data_ptr(), 1e-7, 1000, None,
                                       C.byref(it), C.byref(rr))
        assert rc == 0, L.ep_last_error()
        outs.append((x.double().cpu().numpy(), it.value))
    scale = np.max(np.abs(x_ref))
    tol = 1e-6 if prec == capi.FP64 else 1e-4
    for x, it in outs:
        assert np.max(np.abs(x - x_ref)) <= tol * scale
        assert abs(it - it_ref) <= 1
    # the second call reuses the shared array and reproduces the first
    assert np.array_equal(outs[0][0], outs[1][0]) and outs[0][1] == outs[1][1]


@pytest.mark.gpu
def test_noalloc_rejects_oversize(gpu):
    L = capi.lib()
    n = 262145
    rc = L.ep_cn_half_step_noalloc(capi.FP32, n, (n + 31) // 32, 1, 1, 1, 1, 1, 1, 1e-7, 10, None,
                                   None, None)
    assert rc == -1
    assert b"262144" in L.ep_last_error()


@pytest.mark.gpu
def test_noalloc_leaves_a_capture_intact(gpu, case):
    """Called on a stream that is being captured, the entry point returns
    EP_ERR_ARG before it touches the stream (it waits for its own results,
    which a capture cannot do), and the caller's capture stays usable."""
    import torch
    wl, V, (ns, sp, c, a, b, dinv) = case
    dev = torch.device("cuda", 0)
    bufs = [torch.from_numpy(v).to(dev) for v in (sp, c, a, b, dinv, V)]
    L = capi.lib()
    x = torch.arange(8, device=dev, dtype=torch.float64)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        y = x * 2.0
        rc = L.ep_cn_half_step_noalloc(capi.FP64, wl.mesh.n, ns, *(t.data_ptr() for t in bufs[:5]),
                                       bufs[5].data_ptr(), 1e-7, 1000,
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream), None, None)
    assert rc == -1 and b"captured" in L.ep_last_error()
    x.fill_(3.0)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.all(y == 6.0)
