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
from ucla_cmg_b200 import capi, workloads as W
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


def _sell(csr, S=32):
    """SELL-32 packing of the oracle CSR (A and B share the columns)."""
    rp, col = csr.arr("rowptr"), csr.arr("col")
    A, B = csr.arr("A"), csr.arr("B")
    n = csr.n
    ns = (n + S - 1) // S
    lens = np.diff(rp)
    width = np.array([lens[s * S:(s + 1) * S].max() for s in range(ns)])
    sp = np.concatenate([[0], np.cumsum(width * S)]).astype(np.int32)
    c = np.zeros(sp[-1], np.int32)
    a = np.zeros(sp[-1])
    b = np.zeros(sp[-1])
    for s in range(ns):
        for lane in range(S):
            r = s * S + lane
            rr = min(r, n - 1)
            ln = lens[r] if r < n else 0
            idx = sp[s] + np.arange(width[s]) * S + lane
            c[idx] = rr
            c[idx[:ln]] = col[rp[r]:rp[r] + ln]
            a[idx[:ln]] = A[rp[r]:rp[r] + ln]
            b[idx[:ln]] = B[rp[r]:rp[r] + ln]
    dinv = 1.0 / csr.scipy("A").diagonal()
    return ns, sp, c, a, b, dinv


@pytest.fixture(scope="module")
def case():
    wl = W.shell_c2(h=0.2)
    m = wl.mesh
    rng = np.random.default_rng(11)
    V = -85.0 + 120.0 * (m.xyz[:, 2] < -3.0) + rng.normal(0, 1.0, m.n)
    csr = O.Csr(m.xyz, m.tets, m.fibers, wl.D, 1.0, wl.dt)
    return wl, V, _sell(csr)


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_noalloc_matches_handle_path(gpu, case, prec):
    import torch
    wl, V, (ns, sp, c, a, b, dinv) = case
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


def test_noalloc_rejects_oversize(gpu):
    L = capi.lib()
    n = 262145
    rc = L.ep_cn_half_step_noalloc(capi.FP32, n, (n + 31) // 32, 1, 1, 1, 1, 1, 1, 1e-7, 10, None,
                                   None, None)
    assert rc == -1
    assert b"262144" in L.ep_last_error()
