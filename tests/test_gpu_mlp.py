"""GPU trainer kernels (ep_mlp_*) and the BF16 tensor-core inference kernel
vs the FP64 numpy network in oracle/mlp_oracle.py."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO
from ucla_cmg_b200 import surrogate as SG

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_gradients_match_oracle(gpu):
    dims = [23, 16, 16, 7]
    tr = SG.Trainer(dims, seed=3)
    p = tr.params().astype(np.float64)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(300, 23))
    Y = rng.normal(size=(300, 7))
    w = np.linspace(0.5, 2.0, 7)
    Xd, Yd = _dev(X), _dev(Y)
    loss, g = tr.loss_grad(Xd.data_ptr(), Yd.data_ptr(), 300, w, want_grad=True)
    loss_o, g_o = MO.loss_grad(p, dims, X.astype(np.float32).astype(np.float64),
                               Y.astype(np.float32).astype(np.float64), w)
    assert abs(loss - loss_o) <= 1e-5 * abs(loss_o)
    assert np.max(np.abs(g - g_o)) <= 1e-4 * np.max(np.abs(g_o))
    # forward
    import torch
    out = torch.empty((300, 7), device="cuda")
    tr.forward(Xd.data_ptr(), out.data_ptr(), 300)
    f_o, _ = MO.forward(p, dims, X.astype(np.float32).astype(np.float64))
    assert np.max(np.abs(out.cpu().numpy() - f_o)) < 1e-5 * max(1.0, np.abs(f_o).max())
    tr.close()


def test_adam_fits_a_smooth_map(gpu):
    dims = [23, 32, 32, 4]
    tr = SG.Trainer(dims, seed=1)
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, size=(4096, 23))
    Y = np.stack([np.sin(X[:, 0]), X[:, 1] * X[:, 2], np.tanh(X[:, 3] + X[:, 4]), X[:, 5] ** 2], axis=1)
    Xd, Yd = _dev(X), _dev(Y)
    l0, _ = tr.loss_grad(Xd.data_ptr(), Yd.data_ptr(), 4096)
    for _ in range(400):
        tr.loss_grad(Xd.data_ptr(), Yd.data_ptr(), 4096)
        tr.adam(3e-3)
    l1, _ = tr.loss_grad(Xd.data_ptr(), Yd.data_ptr(), 4096)
    assert l1 < 0.05 * l0
    tr.close()


def test_tensor_core_inference_matches_bf16_reference(gpu):
    """The tcgen05 kernel (BF16 operands, FP32 accumulation in TMEM) against
    the same network evaluated in FP64 with BF16-rounded weights and
    activations; 1000 rows (tail tile included)."""
    tr = SG.Trainer(SG.DIMS, seed=7)
    p = tr.params()
    tr.close()
    rng = np.random.default_rng(4)
    # larger weights than the Xavier init so the tanh layers are not linear
    p = (p * 2.0).astype(np.float32)
    n = 1000
    Xn = rng.normal(size=(n, 23)).astype(np.float32)
    s = SG.Surrogate(p, np.zeros(23, np.float32), np.ones(23, np.float32), np.zeros(19, np.float32),
                     np.ones(19, np.float32), np.full(23, -1e30, np.float32), np.full(23, 1e30, np.float32))
    Y = s.forward_kernel(Xn)
    ref, _ = MO.forward(p.astype(np.float64), SG.DIMS, Xn.astype(np.float64), bf16=True)
    ref32, _ = MO.forward(p.astype(np.float64), SG.DIMS, Xn.astype(np.float64))
    scale = np.abs(ref).max()
    err = np.abs(Y - ref).max() / scale
    # tanh.approx (~2^-11 relative) and BF16 activation rounding
    assert err < 2e-2, err
    assert np.abs(Y - ref32).max() / scale < 5e-2
    assert np.all(np.isfinite(Y))
