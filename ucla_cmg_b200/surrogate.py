"""The learned ionic step: data from the plain model, GPU training, packaging.

The network maps the state of one ten Tusscher node at the start of a global
step (V, the 18 stored states, I_stim, and the node's G_Ks, G_to and s-gate
variant) to the change of V and of the 18 states over that step's ionic phase
(dt = 0.1 ms = 5 sub-steps of 0.02 ms), i.e. it replaces the sub-step loop of
EP_CrankNicholson::Solve (voomEP/src/Solvers/EP_CrankNicholson.cc:114-143)
for one node.  Shape 23 -> 128 -> 128 -> 128 -> 19, tanh.

* :func:`generate` runs plain-model tissue simulations on slabs with
  randomised stimuli and cell parameters, snapshots node states, and computes
  the targets with the plain FP64 ionic phase (``ep_ionic_phase``).  Only
  states inside the learned domain are kept: no active stimulus and a fast
  sodium gate product m^3 h <= ``NAH_MAX`` (the upstroke stays with the
  plain model).
* :func:`train` fits the network on the GPU with the project's own kernels
  (``ep_mlp_*``: FP32 forward, backward and Adam).
* :class:`Surrogate` holds the weights, normalisation and the training
  envelope (per-feature box), and deploys them with ``ep_set_surrogate``
  (BF16 tensor-core inference, per-node fallback to the plain model).
"""
import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import capi, mesh as M
from .capi import check, ptr

DIMS = [23, 128, 128, 128, 19]
NAH_MAX = 2e-4
# states spanning decades (Cai, Xr1, Xs, m, h, j, Cass, d, s, r) enter as
# logarithms and are updated multiplicatively
LOG_FEATURES = (3, 4, 6, 7, 8, 9, 10, 11, 15, 16)
LOG_MASK = sum(1 << k for k in LOG_FEATURES)
# outputs the hybrid form uses: the Newton concentrations Ki, Nai, Cai, Cass,
# CaSR, R' (stored states 1, 2, 3, 10, 17, 18)
CONC_OUTPUTS = (1, 2, 3, 10, 17, 18)
_LOG = np.zeros(23, bool)
_LOG[list(LOG_FEATURES)] = True


def transform(X):
    """Raw features -> the network's input space (log of the wide-range ones)."""
    Xt = np.array(X, dtype=np.float64, copy=True)
    Xt[:, _LOG] = np.log(np.maximum(Xt[:, _LOG], 1e-30))
    return Xt


def target_from_delta(S, Y):
    """Linear changes over the step -> targets (change of log for log states)."""
    T = np.array(Y, dtype=np.float64, copy=True)
    lg = _LOG[:19]
    old = np.maximum(S[:, :19][:, lg], 1e-30)
    T[:, lg] = np.log(np.maximum(old + Y[:, lg], 1e-30)) - np.log(old)
    return T
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PATH = os.path.join(HERE, "data", "tt_surrogate.npz")


@dataclass
class Surrogate:
    params: np.ndarray
    in_mean: np.ndarray
    in_std: np.ndarray
    out_mean: np.ndarray
    out_std: np.ndarray
    env_lo: np.ndarray
    env_hi: np.ndarray
    nah_max: float = NAH_MAX
    log_mask: int = LOG_MASK
    v_update: int = 0
    out_scale: np.ndarray = None       # per output s_j > 0: targets are asinh(delta / s_j)
    out_lo: np.ndarray = None          # accepted range of the de-normalised outputs
    out_hi: np.ndarray = None
    hybrid_substeps: int = 1
    meta: dict = field(default_factory=dict)

    def save(self, path=DEFAULT_PATH):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        sc = np.zeros(DIMS[-1], np.float32) if self.out_scale is None else self.out_scale
        big = np.full(DIMS[-1], 3e38, np.float32)
        np.savez_compressed(path, params=self.params, in_mean=self.in_mean, in_std=self.in_std,
                            out_mean=self.out_mean, out_std=self.out_std, env_lo=self.env_lo,
                            env_hi=self.env_hi, nah_max=self.nah_max, log_mask=self.log_mask,
                            v_update=self.v_update, out_scale=sc,
                            out_lo=-big if self.out_lo is None else self.out_lo,
                            out_hi=big if self.out_hi is None else self.out_hi,
                            hybrid_substeps=self.hybrid_substeps,
                            meta=np.array(repr(self.meta)))

    @classmethod
    def load(cls, path=DEFAULT_PATH):
        z = np.load(path, allow_pickle=False)
        f32 = lambda k: z[k].astype(np.float32)
        opt = lambda k: f32(k) if k in z else None
        return cls(f32("params"), f32("in_mean"), f32("in_std"), f32("out_mean"), f32("out_std"),
                   f32("env_lo"), f32("env_hi"), float(z["nah_max"]),
                   int(z["log_mask"]) if "log_mask" in z else 0,
                   int(z["v_update"]) if "v_update" in z else 0,
                   opt("out_scale"), opt("out_lo"), opt("out_hi"),
                   int(z["hybrid_substeps"]) if "hybrid_substeps" in z else 1, {"meta": str(z["meta"])})

    def decode(self, Yn):
        """Network outputs (normalised) -> changes over the step (log changes
        for the log-scaled states)."""
        U = np.asarray(Yn, np.float64) * self.out_std + self.out_mean
        if self.out_scale is not None:
            sc = np.asarray(self.out_scale, np.float64)
            U = np.where(sc > 0, sc * np.sinh(U), U)
        return U

    def desc(self):
        """capi.SurrogateDesc (and the arrays it points to, keep them alive)."""
        keep = [np.ascontiguousarray(a, dtype=np.float32) for a in
                (self.params, self.in_mean, self.in_std, self.out_mean, self.out_std, self.env_lo,
                 self.env_hi)]
        fp = C.POINTER(C.c_float)
        d = capi.SurrogateDesc()
        d.n_in, d.n_hidden, d.n_hidden_layers, d.n_out = DIMS[0], DIMS[1], 3, DIMS[-1]
        d.params, d.in_mean, d.in_std, d.out_mean, d.out_std, d.env_lo, d.env_hi = [ptr(a, fp) for a in keep]
        d.nah_max = float(self.nah_max)
        d.log_mask = int(self.log_mask)
        d.v_update = int(self.v_update)
        for name in ("out_scale", "out_lo", "out_hi"):
            v = getattr(self, name)
            if v is not None:
                arr = np.ascontiguousarray(v, dtype=np.float32)
                keep.append(arr)
                setattr(d, name, ptr(arr, fp))
        d.hybrid_substeps = int(self.hybrid_substeps)
        return d, keep

    def deploy(self, sim):
        d, keep = self.desc()
        check(capi.lib().ep_set_surrogate(sim._h, C.byref(d)))

    def forward_kernel(self, Xn):
        """The deployed BF16 tensor-core kernel on normalised inputs (tests)."""
        n = len(Xn)
        X = np.zeros((n, 32), np.float32)
        X[:, :Xn.shape[1]] = Xn
        Y = np.zeros((n, 32), np.float32)
        d, keep = self.desc()
        fp = C.POINTER(C.c_float)
        check(capi.lib().ep_surrogate_forward(C.byref(d), n, ptr(X, fp), ptr(Y, fp)))
        return Y[:, :DIMS[-1]]


def features(states, istim_pApF, gks_abs, gto, sflag):
    """(n, 23) inputs: V, 18 states, I_stim [pA/pF], G_Ks, G_to, s-gate variant."""
    n = len(states)
    X = np.empty((n, 23))
    X[:, :19] = states[:, :19]
    X[:, 19] = istim_pApF
    X[:, 20] = gks_abs
    X[:, 21] = gto
    X[:, 22] = sflag
    return X


def in_domain(states, istim, nah_max=NAH_MAX):
    m, h = states[:, 7], states[:, 8]
    return (m ** 3 * h <= nah_max) & (istim == 0.0)


def _random_slab(rng):
    """A slab with random transmural layering, G_Ks field and stimulus."""
    from .workloads import tt_type_consts, TT_XI
    nx, ny, nz = 41, 41, 6
    m = M.slab(nx, ny, nz, 0.8, 0.8, 0.1, fiber_deg=(rng.uniform(-80, -40), rng.uniform(40, 80)))
    # types by random planes through the slab
    ax = rng.integers(0, 2)
    u = m.xyz[:, ax] / 0.8
    cut1, cut2 = sorted(rng.uniform(0.1, 0.9, 2))
    node_type = np.where(u < cut1, 0, np.where(u < cut2, 1, 2)).astype(np.uint8)
    g0, g1 = rng.uniform(0.6, 1.4, 2)
    gks = g0 + (g1 - g0) * (m.xyz[:, 1 - ax] / 0.8)
    tc = tt_type_consts()
    # stimulus: a random corner or edge block, sometimes a second one later.
    # The first beat starts after a random rest of up to 150 ms: in a large
    # tissue most nodes wait that long for the wave, and their gates keep
    # relaxing from the initial state meanwhile (slow Xr1 in particular).
    ids = []
    t_on = []
    t_first = rng.uniform(0.0, 150.0) if rng.random() < 0.7 else 0.0
    for k in range(1 + (rng.random() < 0.5)):
        t_k = t_first if k == 0 else rng.uniform(max(340.0, t_first + 300.0), 480.0)
        if k == 1 and t_k >= 480.0:
            break
        cx, cy = rng.integers(0, 2, 2) * (nx - 4)
        blk = ((m.xyz[:, 0] - cx * 0.02) ** 2 + (m.xyz[:, 1] - cy * 0.02) ** 2 < 0.1 ** 2)
        idx = np.where(blk)[0]
        ids.append(idx)
        t_on.append(np.full(len(idx), t_k))
    ids = np.concatenate(ids).astype(np.int32)
    t_on = np.concatenate(t_on)
    amp = rng.uniform(40.0, 60.0) * TT_XI
    return m, node_type, tc, gks, ids, t_on, amp


def generate(n_target=10_000_000, seed=0, T=500.0, every=5, device=0, verbose=True, max_runs=64,
             nah_max=NAH_MAX):
    """Training pairs (X, Y) from randomised plain-model slab runs.
    X: (N, 23) inputs; Y: (N, 19) changes of V and the 18 states over one
    0.1 ms step's ionic phase (plain FP64 model from the same start)."""
    from .simulation import Monodomain
    from .workloads import TT_XI
    rng = np.random.default_rng(seed)
    Xs, Ys = [], []
    total = 0
    run = 0
    while total < n_target and run < max_runs:
        m, node_type, tc, gks, ids, t_on, amp = _random_slab(rng)
        D = M.sigma_to_D(1.2, 0.2) * rng.uniform(0.7, 1.3)
        g = Monodomain(m, capi.TUSSCHER, capi.FP32, dt=0.1, ionic_dt=0.02, D=D, node_type=node_type,
                       type_consts=tc, gks_scale=gks, tt_jacobian=capi.TT_JAC_TRUE, device=device)
        g.set_voltage(-85.423)
        g.set_stimulus(ids, t_on, t_on + 2.0, amp)
        nsteps = int(round(T / 0.1))
        for s in range(0, nsteps, every):
            g.step(every)
            st = g.states()
            t = (s + every) * 0.1
            istim = np.zeros(m.n)
            act = (t_on <= t) & (t < t_on + 2.0)
            istim[ids[act]] = amp
            keep = in_domain(st, istim, nah_max)
            # keep every state on the way to threshold (the foot of the action
            # potential decides activation times), 20% of the plateau and
            # repolarisation, 4% of rest
            V = st[:, 0]
            u = rng.random(m.n)
            rest = np.abs(V + 85.4) < 1.0
            foot = (V > -84.4) & (V < -45.0) & (st[:, 8] > 0.05)      # h not yet inactivated
            keep &= foot | (rest & (u < 0.04)) | (~rest & ~foot & (u < 0.2))
            idx = np.where(keep)[0]
            if len(idx) == 0:
                continue
            S = np.ascontiguousarray(st[idx])
            X = features(S, istim[idx] / TT_XI, tc[node_type[idx], 15] * gks[idx], tc[node_type[idx], 20],
                         tc[node_type[idx], 53])
            Y = ionic_phase_targets(S, istim[idx], node_type[idx], tc, gks[idx])
            Xs.append(transform(X).astype(np.float32))
            Ys.append(target_from_delta(S, Y).astype(np.float32))
            total += len(idx)
        g.close()
        run += 1
        if verbose:
            print(f"  run {run}: {total} samples", flush=True)
    X = np.concatenate(Xs)
    Y = np.concatenate(Ys)
    perm = rng.permutation(len(X))[:n_target]
    return X[perm], Y[perm]


def ionic_phase_targets(S, istim, node_type, tc, gks, precision=capi.FP64, newton_tol=1e-12):
    """Change of V and the 18 states over one 0.1 ms ionic phase."""
    n = len(S)
    st = np.ascontiguousarray(S, dtype=np.float64).copy()
    V = st[:, 0].copy()
    mo = capi.ModelDesc()
    mo.model = capi.TUSSCHER
    tarr = np.ascontiguousarray(node_type, dtype=np.uint8)
    tcs = np.ascontiguousarray(tc, dtype=np.float64)
    g = np.ascontiguousarray(gks, dtype=np.float64)
    ist = np.ascontiguousarray(istim, dtype=np.float64)
    mo.n_types = tcs.shape[0]
    mo.type_consts = ptr(tcs)
    mo.node_type = ptr(tarr, C.POINTER(C.c_uint8))
    mo.node_gks_scale = ptr(g)
    mo.tt_jacobian = capi.TT_JAC_TRUE
    # The reference stops Newton at |dx| <= 1e-6 absolute, which is the size
    # of one step's change of Cai itself; the targets use a tight tolerance
    # so they are the implicit-Euler solution, not its stopping noise.
    mo.newton_tol = newton_tol
    mo.newton_cap = 200
    check(capi.lib().ep_ionic_phase(C.byref(mo), precision, n, 0.1, 0.02, 1.0, ptr(V), ptr(ist), ptr(st)))
    Y = st[:, :19] - S[:, :19]
    Y[:, 0] = V - S[:, 0]
    return Y


class Trainer:
    """ctypes wrapper of the GPU trainer (ep_mlp_*)."""

    def __init__(self, dims=DIMS, seed=0, device=0):
        self.dims = list(dims)
        d = (C.c_int32 * len(dims))(*dims)
        h = C.c_void_p()
        check(capi.lib().ep_mlp_create(len(dims) - 1, d, seed, device, C.byref(h)))
        self._h = h
        self.np = capi.lib().ep_mlp_num_params(h)

    def params(self):
        out = np.empty(self.np, np.float32)
        check(capi.lib().ep_mlp_get_params(self._h, ptr(out, C.POINTER(C.c_float))))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(capi.lib().ep_mlp_set_params(self._h, ptr(p, C.POINTER(C.c_float))))

    def loss_grad(self, Xd, Yd, B, w=None, want_grad=False, want_loss=True):
        """Xd, Yd: device pointers (int) of FP32 row-major batches.  Without
        want_loss/want_grad nothing is copied back (no host sync)."""
        loss = C.c_double(0)
        g = np.empty(self.np, np.float32) if want_grad else None
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
        check(capi.lib().ep_mlp_loss_grad(self._h, C.c_void_p(Xd), C.c_void_p(Yd),
                                          ptr(wa, C.POINTER(C.c_float)), B,
                                          C.byref(loss) if want_loss else None,
                                          ptr(g, C.POINTER(C.c_float)), None))
        return (loss.value if want_loss else None), g

    def forward(self, Xd, Yd, B):
        check(capi.lib().ep_mlp_forward(self._h, C.c_void_p(Xd), C.c_void_p(Yd), B, None))

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        check(capi.lib().ep_mlp_adam_step(self._h, lr, b1, b2, eps))

    def close(self):
        if getattr(self, "_h", None):
            capi.lib().ep_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train(X, Y, epochs=20, batch=8192, lr=2e-3, seed=0, device=0, verbose=True, w_v=10.0, nah_max=NAH_MAX,
          asinh_q=None, conc_only=False):
    """Fit the network to normalised (X, Y) on the GPU; returns a Surrogate.

    asinh_q: if given, output j is learned as asinh(Y_j / s_j) with s_j the
    asinh_q quantile of |Y_j|, so that the small changes of the plateau and
    of rest are fitted to a relative, not an absolute, accuracy.
    conc_only: fit only the six Newton concentrations (the hybrid form,
    v_update 2, reads nothing else)."""
    import torch
    X = np.asarray(X, np.float32)
    Y = np.asarray(Y, np.float32)
    out_scale = None
    if asinh_q is not None:
        aY = np.abs(Y[: min(len(Y), 2_000_000)]).astype(np.float64)
        sc = np.quantile(aY, asinh_q, axis=0)
        sc = np.maximum(sc, 1e-6 * aY.max(axis=0))
        sc = np.maximum(sc, 1e-30)
        out_scale = sc.astype(np.float32)
        Y = np.arcsinh(Y.astype(np.float64) / sc).astype(np.float32)
    # statistics in FP64 (column sums of millions of FP32 values lose digits)
    X64 = X.astype(np.float64)
    Y64 = Y.astype(np.float64)
    in_mean = X64.mean(axis=0)
    in_std = X64.std(axis=0)
    in_std[in_std < 1e-12] = 1.0
    out_mean = Y64.mean(axis=0)
    out_std = Y64.std(axis=0)
    out_std[out_std < 1e-20] = 1.0
    lo, hi = X64.min(axis=0), X64.max(axis=0)
    # accepted output range: the targets' range widened by 25 % of its span
    ylo, yhi = Y64.min(axis=0), Y64.max(axis=0)
    out_lo = (ylo - 0.25 * (yhi - ylo)).astype(np.float32)
    out_hi = (yhi + 0.25 * (yhi - ylo)).astype(np.float32)
    # training envelope: the data's box widened by 5 % of its span and by
    # 1 % of the magnitude (slow concentrations barely move in the data)
    margin = np.maximum(0.05 * (hi - lo), 0.01 * np.maximum(np.abs(lo), np.abs(hi)))
    env_lo = lo - margin
    env_hi = hi + margin
    del X64, Y64
    in_mean, in_std = in_mean.astype(np.float32), in_std.astype(np.float32)
    out_mean, out_std = out_mean.astype(np.float32), out_std.astype(np.float32)
    dev = torch.device("cuda", device)
    Xn = torch.from_numpy((X - in_mean) / in_std).to(dev)
    Yn = torch.from_numpy((Y - out_mean) / out_std).to(dev)
    n = len(Xn)
    nval = min(200_000, n // 20)
    Xv, Yv = Xn[:nval].contiguous(), Yn[:nval].contiguous()
    Xt, Yt = Xn[nval:], Yn[nval:]
    w = np.ones(DIMS[-1], np.float32)
    w[0] = w_v
    if conc_only:
        w[:] = 0.0
        w[list(CONC_OUTPUTS)] = 1.0
    tr = Trainer(seed=seed, device=device)
    gen = torch.Generator(device=dev).manual_seed(seed)
    steps_per_epoch = max(1, len(Xt) // batch)
    total = epochs * steps_per_epoch
    step = 0
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(len(Xt), device=dev, generator=gen)
        run = 0.0
        for k in range(steps_per_epoch):
            idx = perm[k * batch:(k + 1) * batch]
            xb = Xt[idx].contiguous()
            yb = Yt[idx].contiguous()
            probe = (k % 50 == 0)
            loss, _ = tr.loss_grad(xb.data_ptr(), yb.data_ptr(), len(idx), w, want_loss=probe)
            if probe:
                run += loss * 50
            lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))
            tr.adam(lr_t)
            step += 1
        vloss = 0.0
        for k in range(0, nval, 65536):
            b = min(65536, nval - k)
            l, _ = tr.loss_grad(Xv[k:k + b].data_ptr(), Yv[k:k + b].data_ptr(), b, w)
            vloss += l * b
        vloss /= max(1, nval)
        hist.append((run / steps_per_epoch, vloss))
        if verbose:
            print(f"  epoch {ep + 1}/{epochs}: train {run / steps_per_epoch:.3e} val {vloss:.3e}", flush=True)
    # per-output normalised error on the validation rows
    pred = torch.empty_like(Yv)
    for k in range(0, nval, 65536):
        b = min(65536, nval - k)
        tr.forward(Xv[k:k + b].data_ptr(), pred[k:k + b].data_ptr(), b)
    per_out = ((pred - Yv) ** 2).mean(dim=0).cpu().numpy()
    if verbose:
        print("  validation MSE per output (normalised):", np.array2string(per_out, precision=2), flush=True)
    p = tr.params()
    tr.close()
    return Surrogate(p, in_mean, in_std, out_mean, out_std, env_lo.astype(np.float32),
                     env_hi.astype(np.float32), nah_max=nah_max, log_mask=LOG_MASK,
                     out_scale=out_scale, out_lo=out_lo, out_hi=out_hi,
                     v_update=2 if conc_only else 0, hybrid_substeps=1,
                     meta={"n_samples": int(n), "epochs": epochs, "lr": lr, "batch": batch,
                           "asinh_q": asinh_q, "conc_only": conc_only, "history": hist})


def main():
    import argparse
    import time
    ap = argparse.ArgumentParser(description="generate data, train and save the learned ionic step")
    ap.add_argument("--samples", type=int, default=10_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--asinh-q", type=float, default=None)
    ap.add_argument("--data", default=None, help="cache of the generated pairs (.npz)")
    ap.add_argument("--nah-max", type=float, default=NAH_MAX,
                    help="largest fast sodium gate product m^3 h the network takes (the upstroke bound)")
    ap.add_argument("--conc-only", action="store_true",
                    help="fit only the six Newton concentrations (hybrid form)")
    args = ap.parse_args()
    t0 = time.time()
    if args.data and os.path.exists(args.data):
        z = np.load(args.data)
        X, Y = z["X"], z["Y"]
    else:
        X, Y = generate(args.samples, seed=args.seed, nah_max=args.nah_max)
        if args.data:
            np.savez(args.data, X=X, Y=Y)
    print(f"data: {X.shape} in {time.time() - t0:.1f} s", flush=True)
    t1 = time.time()
    s = train(X, Y, epochs=args.epochs, seed=args.seed, lr=args.lr, batch=args.batch, nah_max=args.nah_max,
              asinh_q=args.asinh_q, conc_only=args.conc_only)
    print(f"training: {time.time() - t1:.1f} s", flush=True)
    s.save(args.out)
    print("saved", args.out)


if __name__ == "__main__":
    main()
