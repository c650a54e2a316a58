"""Generate the golden vectors in this folder from the REFERENCE cell models.

The reference repository ships no test vectors for its ionic models, so the
goldens are produced here by running the reference's own sources
(voomEP/src/IonicModel/{Tusscher,Mahajan,Mahajan_fail,LR,Purkinje}.cc, compiled
unmodified into oracle/_ref/libvoomep_ref.so by oracle/Makefile) through
their IonicModel::Compute_Ion interface.

    python tests/golden/make_golden.py [name ...]   # needs oracle/_ref built
                                                    # (names: tt mahajan ... purkinje; default all)

Outputs (npz):
  tissue_tt_slab.npz  the split step (the oracle's CN/PCG restatement) with the
                    reference's TT objects as the cells: a 13x11x5-node slab,
                    corner stimulus, V at t = 2, 5 and 10 ms (name "tissue")
  cell_<model>.npz  single-cell trajectory under the split update
                    V <- V + dt * Compute_Ion(V, istim) with a 1 ms stimulus:
                    t, V (every sample_every steps), final states
  kat_<model>.npz   one Compute_Ion call on a batch of states sampled from
                    that trajectory with perturbed voltages and stimuli:
                    V, istim, states_in, states_out, dvdt
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

XI = {O.TUSSCHER: 2000.0, O.MAHAJAN: 1.55e-4 / 2.58e-8, O.MAHAJAN_FAIL: 1.55e-4 / 2.58e-8,
      O.LUORUDY: 2 * (11e-4 + 100e-4) / (11e-4 * 100e-4),
      O.LUORUDYWITHGATE: 2 * (11e-4 + 100e-4) / (11e-4 * 100e-4), O.PURKINJE: 2500.0}
NAME = {O.TUSSCHER: "tt", O.MAHAJAN: "mahajan", O.MAHAJAN_FAIL: "mahajan_fail",
        O.LUORUDY: "lr", O.LUORUDYWITHGATE: "lrgate", O.PURKINJE: "purkinje"}
# (dt, T, types, stimulus start): TT needs dt <= 0.01 with the reference
# Newton layout; LR starts with j = 1e-4 and needs ~100 ms to become excitable
CASES = {O.TUSSCHER: (0.01, 400.0, None, 0.0), O.MAHAJAN: (0.02, 400.0, [0, 4, 8], 0.0),
         O.MAHAJAN_FAIL: (0.02, 400.0, [2, 6], 0.0), O.LUORUDY: (0.02, 500.0, None, 100.0),
         O.LUORUDYWITHGATE: (0.02, 500.0, None, 100.0), O.PURKINJE: (0.02, 500.0, None, 10.0)}


def trajectory(model, dt, T, types, sample_every, t_stim):
    n = len(types) if types is not None else 1
    tarr = None if types is None else np.array(types, dtype=np.uint8)
    cells = O.RefCells(model, n, tarr)
    st = cells.state
    V = st[:, 7].copy() if model in (O.LUORUDY, O.LUORUDYWITHGATE) else st[:, 0].copy()
    if model in (O.LUORUDY, O.LUORUDYWITHGATE):
        V[:] = -84.0
    amp = 50.0 * XI[model]                      # 50 uA/cm^2 with C_m = 1
    nsteps = int(round(T / dt))
    ts, Vs, snaps = [], [], []
    for k in range(nsteps):
        ist = np.full(n, amp if t_stim <= k * dt < t_stim + 1.0 else 0.0)
        if k % sample_every == 0:
            ts.append(k * dt); Vs.append(V.copy()); snaps.append((V.copy(), cells.state.copy()))
        V = V + dt * cells.compute_ion(V, ist, dt)
    return cells, np.array(ts), np.array(Vs), V, snaps, tarr


def main():
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libvoomep_ref.so missing: run make -C oracle")
    rng = np.random.default_rng(1234)
    only = set(sys.argv[1:])
    for model, (dt, T, types, t_stim) in CASES.items():
        cells, t, Vs, Vend, snaps, tarr = trajectory(model, dt, T, types, int(round(1.0 / dt)), t_stim)
        if only and NAME[model] not in only:
            rng.choice(len(snaps), size=128, replace=False)      # keep the other models' draws
            n_in = 128 * (len(types) if types is not None else 1)
            rng.normal(0, 2.0, n_in); rng.random(n_in)
            continue
        np.savez_compressed(os.path.join(HERE, f"cell_{NAME[model]}.npz"), t=t, V=Vs, V_end=Vend,
                            states_end=cells.state, dt=dt, t_stim=t_stim, types=tarr if tarr is not None else np.zeros(0, np.uint8))
        # KAT batch: 256 snapshots x cells, perturbed V and stimulus
        pick = rng.choice(len(snaps), size=128, replace=False)
        Vin, Sin, Tin = [], [], []
        for p in pick:
            v, s = snaps[p]
            for c in range(len(v)):
                Vin.append(v[c] + rng.normal(0, 2.0)); Sin.append(s[c]); Tin.append(tarr[c] if tarr is not None else 0)
        Vin = np.array(Vin); Sin = np.array(Sin); Tin = np.array(Tin, dtype=np.uint8)
        ist = np.where(rng.random(len(Vin)) < 0.3, 50.0 * XI[model], 0.0)
        kat = O.RefCells(model, len(Vin), Tin if types is not None else None)
        kat.state = Sin
        dv = kat.compute_ion(Vin, ist, dt)
        np.savez_compressed(os.path.join(HERE, f"kat_{NAME[model]}.npz"), V=Vin, istim=ist,
                            states_in=Sin, states_out=kat.state, dvdt=dv, dt=dt, types=Tin)
        print(NAME[model], "trajectory", Vs.shape, "kat", Vin.shape, "Vmax", Vs.max())


def tissue():
    """V fields of a small slab: reference TT cells, dt 0.01 ms (their Newton
    layout needs dt <= 0.01), CN/PCG to 1e-12, stimulus 50 uA/cm^2 for 1 ms on
    a 3x3 full-thickness corner block."""
    from ucla_cmg_b200 import mesh as M
    m = M.slab(13, 11, 5, 0.6, 0.5, 0.2)
    D = M.sigma_to_D(1.2, 0.2)
    dt = 0.01
    blk = M.corner_block(m, 3, 3)
    c = O.Csr(m.xyz, m.tets, m.fibers, D, 1.0, dt)
    cells = O.RefCells(O.TUSSCHER, m.n)
    s = O.Sim(c, cells, dt, dt, cg_tol=1e-12, cg_maxit=2000, jacobi_steps=1)
    s.V[:] = -85.423
    snaps, times = [], (2.0, 5.0, 10.0)
    for k in range(int(round(times[-1] / dt))):
        s.istim[:] = 0.0
        if k * dt < 1.0:
            s.istim[blk] = 50.0 * 2000.0
        s.step(1)
        if any(abs((k + 1) * dt - t) < 1e-9 for t in times):
            snaps.append(s.V.copy())
    np.savez_compressed(os.path.join(HERE, "tissue_tt_slab.npz"), t=np.array(times), V=np.array(snaps),
                        dt=dt, nx=13, ny=11, nz=5, L=np.array([0.6, 0.5, 0.2]), stim_nodes=blk)
    print("tissue", np.array(snaps).shape, "Vmax", np.max(snaps))


if __name__ == "__main__":
    if sys.argv[1:] == ["tissue"]:
        tissue()
    else:
        main()
