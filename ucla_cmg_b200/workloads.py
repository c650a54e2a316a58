"""The benchmark workloads as runnable set-ups (synthetic, seeded).

* :func:`slab_c0` -- 1.0 x 1.0 x 0.2 cm slab, 51 x 51 x 11 nodes (28,611),
  ten Tusscher epicardial, fibres -60..+60 deg through the thickness,
  50 uA/cm^2 for 1 ms at the 5 x 5 x 11 corner block, dt = 0.02 ms,
  2 electrodes 2 cm from the centre along x.
* :func:`slab_c1` -- 4.0 x 4.0 x 0.4 cm, 201 x 201 x 21 (848,421 nodes),
  Mahajan (26 states), stimulus on x <= 0.1 cm, dt = 0.01 ms.
* :func:`shell_c2` -- truncated prolate-ellipsoid shell, ~2.0M nodes /
  ~11.4M tets, ten Tusscher with a transmural endo/M/epi split of
  40/30/30 % and an apex->base G_Ks scale 0.8 -> 1.2, 200 PMJ stimuli on
  the endocardium (seed 0) at t ~ U(0, 30) ms, 10 electrodes on a sphere of
  radius 15 cm; dt = 0.1 ms with ionic sub-steps of 0.02 ms.
Conductivities sigma_l = 1.2, sigma_t = 0.2 mS/cm become D = sigma /
(chi C_m) with chi = 1400 /cm.  A stimulus of I uA/cm^2 enters the
reference's units as I * C_m * Xi_model uA/cm^3, so each model sees I uA/uF.
"""
from dataclasses import dataclass

import numpy as np

from . import capi, mesh as M

TT_XI = 2000.0
MH_XI = 1.55e-4 / 2.58e-8


def tt_type_consts(epi=None):
    """ten Tusscher 2006 parameter sets: 0 endo, 1 M, 2 epi.

    The reference ships the epicardial set only (SetUpIonicConstants.h:88-147);
    the endocardial (G_to 0.073, slow s-gate) and M-cell (G_Ks 0.098) sets are
    the TT2006 paper's values on top of it.  ``epi``: the epicardial set to
    start from (default: the library's copy of SetUpTusscherParameters; a CPU
    caller that must not load the GPU library passes its own)."""
    epi = capi.default_consts(capi.TUSSCHER) if epi is None else np.array(epi, dtype=np.float64)
    endo = epi.copy(); endo[20] = 0.073; endo[53] = 1.0
    mid = epi.copy(); mid[15] = 0.098
    return np.stack([endo, mid, epi])


@dataclass
class Workload:
    name: str
    mesh: object
    model: int
    dt: float
    ionic_dt: float
    T: float
    D: np.ndarray
    V0: float
    stim_ids: np.ndarray
    stim_on: np.ndarray
    stim_off: np.ndarray
    stim_amp: np.ndarray
    electrodes: np.ndarray
    node_type: np.ndarray = None
    type_consts: np.ndarray = None
    gks_scale: np.ndarray = None

    def create(self, precision, tt_jacobian=capi.TT_JAC_TRUE, ecg_every=None, **kw):
        from .simulation import Monodomain
        if ecg_every is None:
            ecg_every = max(1, int(round(1.0 / self.dt)))           # 1 ms samples
        g = Monodomain(self.mesh, self.model, precision, dt=self.dt, ionic_dt=self.ionic_dt,
                       D=self.D, node_type=self.node_type, type_consts=self.type_consts,
                       gks_scale=self.gks_scale, tt_jacobian=tt_jacobian, ecg_every=ecg_every, **kw)
        if self.V0 is not None:
            g.set_voltage(self.V0)
        g.set_stimulus(self.stim_ids, self.stim_on, self.stim_off, self.stim_amp)
        g.set_electrodes(self.electrodes)
        return g


def slab_c0(nx=51, ny=51, nz=11):
    m = M.slab(nx, ny, nz, 1.0, 1.0, 0.2)
    blk = M.corner_block(m, 5, 5)
    c = np.array([0.5, 0.5, 0.1])
    el = np.array([c + [2.0, 0, 0], c - [2.0, 0, 0]])
    k = len(blk)
    return Workload("slab_c0", m, capi.TUSSCHER, 0.02, 0.02, 100.0, M.sigma_to_D(1.2, 0.2), -85.423,
                    blk, np.zeros(k), np.ones(k), np.full(k, 50.0 * TT_XI), el)


def slab_c1(nx=201, ny=201, nz=21):
    m = M.slab(nx, ny, nz, 4.0, 4.0, 0.4)
    ids = np.where(m.xyz[:, 0] <= 0.1 + 1e-12)[0].astype(np.int32)
    k = len(ids)
    c = np.array([2.0, 2.0, 0.2])
    el = np.array([c + [6.0, 0, 0], c - [6.0, 0, 0]])
    return Workload("slab_c1", m, capi.MAHAJAN, 0.01, 0.01, 300.0, M.sigma_to_D(1.2, 0.2), None,
                    ids, np.zeros(k), np.full(k, 2.0), np.full(k, 50.0 * MH_XI), el,
                    node_type=np.zeros(m.n, np.uint8))


def shell_c2(h=0.0365, n_rho=20, seed=0, n_pmj=200, epi=None):
    m = M.shell(h=h, n_rho=n_rho)
    rho, height = m.meta["rho"], m.meta["height"]
    node_type = np.where(rho < 0.4, 0, np.where(rho < 0.7, 1, 2)).astype(np.uint8)
    gks = 0.8 + 0.4 * height
    sites, balls = M.pmj_sites(m, n_pmj, seed, 0.1)
    rng = np.random.default_rng(seed)
    t_on = rng.uniform(0.0, 30.0, n_pmj)
    ids = np.concatenate(balls).astype(np.int32)
    on = np.concatenate([np.full(len(b), t_on[i]) for i, b in enumerate(balls)])
    el = M.fibonacci_sphere(10, 15.0, m.xyz.mean(axis=0))
    return Workload("shell_c2", m, capi.TUSSCHER, 0.1, 0.02, 500.0, M.sigma_to_D(1.2, 0.2), -85.423,
                    ids, on, on + 2.0, np.full(len(ids), 50.0 * TT_XI), el,
                    node_type=node_type, type_consts=tt_type_consts(epi), gks_scale=gks)


@dataclass
class BatchWorkload:
    name: str
    instances: list          # dicts: mesh, D, node_type, type_consts
    model: int
    dt: float
    ionic_dt: float
    T: float
    V0: float
    stim_ids: np.ndarray     # concatenated node ids
    stim_on: np.ndarray
    stim_off: np.ndarray
    stim_amp: np.ndarray

    @property
    def n_nodes(self):
        return sum(inst["mesh"].n for inst in self.instances)

    def create(self, precision=capi.FP32, tt_jacobian=capi.TT_JAC_TRUE, **kw):
        from .simulation import Batch
        b = Batch(self.instances, self.model, precision, dt=self.dt, ionic_dt=self.ionic_dt,
                  tt_jacobian=tt_jacobian, **kw)
        b.set_voltage(self.V0)
        b.set_stimulus(self.stim_ids, self.stim_on, self.stim_off, self.stim_amp)
        return b


def batch_c3(n_inst=64, seed=0, h=0.02, lo=(21, 21, 6), hi=(101, 101, 11), epi=None):
    """64 independent ten Tusscher slabs of uneven size (grid uniform in
    21x21x6 .. 101x101x11 nodes, spacing 0.02 cm), each with G_Ks, G_to and
    G_CaL scaled by U(0.5, 1.5) and a 5x5-node full-thickness stimulus block
    at a random one of its four vertical edges (50 uA/cm^2, 1 ms at t = 0);
    FP32, dt = 0.02 ms, 200 ms.  ``epi`` as for :func:`tt_type_consts`."""
    rng = np.random.default_rng(seed)
    epi = capi.default_consts(capi.TUSSCHER) if epi is None else np.array(epi, dtype=np.float64)
    inst, ids, off = [], [], 0
    for k in range(n_inst):
        nx, ny = (int(v) for v in rng.integers(lo[:2], np.asarray(hi[:2]) + 1))
        nz = int(rng.integers(lo[2], hi[2] + 1))
        m = M.slab(nx, ny, nz, (nx - 1) * h, (ny - 1) * h, (nz - 1) * h)
        tc = epi.copy()
        for c in (15, 20, 18):                       # G_Ks, G_to, G_CaL
            tc[c] *= rng.uniform(0.5, 1.5)
        corner = int(rng.integers(0, 4))
        ci = (nx - 5) if corner & 1 else 0
        cj = (ny - 5) if corner & 2 else 0
        i, j, kk = np.meshgrid(np.arange(ci, ci + 5), np.arange(cj, cj + 5), np.arange(nz), indexing="ij")
        blk = (i + nx * (j + ny * kk)).ravel()
        ids.append(blk + off)
        inst.append(dict(mesh=m, D=M.sigma_to_D(1.2, 0.2), type_consts=tc[None, :], n_types=1))
        off += m.n
    ids = np.concatenate(ids).astype(np.int32)
    k = len(ids)
    return BatchWorkload("batch_c3", inst, capi.TUSSCHER, 0.02, 0.02, 200.0, -85.423, ids,
                         np.zeros(k), np.ones(k), np.full(k, 50.0 * TT_XI))
