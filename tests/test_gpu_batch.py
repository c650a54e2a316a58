"""Batched instances, graph replay and the autotuner on the GPU.

* A batch of slabs of different sizes, parameters and stimuli matches the
  same slabs run one by one (FP64: within 1e-9 mV; the only difference is
  the CTA split of the CG dot products, i.e. summation order).
* Replaying the steps from a CUDA graph gives bit-identical results to
  launching every kernel from the host, ECG samples included.
* The autotuner leaves the simulation state where it found it.
"""
import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200.simulation import Batch, Monodomain

pytestmark = pytest.mark.gpu
D = M.sigma_to_D(1.2, 0.2)
AMP = 50.0 * 2000.0


def _instances():
    epi = capi.default_consts(capi.TUSSCHER)
    out = []
    for k, (nx, ny, nz, s) in enumerate([(9, 9, 4, 1.0), (17, 11, 5, 1.4), (23, 13, 4, 0.6)]):
        m = M.slab(nx, ny, nz, (nx - 1) * 0.02, (ny - 1) * 0.02, (nz - 1) * 0.02)
        tc = epi.copy()
        tc[15] *= s
        tc[18] *= 2.0 - s
        out.append(dict(mesh=m, D=D, type_consts=tc[None, :], n_types=1))
    return out


def _stims(insts):
    """corner block of each instance (local ids)"""
    return [M.corner_block(inst["mesh"], 3, 3) for inst in insts]


def _single(inst, blk, prec, nsteps, **kw):
    g = Monodomain(inst["mesh"], capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, D=inst["D"],
                   type_consts=inst["type_consts"], tt_jacobian=capi.TT_JAC_TRUE, **kw)
    g.set_voltage(-85.423)
    g.set_stimulus(blk, 0.0, 1.0, AMP)
    g.step(nsteps)
    V = g.voltage()
    ta, _ = g.activation()
    g.close()
    return V, ta


def _batch(insts, blks, prec, **kw):
    b = Batch(insts, capi.TUSSCHER, prec, dt=0.02, ionic_dt=0.02, tt_jacobian=capi.TT_JAC_TRUE, **kw)
    b.set_voltage(-85.423)
    ids = np.concatenate([blk + b.offsets[k] for k, blk in enumerate(blks)]).astype(np.int32)
    b.set_stimulus(ids, 0.0, 1.0, AMP)
    return b


def test_batch_layout(gpu):
    insts = _instances()
    b = _batch(insts, _stims(insts), capi.FP64)
    n = [inst["mesh"].n for inst in insts]
    assert list(b.offsets) == [0, n[0], n[0] + n[1], sum(n)]
    cta = np.diff(b.cta_offsets)
    assert cta.min() >= 1
    # the largest instance has the most CTAs
    assert np.argmax(cta) == np.argmax(n)
    b.close()


def test_batch_matches_single_fp64(gpu):
    insts = _instances()
    blks = _stims(insts)
    b = _batch(insts, blks, capi.FP64, cg_tol=1e-12)
    b.step(600)                                   # 12 ms: the waves cross the slabs
    Vb = b.split(b.voltage())
    tb = b.split(b.activation()[0])
    for k, inst in enumerate(insts):
        Vs, ts = _single(inst, blks[k], capi.FP64, 600, cg_tol=1e-12)
        assert np.max(Vs) > 0.0
        assert np.max(np.abs(Vb[k] - Vs)) <= 1e-9, (k, np.max(np.abs(Vb[k] - Vs)))
        assert np.max(np.abs(tb[k] - ts)) <= 1e-4
    it, rr = b.cg_last()
    # each instance stops on its own test: ||r|| <= 1e-12 ||r0||, or at the
    # FP64 resolution of B V
    assert np.all(it >= 1) and np.all(rr <= 1e-10)
    b.close()


def test_batch_matches_single_fp32(gpu):
    insts = _instances()
    blks = _stims(insts)
    b = _batch(insts, blks, capi.FP32)
    b.step(600)
    tb = b.split(b.activation()[0])
    for k, inst in enumerate(insts):
        _, ts = _single(inst, blks[k], capi.FP32, 600)
        both = (ts >= 0) & (tb[k] >= 0)
        assert both.mean() > 0.5
        assert np.array_equal(ts >= 0, tb[k] >= 0)
        assert np.max(np.abs(tb[k][both] - ts[both])) <= 0.05
    b.close()


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_graph_replay_bit_identical(gpu, prec):
    insts = _instances()
    blks = _stims(insts)
    out = []
    for gs in (0, 25):
        b = _batch(insts, blks, prec)
        b.set_launch_config(graph_steps=gs)
        st = b.step(210)                           # 8 graphs + 10 direct steps
        out.append((b.voltage(), b.states(), b.activation()[0], b.time()))
        assert st["launches"] >= 4 * 210
        b.close()
    for a, c in zip(out[0][:3], out[1][:3]):
        assert np.array_equal(a, c)
    assert out[0][3] == out[1][3]


def test_graph_replay_ecg(gpu):
    m = M.slab(15, 15, 4, 0.28, 0.28, 0.06)
    blk = M.corner_block(m, 3, 3)
    el = np.array([[1.0, 0.14, 0.03], [-0.8, 0.14, 0.03]])
    res = []
    for gs in (0, 20):
        g = Monodomain(m, capi.TUSSCHER, capi.FP32, dt=0.02, ionic_dt=0.02, D=D, ecg_every=5,
                       tt_jacobian=capi.TT_JAC_TRUE)
        g.set_voltage(-85.423)
        g.set_stimulus(blk, 0.0, 1.0, AMP)
        g.set_electrodes(el)
        g.set_launch_config(graph_steps=gs)
        g.step(3)                                  # off the ECG phase on purpose
        g.step(297)
        t, e = g.ecg()
        res.append((g.voltage(), t, e))
        g.close()
    assert len(res[0][1]) == 60
    assert np.array_equal(res[0][1], res[1][1])
    assert np.array_equal(res[0][2], res[1][2])
    assert np.array_equal(res[0][0], res[1][0])


def test_autotune_restores_state(gpu):
    insts = _instances()
    blks = _stims(insts)
    b = _batch(insts, blks, capi.FP32)
    b.step(50)
    V0, S0, t0 = b.voltage(), b.states(), b.time()
    cfg, best, start, tried = b.autotune(trial_steps=10)
    assert tried >= 3 and best <= start
    assert b.launch_config() == cfg
    assert np.array_equal(b.voltage(), V0)
    assert np.array_equal(b.states(), S0)
    assert b.time() == t0
    b.step(50)
    assert np.all(np.isfinite(b.voltage()))
    b.close()


def test_graph_survives_state_upload(gpu):
    """Setting the voltage and the states between replays writes into the
    same device buffers, so the instantiated graph stays valid and the run
    matches one without graphs."""
    insts = _instances()
    blks = _stims(insts)
    out = []
    for gs in (0, 20):
        b = _batch(insts, blks, capi.FP32)
        b.set_launch_config(graph_steps=gs)
        b.step(60)
        S, V = b.states(), b.voltage()
        b.set_states(S)
        b.set_voltage(V)
        b.step(60)
        out.append(b.voltage())
        b.close()
    assert np.array_equal(out[0], out[1])
