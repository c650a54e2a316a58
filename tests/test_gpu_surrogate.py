"""The learned ionic step deployed in tissue (EP_SURROGATE handles).

* Fallback path: with an empty training envelope, or with every output
  outside its accepted range, every node runs the plain FP32 model, and the
  run is bit-identical to an EP_FP32 handle.
* Accuracy: the committed network (ucla_cmg_b200/data/tt_surrogate.npz) on
  a slab with endo/M/epi bands, a G_Ks gradient and a corner stimulus,
  judged by the plain FP64 run against the metric's targets: activation time
  within 0.5 ms, pseudo-ECG within 2 %.
* Ablation: the same deployment with the untrained network (the trainer's
  initial weights, same normalisation and envelope) against the trained one;
  the trained network takes most node-steps off the plain model at that
  accuracy, the untrained one cannot.
"""
import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M, workloads as W
from ucla_cmg_b200 import surrogate as SG
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


def _setup(nx=41, ny=41):
    m = M.slab(nx, ny, 5, 0.02 * (nx - 1), 0.02 * (ny - 1), 0.08)
    node_type = np.where(m.xyz[:, 0] < 0.32, 0, np.where(m.xyz[:, 0] < 0.56, 1, 2)).astype(np.uint8)
    gks = 0.8 + 0.4 * m.xyz[:, 1] / 0.8
    blk = np.where((m.xyz[:, 0] < 0.07) & (m.xyz[:, 1] < 0.07))[0].astype(np.int32)
    return m, node_type, gks, blk


def _run(prec, sg=None, T=60.0, ecg=True, size=(41, 41)):
    m, node_type, gks, blk = _setup(*size)
    g = Monodomain(m, capi.TUSSCHER, prec, dt=0.1, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                   node_type=node_type, type_consts=W.tt_type_consts(), gks_scale=gks,
                   tt_jacobian=capi.TT_JAC_TRUE, ecg_every=10 if ecg else 0)
    if sg is not None:
        sg.deploy(g)
    g.set_voltage(-85.423)
    g.set_stimulus(blk, 0.0, 2.0, 50.0 * W.TT_XI)
    if ecg:
        g.set_electrodes(np.array([[2.4, 0.4, 0.04], [-1.6, 0.4, 0.04], [0.4, 2.4, 0.04]]))
    g.set_profiling(True)
    steps = int(round(T / 0.1))
    fb = 0
    ion = 0.0
    for k in range(0, steps, 100):
        st = g.step(min(100, steps - k))
        fb += st["fallback_nodes"]
        ion += st["ionic_ms"]
        assert st["nonfinite"] == 0 and st["timeouts"] == 0
    out = dict(V=g.voltage(), ta=g.activation()[0], fb=fb / float(m.n * steps), ion_ms=ion / steps)
    if ecg:
        out["ecg"] = g.ecg()[1]
    g.close()
    return out


def _trained():
    return SG.Surrogate.load()


def test_empty_envelope_is_the_plain_model(gpu):
    s = _trained()
    s.env_lo = np.full_like(s.env_lo, 1e30)
    s.env_hi = np.full_like(s.env_hi, -1e30)
    a = _run(capi.SURROGATE, s, T=20.0)
    b = _run(capi.FP32, None, T=20.0)
    assert a["fb"] == 1.0
    assert np.array_equal(a["V"], b["V"])
    assert np.array_equal(a["ta"], b["ta"])


def test_short_fallback_list_runs_by_warps_with_the_same_bits(gpu):
    """A fallback list of at most 4096 nodes runs one warp per node (the
    Jacobian's rate evaluations side by side); it reproduces the one-thread-
    per-node model bit for bit: an empty envelope on a 765-node slab sends
    every node down that path, and the run equals the EP_FP32 handle's."""
    s = _trained()
    s.env_lo = np.full_like(s.env_lo, 1e30)
    s.env_hi = np.full_like(s.env_hi, -1e30)
    a = _run(capi.SURROGATE, s, T=20.0, size=(17, 9))
    b = _run(capi.FP32, None, T=20.0, size=(17, 9))
    assert a["fb"] == 1.0
    assert np.max(b["V"]) > 0.0
    assert np.array_equal(a["V"], b["V"])
    assert np.array_equal(a["ta"], b["ta"])


def test_graph_replay_with_the_fallback_stream(gpu):
    """The learned step forks its fallback list onto a second stream and joins
    it before the next kernel; replayed from CUDA graphs of 20 steps (the fork
    and join captured) the run equals the directly launched one bit for bit."""
    out = []
    for gs in (0, 20):
        m, node_type, gks, blk = _setup()
        g = Monodomain(m, capi.TUSSCHER, capi.SURROGATE, dt=0.1, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                       node_type=node_type, type_consts=W.tt_type_consts(), gks_scale=gks,
                       tt_jacobian=capi.TT_JAC_TRUE)
        _trained().deploy(g)
        g.set_launch_config(graph_steps=gs)
        g.set_voltage(-85.423)
        g.set_stimulus(blk, 0.0, 2.0, 50.0 * W.TT_XI)
        fb = 0
        for k in range(4):
            st = g.step(100)
            fb += st["fallback_nodes"]
            assert st["nonfinite"] == 0 and st["timeouts"] == 0
        out.append((g.voltage(), g.activation()[0], fb))
        g.close()
    assert out[0][2] > 0                         # the fallback list did run
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


def test_output_range_check_falls_back(gpu):
    s = _trained()
    s.out_lo = np.full(SG.DIMS[-1], 1e30, np.float32)
    s.out_hi = np.full(SG.DIMS[-1], -1e30, np.float32)
    a = _run(capi.SURROGATE, s, T=20.0, ecg=False)
    b = _run(capi.FP32, None, T=20.0, ecg=False)
    assert a["fb"] == 1.0
    assert np.array_equal(a["V"], b["V"])


def test_accuracy_against_fp64(gpu):
    ref = _run(capi.FP64)
    sg = _run(capi.SURROGATE, _trained())
    both = (ref["ta"] >= 0) & (sg["ta"] >= 0)
    assert np.array_equal(ref["ta"] >= 0, sg["ta"] >= 0)
    err = np.abs(sg["ta"] - ref["ta"])[both]
    ecg_l2 = np.linalg.norm(sg["ecg"] - ref["ecg"]) / np.linalg.norm(ref["ecg"])
    print(f"act err mean {err.mean():.3f} max {err.max():.3f} ms, ECG rel L2 {ecg_l2:.4f}, "
          f"fallback {sg['fb']:.3f}")
    # the metric's own targets: activation time within 0.5 ms, pseudo-ECG within 2 %
    # (this slab, 60 ms: mean 0.05 ms, max 0.10 ms, ECG 1.9 %)
    assert err.mean() <= 0.5
    assert err.max() <= 0.5
    assert ecg_l2 <= 0.02


def test_ablation_untrained_network(gpu):
    s = _trained()
    tr = SG.Trainer(SG.DIMS, seed=0)
    untrained = SG.Surrogate(**{**s.__dict__, "params": tr.params()})
    tr.close()
    ref = _run(capi.FP64, ecg=False)
    a = _run(capi.SURROGATE, s, ecg=False)
    b = _run(capi.SURROGATE, untrained, ecg=False)
    plain = _run(capi.FP32, ecg=False)
    both = (ref["ta"] >= 0) & (a["ta"] >= 0)
    err_a = np.abs(a["ta"] - ref["ta"])[both].mean()
    print(f"trained: fallback {a['fb']:.3f}, ionic {a['ion_ms']:.4f} ms/step, act err {err_a:.3f} ms; "
          f"untrained: fallback {b['fb']:.3f}, ionic {b['ion_ms']:.4f} ms/step; "
          f"plain FP32 ionic {plain['ion_ms']:.4f} ms/step")
    # the trained network takes most node-steps; the untrained one is either
    # rejected by the output-range check (fallback) or wrong
    assert a["fb"] < 0.5
    bb = (ref["ta"] >= 0) & (b["ta"] >= 0)
    err_b = np.abs(b["ta"] - ref["ta"])[bb].mean() if bb.any() else np.inf
    assert b["fb"] > 2 * a["fb"] or err_b > 4 * max(err_a, 0.05) or not np.array_equal(ref["ta"] >= 0, b["ta"] >= 0)


def test_four_pipeline_kernel_gives_the_same_bits(gpu):
    """sg_variant 1 (one CTA per SM running four 128-node tiles at once in
    four warpgroups) issues the same MMA and epilogue instructions per tile
    as sg_variant 0 (two CTAs per SM): the learned runs are bit-identical,
    fallbacks included, with a node count that leaves a partial last tile."""
    m, node_type, gks, blk = _setup()
    sg = _trained()
    out = []
    for var in (0, 1):
        g = Monodomain(m, capi.TUSSCHER, capi.SURROGATE, dt=0.1, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                       node_type=node_type, type_consts=W.tt_type_consts(), gks_scale=gks,
                       tt_jacobian=capi.TT_JAC_TRUE)
        sg.deploy(g)
        g.set_launch_config(sg_variant=var)
        assert g.launch_config()["sg_variant"] == var
        g.set_voltage(-85.423)
        g.set_stimulus(blk, 0.0, 2.0, 50.0 * W.TT_XI)
        st = g.step(300)
        assert st["timeouts"] == 0
        out.append((g.voltage(), g.states(), st["fallback_nodes"]))
        g.close()
    assert m.n % 128 != 0 and out[0][2] > 0
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
