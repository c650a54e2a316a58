"""GPU cell models through the C ABI (ep_ionic_step) vs the reference's
golden vectors and the CPU oracle."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import capi
from ucla_cmg_b200.simulation import ionic_step

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"tt": capi.TUSSCHER, "mahajan": capi.MAHAJAN, "mahajan_fail": capi.MAHAJAN_FAIL,
         "lr": capi.LUORUDY, "lrgate": capi.LUORUDYWITHGATE, "purkinje": capi.PURKINJE}

pytestmark = pytest.mark.gpu


def _kat(name):
    g = np.load(os.path.join(GOLD, f"kat_{name}.npz"))
    model = CASES[name]
    types = g["types"] if model in (capi.MAHAJAN, capi.MAHAJAN_FAIL) else None
    return g, model, types


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_kat(gpu, name):
    """FP64: one Compute_Ion call reproduces the reference outputs."""
    g, model, types = _kat(name)
    st = np.ascontiguousarray(g["states_in"].copy())
    dv = ionic_step(model, g["V"], g["istim"], st, float(g["dt"]), node_type=types)
    scale = np.maximum(np.abs(g["dvdt"]), 1.0)
    err_dv = np.max(np.abs(dv - g["dvdt"]) / scale)
    ref = g["states_out"]
    mask = np.ones(ref.shape[1], bool)
    mask[7 if model in (capi.LUORUDY, capi.LUORUDYWITHGATE) else 0] = False
    err_s = np.max(np.abs(st - ref)[:, mask] / np.maximum(np.abs(ref[:, mask]), 1e-12))
    assert err_dv < 1e-8, err_dv
    assert err_s < 1e-8, err_s


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_kat(gpu, name):
    """FP32: the same call, error bounded in single precision terms."""
    g, model, types = _kat(name)
    st = np.ascontiguousarray(g["states_in"].copy())
    dv = ionic_step(model, g["V"], g["istim"], st, float(g["dt"]), node_type=types,
                    precision=capi.FP32)
    scale = np.maximum(np.abs(g["dvdt"]), 1.0)
    # FD Jacobians and Newton stopping differ in FP32; the returned rate is
    # dominated by the fast currents and stays within 1e-2 relative
    assert np.median(np.abs(dv - g["dvdt"]) / scale) < 1e-4
    assert np.max(np.abs(dv - g["dvdt"]) / scale) < 5e-2


def test_tt_true_jacobian_matches_oracle(gpu):
    g, model, _ = _kat("tt")
    st = np.ascontiguousarray(g["states_in"].copy())
    dv = ionic_step(model, g["V"], g["istim"], st, 0.02, tt_jacobian=capi.TT_JAC_TRUE)
    c = O.Cells(O.TUSSCHER, len(g["V"]), tt_jac_true=1, newton_cap=100)
    c.state[:] = g["states_in"]
    dv_o = c.compute_ion(g["V"], g["istim"], 0.02)
    assert np.max(np.abs(dv - dv_o) / np.maximum(np.abs(dv_o), 1.0)) < 1e-8
    assert np.max(np.abs(st - c.state)[:, 1:] / np.maximum(np.abs(c.state[:, 1:]), 1e-12)) < 1e-8


def test_per_node_gks_scale(gpu):
    g, model, _ = _kat("tt")
    n = len(g["V"])
    scale = np.linspace(0.5, 1.5, n)
    st = np.ascontiguousarray(g["states_in"].copy())
    dv = ionic_step(model, g["V"], g["istim"], st, float(g["dt"]), gks_scale=scale)
    c = O.Cells(O.TUSSCHER, n, gks_scale=scale)
    c.state[:] = g["states_in"]
    dv_o = c.compute_ion(g["V"], g["istim"], float(g["dt"]))
    assert np.max(np.abs(dv - dv_o) / np.maximum(np.abs(dv_o), 1.0)) < 1e-8
