"""The C ABI library loads and exports every entry point include/ep_gpu.h
declares (no compute calls: runs without a GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from ucla_cmg_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_symbols_exported():
    syms = capi.exported_symbols()
    assert len(syms) >= 20
    missing = [n for n, ok in syms if not ok]
    assert not missing, missing


def test_every_header_function_bound():
    hdr = open(os.path.join(ROOT, "include", "ep_gpu.h")).read()
    names = set(re.findall(r"\b(ep_[a-z0-9_]+)\s*\(", hdr))
    L = capi.lib()
    for n in names:
        assert hasattr(L, n)


def test_host_only_entry_points():
    L = capi.lib()
    assert L.ep_version() == 3
    assert L.ep_model_nstate(capi.TUSSCHER) == 19
    assert L.ep_model_nstate(capi.MAHAJAN) == 26
    assert L.ep_model_nstate(capi.LUORUDY) == 8
    assert L.ep_model_nstate(99) < 0
    c = capi.default_consts(capi.TUSSCHER)
    assert c[15] == 0.392 and c[20] == 0.294 and c[18] == 0.0000398 and c[53] == 0.0
    m0 = capi.default_consts(capi.MAHAJAN, 0)
    assert np.isclose(m0[10], 1.9 * 0.32) and np.isclose(m0[24], 96.485 / (8.314 * 308.0))
    mf = capi.default_consts(capi.MAHAJAN_FAIL, 8)
    assert np.isclose(mf[7], 0.12 * 0.77 * 0.67) and np.isclose(mf[10], 0.9 * 0.1386 * 0.6)


def test_constants_match_oracle():
    from oracle import oracle as O
    assert np.array_equal(capi.default_consts(capi.TUSSCHER), O.tt_constants())
    for t in range(9):
        assert np.array_equal(capi.default_consts(capi.MAHAJAN, t), O.mh_constants(t))
        assert np.array_equal(capi.default_consts(capi.MAHAJAN_FAIL, t), O.mh_constants(t, True))
    assert capi.lib().ep_model_nstate(capi.PURKINJE) == 22
    assert np.array_equal(capi.default_consts(capi.PURKINJE), O.pk_constants())


def test_bad_arguments_return_codes():
    L = capi.lib()
    h = C.c_void_p()
    rc = L.ep_create(None, None, None, 0, C.byref(h))
    assert rc == -1 and b"null" in L.ep_last_error()


def test_batch_plan_host():
    """CTA groups of the batched CG launch: at least one CTA per instance,
    all CTAs used, the rest in proportion to the SELL-32 slices."""
    from ucla_cmg_b200.simulation import batch_plan
    rng = np.random.default_rng(3)
    sizes = rng.integers(2646, 112212, 64)
    row = np.concatenate([[0], np.cumsum(sizes)])
    for grid in (64, 148, 296, 592):
        blk = batch_plan(row, grid)
        cnt = np.diff(blk)
        assert blk[0] == 0 and blk[-1] == grid and cnt.min() >= 1
        slices = (row[1:] + 31) // 32 - row[:-1] // 32
        ideal = 1 + (grid - 64) * slices / slices.sum()
        assert np.all(np.abs(cnt - ideal) < 1.0 + 1e-9)
    with pytest.raises(capi.EPError):
        batch_plan(row, 63)


def test_purkinje_is_not_a_tissue_model():
    """EP_PURKINJE is accepted by the plugin entry (ep_ionic_step) and on the
    .purk nodes of mixed tissues (ep_create_mixed), and refused as a tissue
    model of its own by ep_create, before any device work."""
    from ucla_cmg_b200 import mesh as M, simulation as S
    m = M.slab(3, 3, 2, 0.2, 0.2, 0.1)
    md, mo, keep = S._instance_descs(m, capi.PURKINJE, (1e-3,) * 3, 1.0, None, None, None, None, 0.0, 0, 0, 0, None)
    sd = S._solver_desc(0.02, 0.02, 1e-7, 1000, 0.0, capi.FP64, 0.0, 0, -40.0)
    h = C.c_void_p()
    rc = capi.lib().ep_create(C.byref(md), C.byref(mo), C.byref(sd), 0, C.byref(h))
    assert rc == -1 and b"not a tissue model" in capi.lib().ep_last_error()
