"""The EPSimulator-compatible driver on the GPU: an input file and
reference-format mesh files in, Voltage_time_* files out, equal to the same
run made directly through the API."""
import os

import numpy as np
import pytest

from ucla_cmg_b200 import capi, mesh as M
from ucla_cmg_b200 import driver as D
from ucla_cmg_b200 import voomep_io as IO
from ucla_cmg_b200.simulation import Monodomain

pytestmark = pytest.mark.gpu


def test_driver_matches_direct_run(gpu, tmp_path):
    m = M.slab(13, 11, 5, 0.24, 0.2, 0.08)
    IO.write_mesh(str(tmp_path / "slab"), m)
    blk = M.corner_block(m, 3, 3)
    np.savetxt(tmp_path / "stim.txt", blk + 1, fmt="%d")
    dtxt = " ".join(repr(float(v)) for v in M.sigma_to_D(1.2, 0.2))
    (tmp_path / "case.input").write_text("MODEL slab\nOutputDir out/\nCellModel TUSSCHER\nDT 0.02\n"
                                         "IonicDT 0.02\nSimulationTime 5\nFrequency 1\n"
                                         f"TissueDiffusion {dtxt}\n"
                                         "Stimulus Nodal stim.txt 0. 1.0 100000\n")
    cfg, nsteps = D.run(str(tmp_path / "case.input"), capi.FP64, rest_voltage=True, verbose=False)
    # simtime accumulates 0.02 per step and is still below 5 after 250 steps,
    # so the loop (as the reference's) takes 251; the last output is at 250
    assert nsteps == 251
    out = tmp_path / "out"
    files = sorted(f for f in os.listdir(out) if f.startswith("Voltage_time_"))
    assert len(files) == 6 and files[0] == "Voltage_time_00000.00.00" and files[-1] == "Voltage_time_00005.00.00"
    Vd = np.fromfile(out / files[-1], dtype=np.float64)
    m2, _, _, _ = IO.read_mesh(str(tmp_path / "slab"))
    g = Monodomain(m2, capi.TUSSCHER, capi.FP64, dt=0.02, ionic_dt=0.02, D=M.sigma_to_D(1.2, 0.2),
                   tt_jacobian=capi.TT_JAC_TRUE)
    g.set_voltage(g.states()[:, 0])
    g.set_stimulus(blk, 0.0, 1.0, 100000.0)
    g.step(250)
    V = g.voltage()
    g.close()
    assert np.max(V) > 0.0                              # the wave is up
    assert np.array_equal(Vd, V)
