"""The ComputeECG drop-in (ucla_cmg_b200.compute_ecg) without a GPU: the
positional parameter file, the float frame-time loop and file names, the
frames of several ranks put back in node order, and the output format
(ComputeECG.cc:26-162)."""
import os

import numpy as np

from ucla_cmg_b200 import compute_ecg as E


def _params(tmp_path, fmt="BINARY", nparts=2, start="0.", end="1.", freq="0.1"):
    p = tmp_path / "ECG.input"
    p.write_text(f"slab\nmesh\nvolt\nout\n2\nTET\n2 3\n1.0 2.0 3.0\n-4.5E+00 5.0e-1 6\n{nparts}\n{start}\n{end}\n"
                 f"{freq}\n{fmt}\n")
    return str(p)


def test_parameter_file(tmp_path):
    p = E.parse_params(_params(tmp_path))
    assert p["model"] == "slab" and p["mesh_dir"] == "mesh" and p["voltage_dir"] == "volt"
    assert p["quad_order"] == 2 and p["mesh_type"] == "TET" and p["nparts"] == "2" and p["fmt"] == "BINARY"
    assert np.array_equal(p["points"], [[1.0, 2.0, 3.0], [-4.5, 0.5, 6.0]])
    assert (p["start"], p["end"], p["frequency"]) == (0.0, 1.0, 0.1)


def test_frame_times_are_float_accumulated():
    """``float step`` advanced by a double frequency, as the reference's loop
    (values from the same loop compiled in C): 0 .. 1 by 0.1 gives 10 frames
    ending at 0.900000095; 0.25 .. 1.5 by 0.05 gives 26 frames; the
    published 0 .. 5001 by 1 gives 5001."""
    t = E.frame_times(0.0, 1.0, 0.1)
    assert len(t) == 10 and abs(float(t[-1]) - 0.900000095) < 1e-9
    assert "Voltage_time_%08.2f.%02.0f" % (t[-1], 0.0) == "Voltage_time_00000.90.00"
    assert len(E.frame_times(0.25, 1.5, 0.05)) == 26
    assert len(E.frame_times(0.0, 5001.0, 1.0)) == 5001
    assert E.cpp_default(np.float32(0.1)) == "0.1" and E.cpp_default(1.23456789e-5) == "1.23457e-05"


def test_frames_from_several_ranks(tmp_path):
    """Each node's value comes from its rank's file, the rank's values in
    increasing node order (ComputeECG.cc:132-139); BINARY and ASCII."""
    n = 7
    npart = np.array([1, 0, 1, 1, 0, 0, 1])
    V = np.arange(n) * 1.5 - 3.0
    for fmt in ("BINARY", "ASCII"):
        d = tmp_path / fmt
        d.mkdir()
        for r in (0, 1):
            name = d / ("Voltage_time_%08.2f.%02.0f" % (2.0, float(r)))
            vals = V[npart == r]
            if fmt == "ASCII":
                np.savetxt(name, vals)
            else:
                vals.tofile(name)
        assert np.array_equal(E.read_frame(str(d), np.float32(2.0), npart, fmt, n), V)
        assert E.read_frame(str(d), np.float32(3.0), npart, fmt, n) is None     # missing: the run stops
