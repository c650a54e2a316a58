"""ComputeECG on the GPU path against the reference's own ComputeECG chain.

The reference's Mesh::New, MixedMesh3D/TetMesh::Compute and ComputeECG.h
(compiled unmodified into oracle/_ref/libvoomep_fem.so) evaluate each frame
from the same files; ucla_cmg_b200.compute_ecg reads the parameter file,
the frames of two ranks and the MIX3D cables, and reduces the frames on the
GPU (ep_ecg_eval).  Bar: 1e-12 of the largest lead value, per frame.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from ucla_cmg_b200 import compute_ecg as E, mesh as M

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.ref_fem_lib() is None, reason="oracle/_ref/libvoomep_fem.so not built")]
D_REF = (1e-3, 5e-4, 2.5e-4)


def _write_case(tmp_path, xyz, elements, fibers, purk=None, angle=None, nparts=2):
    mdir = tmp_path / "mesh"
    mdir.mkdir()
    base = str(mdir / "heart")
    O.write_reference_case(base, xyz, elements, fibers, purk=purk, angle=angle)
    npart = (np.arange(len(xyz)) * 7 % nparts).astype(int)
    np.savetxt(f"{base}.metis.npart.{nparts}", npart, fmt="%d")
    rng = np.random.default_rng(9)
    vdir = tmp_path / "volt"
    vdir.mkdir()
    frames = []
    for t in E.frame_times(1.0, 2.0, 0.25):
        V = np.where(xyz[:, 0] < 0.1 + 0.2 * float(t), 20.0, -85.0) + rng.normal(0.0, 1.0, len(xyz))
        frames.append(V)
        for r in range(nparts):
            V[npart == r].tofile(str(vdir / ("Voltage_time_%08.2f.%02.0f" % (t, float(r)))))
    return base, frames


def _params(tmp_path, kind, points, nparts=2):
    p = tmp_path / "ECG.input"
    pts = "\n".join(" ".join(f"{v:.17g}" for v in q) for q in points)
    p.write_text(f"heart\nmesh\nvolt\nout\n2\n{kind}\n{len(points)} 3\n{pts}\n{nparts}\n1.\n2.\n0.25\nBINARY\n")
    return str(p)


@pytest.mark.parametrize("kind", ["TET", "MIX3D"])
def test_compute_ecg_equals_the_reference_chain(gpu, tmp_path, kind):
    m = M.slab(8, 6, 4, 0.7, 0.5, 0.3)
    xyz, elements, fibers, purk, angle = m.xyz, [list(t) for t in m.tets], m.fibers, None, None
    if kind == "MIX3D":
        n0 = m.n
        xyz = np.vstack([m.xyz, m.xyz[[0]] + [[0.0, 0.0, -0.05], [0.0, 0.0, -0.1], [0.02, 0.0, -0.15]]])
        bars = [[0, n0], [n0, n0 + 1], [n0 + 1, n0 + 2]]
        elements = elements[:30] + [bars[0]] + elements[30:] + bars[1:]
        rng = np.random.default_rng(2)
        fib = []
        it = iter(m.fibers)
        for el in elements:
            if len(el) == 4:
                fib.append(next(it))
            else:
                q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
                fib.append(q.T.reshape(-1))
        fibers = np.array(fib)
        purk = np.array([n0, n0 + 1, n0 + 2])
        angle = {n0 + 1: (0.0, 0.6, -0.8, 0.06)}
    base, frames = _write_case(tmp_path, xyz, elements, fibers, purk=purk, angle=angle)
    c = xyz.mean(axis=0)
    points = np.vstack([M.fibonacci_sphere(5, 10.0, c), xyz[-1] + [0.03, 0.0, -0.04]])
    t, ecg = E.run(_params(tmp_path, kind, points), base_dir=str(tmp_path))
    assert len(t) == len(frames) == 4
    rm = O.RefFemMesh(base, mixed=(kind == "MIX3D"), radius=0.0275, compute=True)
    for k, V in enumerate(frames):
        ref = rm.ecg(D_REF, points, V)
        assert np.max(np.abs(ecg[k] - ref)) <= 1e-12 * np.max(np.abs(ref)), k
    # the output file: time and leads, tab separated, C++ stream defaults
    lines = open(tmp_path / "out" / "ECG_Data.00").read().splitlines()
    assert len(lines) == 4 and lines[1].split("\t")[0] == "1.25"
    assert np.allclose([float(v) for v in lines[2].split("\t")[1:-1]], ecg[2], rtol=1e-5)
