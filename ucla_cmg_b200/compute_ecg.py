"""ComputeECG on the GPU path: the pseudo-ECG of stored Voltage_time_* frames
(voomEP/src/Applications/CardiacEP/ComputeECG.cc:26-162).

    python -m ucla_cmg_b200.compute_ecg ECG.input [--device N]

Same as the reference:

* the parameter file is read positionally: model name, mesh directory,
  voltage directory, output directory, quadrature order, mesh type (TET or
  MIX3D here; HEX, QUAD and TRIA meshes are not on this path), the number of
  leads and their dimension, the lead coordinates, the number of ranks that
  wrote the frames, start, end and step of the frame times, and BINARY or
  ASCII (ComputeECG.cc:44-54);
* the mesh is <mesh directory>/<model name> in the reference's formats; a
  MIX3D mesh's 2-node cables enter the sums with the radius ComputeECG
  fixes, 0.0275 cm (ComputeECG.cc:75), and D is its hard-coded
  {1e-3, 5e-4, 2.5e-4} (ComputeECG.cc:88);
* frame times run as a float: ``for (float step = start; step < end; step +=
  frequency)``; frame t comes from Voltage_time_%08.2f.%02.0f of each rank,
  every node's value from the rank the .metis.npart.<ranks> file gives it,
  in increasing node order (ComputeECG.cc:120-139); the run stops at the
  first frame whose file is missing, as the reference does;
* output <output directory>/ECG_Data.00: per frame the time and the leads,
  tab separated, with C++ stream defaults (6 significant digits).

The per-node weights are built once (ep_ecg_create), and each frame is a dot
product per lead on the GPU (ep_ecg_eval).
"""
import argparse
import ctypes as C
import os

import numpy as np

from . import capi
from .capi import check, ptr
from .voomep_io import read_cables, read_mesh

KINDS = {"TET", "MIX3D", "HEX", "QUAD", "TRIA"}


def parse_params(path):
    """The positional ECG parameter file (ComputeECG.cc:44-54)."""
    tok = open(path).read().split()
    p = {"model": tok[0], "mesh_dir": tok[1], "voltage_dir": tok[2], "out_dir": tok[3],
         "quad_order": int(tok[4]), "mesh_type": tok[5]}
    npts, dim = int(tok[6]), int(tok[7])
    k = 8
    pts = np.array([float(v) for v in tok[k:k + npts * dim]]).reshape(npts, dim)
    k += npts * dim
    p.update(points=pts, nparts=tok[k], start=float(tok[k + 1]), end=float(tok[k + 2]),
             frequency=float(tok[k + 3]), fmt=tok[k + 4])
    if p["mesh_type"] not in KINDS:
        raise ValueError(f"unknown mesh type {p['mesh_type']} (QUAD, TRIA, HEX, TET, MIX3D)")
    return p


def frame_times(start, end, frequency):
    """The frame times of ComputeECG's ``for (float step = startStep; step <
    endStep; step = step + frequency)`` with double start, end and frequency
    (ComputeECG.cc:31, 112): each sum is taken in double and rounded to
    float, each test compares the float with the double end."""
    s = np.float32(start)
    out = []
    while float(s) < float(end):
        out.append(s)
        s = np.float32(float(s) + float(frequency))
    return out


def cpp_default(x):
    """A double as std::ostream prints it by default (%g, 6 digits)."""
    return "%g" % float(x)


def read_frame(vdir, t, npart, fmt, n):
    """One frame in global node order from the ranks' files, or None when a
    file is missing (the reference stops there)."""
    nparts = int(npart.max()) + 1 if len(npart) else 1
    V = np.empty(n)
    for r in range(nparts):
        name = os.path.join(vdir, "Voltage_time_%08.2f.%02.0f" % (t, float(r)))
        if not os.path.exists(name):
            return None
        nodes = np.where(npart == r)[0]
        if fmt == "ASCII":
            vals = np.loadtxt(name, dtype=np.float64, ndmin=1)
        else:
            vals = np.fromfile(name, dtype=np.float64)
        if len(vals) < len(nodes):
            raise ValueError(f"{name}: {len(vals)} values for {len(nodes)} nodes")
        V[nodes] = vals[:len(nodes)]
    return V


class Ecg:
    """ep_ecg: per-node weights of a mesh (tets + cables) on the GPU."""

    def __init__(self, mesh, electrodes, cables=None, D=None, device=0):
        from .simulation import _cables_desc, _instance_descs
        md, _, self._keep = _instance_descs(mesh, capi.TUSSCHER, (0.0, 0.0, 0.0), 1.0, None, None, None, None,
                                            0.0, 0, 0, 0, None)
        cd = _cables_desc(self._keep, **cables) if cables is not None else None
        el = np.ascontiguousarray(electrodes, dtype=np.float64).reshape(-1, 3)
        self._keep["el"] = el
        Dp = None if D is None else np.ascontiguousarray(D, dtype=np.float64)
        self._keep["D"] = Dp
        self.ne, self.n = len(el), mesh.n
        h = C.c_void_p()
        check(capi.lib().ep_ecg_create(C.byref(md), C.byref(cd) if cd is not None else None, self.ne, ptr(el),
                                       ptr(Dp), int(device), C.byref(h)))
        self._h = h

    def __call__(self, frames):
        V = np.ascontiguousarray(frames, dtype=np.float64).reshape(-1, self.n)
        out = np.empty((len(V), self.ne))
        check(capi.lib().ep_ecg_eval(self._h, len(V), ptr(V), ptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            capi.lib().ep_ecg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(param_file, device=0, base_dir=None, batch=64):
    """Run the parameter file; returns (frame times, ECG [frames x leads]).
    Relative paths are taken from ``base_dir`` (default: the current one, as
    for the reference's executable)."""
    p = parse_params(param_file)
    base = base_dir or os.getcwd()
    j = lambda d: d if os.path.isabs(d) else os.path.join(base, d)
    if p["mesh_type"] not in ("TET", "MIX3D"):
        raise ValueError(f"{p['mesh_type']} meshes are not on this path (TET and MIX3D are)")
    if p["points"].shape[1] != 3:
        raise ValueError("leads must be 3-D points")
    mbase = os.path.join(j(p["mesh_dir"]), p["model"])
    mesh, node_type, purk, other = read_mesh(mbase)
    cables = None
    if p["mesh_type"] == "MIX3D" and other:
        cab = read_cables(mbase, node_type)
        if len(cab["bars"]):
            cables = dict(bars=cab["bars"], bar_fibers=cab["fibers"], angle=cab["angle"],
                          bar_angle_node=cab["angle_node"], quad_order=p["quad_order"])
    npart = np.loadtxt(f"{mbase}.metis.npart.{p['nparts']}", dtype=np.int64, ndmin=1)[:mesh.n]
    e = Ecg(mesh, p["points"], cables, device=device)
    times, rows = [], []
    pend_t, pend_V = [], []

    def flush():
        if pend_V:
            rows.append(e(np.stack(pend_V)))
            times.extend(pend_t)
            pend_t.clear()
            pend_V.clear()
    for t in frame_times(p["start"], p["end"], p["frequency"]):
        V = read_frame(j(p["voltage_dir"]), t, npart, p["fmt"], mesh.n)
        if V is None:
            break
        pend_t.append(t)
        pend_V.append(V)
        if len(pend_V) >= batch:
            flush()
    flush()
    e.close()
    ecg = np.concatenate(rows) if rows else np.zeros((0, len(p["points"])))
    os.makedirs(j(p["out_dir"]), exist_ok=True)
    with open(os.path.join(j(p["out_dir"]), "ECG_Data.00"), "w") as f:
        for t, row in zip(times, ecg):
            f.write(cpp_default(t) + "\t" + "".join(cpp_default(v) + "\t" for v in row) + "\n")
    return np.array(times, dtype=np.float64), ecg


def main():
    ap = argparse.ArgumentParser(description="ComputeECG on the GPU path")
    ap.add_argument("params")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    t, ecg = run(a.params, a.device)
    print(f"** {len(t)} frames, {ecg.shape[1] if ecg.ndim == 2 else 0} leads")


if __name__ == "__main__":
    main()
