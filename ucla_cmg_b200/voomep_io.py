"""voomEP mesh files: readers (and writers, for fixtures and converted meshes).

Formats as the reference reads them (voomEP/src/Mesh/Mesh.cc):

* ``<base>.node``: header ``nNodes dim x x``, then ``id x y [z]`` per node
  (Mesh.cc:201, 316-323);
* ``<base>.ele``: header ``nElems x x``, then ``id nPerElem n1 .. nk`` with
  1-based node ids (Mesh.cc:279-290, 330-335); a 3D EP mesh holds 4-node
  tets, plus 2-node Purkinje cables in mixed (MIX3D) meshes;
* ``<base>.fibers``: per element, in ``.ele`` order, the 9 numbers
  f, s, n (Mesh.cc:337-341, CardiacBody.cc:158-167);
* ``<base>.cell``: lines ``nodeID typeID`` (1-based node ids), the tissue
  type of each node, default 0 (Mesh.cc:391-401);
* ``<base>.purk``: ``n`` then n 1-based node ids of Purkinje nodes
  (Mesh.cc:377-388);
* ``<base>.angle``: lines ``nodeID dx dy dz length`` overriding the direction
  and length of the cable that starts at that node (Mesh.cc:403-416,
  MixedMesh3D.cc:31-34, 89-92).

Outputs (EPSolver.cc:116-211, one rank): ``Voltage_time_%08.2f.00`` (raw
FP64 V per node) and ``InterVariables_time_%08.2f.00`` (per node a native
int nVar and nVar FP64 states; nVar differs between a tissue model and the
Purkinje cell of a mixed tissue).
"""
import os

import numpy as np

from .mesh import TetMesh


def read_node(path):
    with open(path) as f:
        tok = f.read().split()
    n, dim = int(tok[0]), int(tok[1])
    a = np.array(tok[4:4 + n * (dim + 1)], dtype=np.float64).reshape(n, dim + 1)
    xyz = np.zeros((n, 3))
    xyz[:, :dim] = a[:, 1:]
    return xyz


def read_ele(path):
    """(tets [m x 4] zero-based, element index of each tet, number of
    elements that are not 4-node tets)."""
    with open(path) as f:
        tok = f.read().split()
    ne = int(tok[0])
    pos = 3
    tets, which, other = [], [], 0
    for e in range(ne):
        k = int(tok[pos + 1])
        conn = tok[pos + 2:pos + 2 + k]
        pos += 2 + k
        if k == 4:
            tets.append([int(c) - 1 for c in conn])
            which.append(e)
        else:
            other += 1
    return np.array(tets, dtype=np.int32).reshape(-1, 4), np.array(which, dtype=np.int64), other


def bar_angle_nodes(first_nodes, is_bar, angle, sticky=True):
    """Per cable, the node whose .angle row overrides its direction and
    length, or -1 -- MixedMesh3D::Compute's rule over the whole .ele order
    (MixedMesh3D.cc:30-34, 78-87): every element whose first node is listed,
    a tet as much as a cable, switches the override on with that node's row,
    and it stays on for every later cable (``sticky``; False applies a row
    to the cable that starts at its node only).  ``first_nodes``: each
    element's first node (zero-based) in .ele order; ``is_bar``: which
    elements are cables."""
    out, cur = [], -1
    for v, b in zip(first_nodes, is_bar):
        v = int(v)
        if v in angle:
            cur = v
        if b:
            out.append(cur if sticky else (v if v in angle else -1))
    return np.array(out, dtype=np.int32)


def read_cables(base, node_type=None, angle_sticky=True):
    """The 2-node Purkinje cables of a mixed mesh ``base``: dict with
    ``bars`` [nb x 2] zero-based in .ele order, ``fibers`` [nb x 9] or None
    (from .fibers, in .ele order), ``lv`` [nb] (1 where either node has
    tissue type 11: the left-ventricular Purkinje diffusion,
    CardiacBody.cc:107-110), ``angle`` {zero-based node: (dx, dy, dz,
    length)} from .angle (empty if absent) and ``angle_node`` [nb], the node
    whose .angle row overrides each cable (-1: none) by the reference's
    element-order rule (:func:`bar_angle_nodes`)."""
    with open(base + ".ele") as f:
        tok = f.read().split()
    ne = int(tok[0])
    pos = 3
    bars, which, first, isbar = [], [], [], []
    for e in range(ne):
        k = int(tok[pos + 1])
        conn = tok[pos + 2:pos + 2 + k]
        pos += 2 + k
        first.append(int(conn[0]) - 1)
        isbar.append(k == 2)
        if k == 2:
            bars.append([int(c) - 1 for c in conn])
            which.append(e)
    bars = np.array(bars, dtype=np.int32).reshape(-1, 2)
    fib = None
    if os.path.exists(base + ".fibers") and len(bars):
        fib = read_fibers(base + ".fibers", ne)[np.array(which, dtype=np.int64)]
    lv = np.zeros(len(bars), np.uint8)
    if node_type is not None and len(bars):
        lv = ((node_type[bars[:, 0]] == 11) | (node_type[bars[:, 1]] == 11)).astype(np.uint8)
    angle = {}
    if os.path.exists(base + ".angle"):
        with open(base + ".angle") as f:
            a = f.read().split()
        for k in range(len(a) // 5):
            angle[int(a[5 * k]) - 1] = tuple(float(v) for v in a[5 * k + 1:5 * k + 5])
    return {"bars": bars, "fibers": fib, "lv": lv, "angle": angle,
            "angle_node": bar_angle_nodes(first, isbar, angle, angle_sticky)}


def read_fibers(path, n_elems):
    a = np.loadtxt(path, dtype=np.float64).reshape(-1)
    if a.size < 9 * n_elems:
        raise ValueError(f"{path}: {a.size} numbers for {n_elems} elements")
    return a[:9 * n_elems].reshape(n_elems, 9)


def read_cell(path, n):
    t = np.zeros(n, dtype=np.uint8)
    with open(path) as f:
        tok = f.read().split()
    a = np.array(tok[:len(tok) // 2 * 2], dtype=np.int64).reshape(-1, 2)
    t[a[:, 0] - 1] = a[:, 1]
    return t


def read_purk(path):
    with open(path) as f:
        tok = f.read().split()
    k = int(tok[0])
    return np.array(tok[1:1 + k], dtype=np.int64)


def read_mesh(base):
    """The tet mesh of ``base`` (.node/.ele, optional .fibers/.cell/.purk).
    Returns (TetMesh, node_type or None, purkinje node ids (1-based) or None,
    number of non-tet elements)."""
    xyz = read_node(base + ".node")
    tets, which, other = read_ele(base + ".ele")
    fib = None
    if os.path.exists(base + ".fibers"):
        with open(base + ".ele") as f:
            n_elems = int(f.readline().split()[0])
        fib = read_fibers(base + ".fibers", n_elems)[which]
    ntype = read_cell(base + ".cell", len(xyz)) if os.path.exists(base + ".cell") else None
    purk = read_purk(base + ".purk") if os.path.exists(base + ".purk") else None
    return TetMesh(xyz, tets, fib, {}), ntype, purk, other


def write_mesh(base, mesh, node_type=None):
    """Write ``mesh`` in the reference's formats (1-based ids)."""
    n, m = mesh.n, mesh.m
    with open(base + ".node", "w") as f:
        f.write(f"{n} 3 0 0\n")
        for i in range(n):
            x, y, z = mesh.xyz[i]
            f.write(f"{i + 1} {x:.17g} {y:.17g} {z:.17g}\n")
    with open(base + ".ele", "w") as f:
        f.write(f"{m} 4 0\n")
        for e in range(m):
            a, b, c, d = mesh.tets[e] + 1
            f.write(f"{e + 1} 4 {a} {b} {c} {d}\n")
    if mesh.fibers is not None:
        np.savetxt(base + ".fibers", mesh.fibers, fmt="%.17g")
    if node_type is not None:
        with open(base + ".cell", "w") as f:
            for i in range(n):
                f.write(f"{i + 1} {int(node_type[i])}\n")


def output_name(directory, kind, t, rank=0):
    """``<dir>/<kind>_time_%08.2f.%02d`` with kind "Voltage" or "InterVariables"."""
    return os.path.join(directory, "%s_time_%08.2f.%02.0f" % (kind, t, rank))


def read_voltage(path):
    return np.fromfile(path, dtype=np.float64)


def read_intervariables(path):
    """The per-node state vectors of an InterVariables file: a 2-D array when
    every node has the same nVar, else a list of 1-D arrays."""
    raw = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(raw):
        if pos + 4 > len(raw):
            raise ValueError(f"{path}: truncated at byte {pos}")
        nv = int(np.frombuffer(raw, dtype=np.int32, count=1, offset=pos)[0])
        pos += 4
        if nv < 0 or pos + 8 * nv > len(raw):
            raise ValueError(f"{path}: truncated or corrupt at byte {pos}")
        out.append(np.frombuffer(raw, dtype=np.float64, count=nv, offset=pos).copy())
        pos += 8 * nv
    if out and all(len(v) == len(out[0]) for v in out):
        return np.stack(out)
    return out


def write_intervariables(path, states):
    """Inverse of read_intervariables (a 2-D array or a list of vectors)."""
    with open(path, "wb") as f:
        for v in states:
            v = np.ascontiguousarray(v, dtype=np.float64)
            f.write(np.int32(len(v)).tobytes())
            f.write(v.tobytes())
