"""Synthetic linear-tet meshes, fibres, cell-type maps and stimulus sites.

The reference reads its geometry from ``.node/.ele/.fibers/.cell`` files
(voomEP/src/Mesh/Mesh.cc:142-483).  The workloads here are generated:

* :func:`slab` -- a box of ``nx*ny*nz`` nodes, every hexahedron split into 6
  tetrahedra along its main diagonal (Kuhn split, conforming), with the fibre
  angle rotating linearly through the thickness;
* :func:`shell` -- a truncated prolate-ellipsoid shell (a ventricle-like
  wall): a ring-by-ring surface triangulation of near-uniform spacing,
  extruded through the wall into prisms of 3 tets each.

Element fibres use the reference's 9-number layout per element (f, s, n;
voomEP/src/Body/CardiacBody.cc:158-167).  Node ids are zero-based here; the
``.ele`` files of the reference are one-based.
"""
from dataclasses import dataclass, field
import itertools

import numpy as np

CHI = 1400.0          # surface-to-volume ratio used to turn sigma into D [1/cm]


def sigma_to_D(sigma_l, sigma_t, Cm=1.0, chi=CHI):
    """D = sigma / (chi * Cm)  [cm^2/ms] for (fibre, sheet, normal)."""
    return np.array([sigma_l, sigma_t, sigma_t]) / (chi * Cm)


@dataclass
class TetMesh:
    xyz: np.ndarray                 # (n, 3) float64, cm
    tets: np.ndarray                # (m, 4) int32, zero-based, positive volume
    fibers: np.ndarray = None       # (m, 9) float64 or None (isotropic)
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.xyz)

    @property
    def m(self):
        return len(self.tets)

    def volumes(self):
        x = self.xyz[self.tets]
        a, b, c = x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]
        return np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0


_PERMS = list(itertools.permutations(range(3)))


def _kuhn_local():
    """The 6 Kuhn tets of the unit cube as corner bit-vectors."""
    out = []
    for p in _PERMS:
        v = [0, 0, 0]
        path = [tuple(v)]
        for ax in p:
            v[ax] = 1
            path.append(tuple(v))
        out.append(path)
    return out


def _orient(xyz, tets):
    x = xyz[tets]
    a, b, c = x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]
    vol = np.einsum("ij,ij->i", a, np.cross(b, c))
    neg = vol < 0
    tets = tets.copy()
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    return tets, np.abs(vol) / 6.0


def slab(nx, ny, nz, Lx, Ly, Lz, fiber_deg=(-60.0, 60.0), origin=(0.0, 0.0, 0.0)):
    """Box mesh, node id = i + nx*(j + ny*k), 6 tets per hex.

    ``fiber_deg`` = (angle at z=0, angle at z=Lz) in degrees for the fibre
    f = (cos t, sin t, 0), sheet s = (-sin t, cos t, 0), normal (0, 0, 1),
    evaluated at each element's centroid; ``None`` gives an isotropic mesh.
    """
    xs = np.linspace(0.0, Lx, nx) + origin[0]
    ys = np.linspace(0.0, Ly, ny) + origin[1]
    zs = np.linspace(0.0, Lz, nz) + origin[2]
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    i, j, k = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    tets = []
    for path in _kuhn_local():
        ids = [(i + c[0]) + nx * ((j + c[1]) + ny * (k + c[2])) for c in path]
        tets.append(np.stack(ids, axis=1))
    tets = np.concatenate(tets, axis=0).astype(np.int32)
    tets, _ = _orient(xyz, tets)
    fib = None
    if fiber_deg is not None:
        zc = xyz[tets][:, :, 2].mean(axis=1) - origin[2]
        t = np.deg2rad(fiber_deg[0] + (fiber_deg[1] - fiber_deg[0]) * zc / Lz)
        c, s = np.cos(t), np.sin(t)
        z0 = np.zeros_like(c)
        fib = np.stack([c, s, z0, -s, c, z0, z0, z0, np.ones_like(c)], axis=1)
    meta = dict(kind="slab", shape=(nx, ny, nz), size=(Lx, Ly, Lz))
    return TetMesh(xyz, tets, fib, meta)


def _zip_rings(ring_a, ang_a, ring_b, ang_b):
    """Triangulate the band between two closed rings of nodes (angles
    increasing in [0, 2pi)), advancing along whichever ring is behind."""
    na, nb = len(ring_a), len(ring_b)
    tris = []
    i = j = 0
    while i < na or j < nb:
        a0, b0 = ring_a[i % na], ring_b[j % nb]
        ta = ang_a[i + 1] if i + 1 <= na else np.inf
        tb = ang_b[j + 1] if j + 1 <= nb else np.inf
        if j >= nb or (i < na and ta <= tb):
            tris.append((a0, ring_a[(i + 1) % na], b0))
            i += 1
        else:
            tris.append((a0, ring_b[(j + 1) % nb], b0))
            j += 1
    return tris


def shell(h=0.0365, n_rho=20, a_in=2.5, c_in=5.0, wall=1.0, z_base=2.0,
          helix_deg=(60.0, -60.0)):
    """Truncated prolate-ellipsoid shell with near-uniform element size.

    Inner surface x^2/a^2 + y^2/a^2 + z^2/c^2 = 1 with (a, c) = (a_in, c_in),
    outer surface (a_in + wall, c_in + wall); apex at z = -c, cut by the base
    plane z = ``z_base``.  A surface mesh of rings (ring j has as many nodes
    as its mid-wall circumference holds at spacing ``h``; one apex node) is
    zipped into triangles and extruded through ``n_rho`` transmural layers;
    each prism is split into 3 tets.  Defaults give ~2.0M nodes / ~11.5M
    tets.  Fibres: helix angle rotating linearly endo->epi.
    meta["rho"] (per node, 0 endo .. 1 epi) and meta["height"] (0 apex .. 1
    base) feed the transmural and apicobasal parameter maps.
    """
    rho = np.linspace(0.0, 1.0, n_rho + 1)
    a = a_in + wall * rho
    c = c_in + wall * rho
    tmax = np.arccos(-z_base / c)
    # mid-wall meridian arc length -> number of rings
    am, cm = a_in + 0.5 * wall, c_in + 0.5 * wall
    tm = np.arccos(-z_base / cm)
    tt = np.linspace(0.0, tm, 4001)
    seg = np.hypot(np.diff(am * np.sin(tt)), np.diff(cm * np.cos(tt)))
    arc = np.concatenate([[0.0], np.cumsum(seg)])
    n_theta = max(2, int(round(arc[-1] / h)))
    u = np.interp(np.linspace(0.0, arc[-1], n_theta + 1), arc, tt) / tm   # fraction of tmax
    ring_n = [1] + [max(6, int(round(2 * np.pi * am * np.sin(u[j] * tm) / h))) for j in range(1, n_theta + 1)]
    offs = np.concatenate([[0], np.cumsum(ring_n)])
    n_surf = int(offs[-1])
    # surface triangulation (same for every layer)
    tris = [(0, offs[1] + k, offs[1] + (k + 1) % ring_n[1]) for k in range(ring_n[1])]
    for j in range(1, n_theta):
        na, nb = ring_n[j], ring_n[j + 1]
        ang_a = np.concatenate([2 * np.pi * np.arange(na) / na, [2 * np.pi]])
        ang_b = np.concatenate([2 * np.pi * np.arange(nb) / nb, [2 * np.pi]])
        tris += _zip_rings(offs[j] + np.arange(na), ang_a, offs[j + 1] + np.arange(nb), ang_b)
    tris = np.array(tris, dtype=np.int64)
    # node coordinates, node id = layer * n_surf + surface id
    jj = np.zeros(n_surf, dtype=np.int64)
    phi = np.zeros(n_surf)
    for j in range(1, n_theta + 1):
        jj[offs[j]:offs[j + 1]] = j
        phi[offs[j]:offs[j + 1]] = 2 * np.pi * np.arange(ring_n[j]) / ring_n[j]
    xyz = np.zeros(((n_rho + 1) * n_surf, 3))
    for k in range(n_rho + 1):
        th = u[jj] * tmax[k]
        sl = slice(k * n_surf, (k + 1) * n_surf)
        xyz[sl, 0] = a[k] * np.sin(th) * np.cos(phi)
        xyz[sl, 1] = a[k] * np.sin(th) * np.sin(phi)
        xyz[sl, 2] = -c[k] * np.cos(th)
    # prisms -> tets
    bot = np.concatenate([tris + k * n_surf for k in range(n_rho)])
    tets = _split_prisms(bot, bot + n_surf)
    tets, vol = _orient(xyz, tets.astype(np.int32))
    rho_n = np.repeat(rho, n_surf)
    zmin = -c[0]
    height = np.clip((xyz[:, 2] - zmin) / (z_base - zmin), 0.0, 1.0)
    fib = _helix_fibers(xyz, tets, rho_n, a_in, c_in, wall, helix_deg)
    meta = dict(kind="shell", rho=rho_n, height=height, n_theta=n_theta, n_rho=n_rho,
                endo_nodes=np.arange(n_surf), z_base=z_base, h=h, ring_n=np.array(ring_n))
    return TetMesh(xyz, tets, fib, meta)


def _split_prisms(bot, top):
    """Conforming 3-tet split of prisms (bottom tri, top tri): every quad
    face is cut along the diagonal through its smallest global node id
    (the face diagonals then never form a cycle, so 3 tets always fit)."""
    P = np.concatenate([bot, top], axis=1)
    m = np.argmin(P, axis=1)
    flip = m >= 3
    P[flip] = np.concatenate([P[flip, 3:], P[flip, :3]], axis=1)
    m = np.where(flip, m - 3, m)
    r = np.arange(len(P))
    i0, i1, i2 = m, (m + 1) % 3, (m + 2) % 3
    v0, v1, v2 = P[r, i0], P[r, i1], P[r, i2]
    v3, v4, v5 = P[r, 3 + i0], P[r, 3 + i1], P[r, 3 + i2]
    d15 = np.minimum(v1, v5) < np.minimum(v2, v4)
    t1 = np.where(d15[:, None], np.stack([v0, v1, v2, v5], 1), np.stack([v0, v1, v2, v4], 1))
    t2 = np.where(d15[:, None], np.stack([v0, v1, v5, v4], 1), np.stack([v0, v4, v2, v5], 1))
    t3 = np.stack([v0, v4, v5, v3], 1)
    return np.concatenate([t1, t2, t3], axis=0)


def _helix_fibers(xyz, tets, rho_n, a_in, c_in, wall, helix_deg):
    if helix_deg is None:
        return None
    cen = xyz[tets].mean(axis=1)
    rc = rho_n[tets].mean(axis=1)
    r_xy = np.hypot(cen[:, 0], cen[:, 1])
    ec = np.stack([-cen[:, 1], cen[:, 0], np.zeros(len(cen))], axis=1)
    ec[r_xy < 1e-9] = np.array([1.0, 0.0, 0.0])
    ec /= np.linalg.norm(ec, axis=1, keepdims=True)
    ae = a_in + wall * rc
    ce = c_in + wall * rc
    nrm = np.stack([cen[:, 0] / ae ** 2, cen[:, 1] / ae ** 2, cen[:, 2] / ce ** 2], axis=1)
    nrm -= np.einsum("ij,ij->i", nrm, ec)[:, None] * ec
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    el = np.cross(nrm, ec)
    al = np.deg2rad(helix_deg[0] + (helix_deg[1] - helix_deg[0]) * rc)
    f = np.cos(al)[:, None] * ec + np.sin(al)[:, None] * el
    s = -np.sin(al)[:, None] * ec + np.cos(al)[:, None] * el
    return np.concatenate([f, s, nrm], axis=1)


def lumped_volume(mesh):
    """Nodal volume (row sums of the P1 mass matrix)."""
    vol = mesh.volumes()
    out = np.zeros(mesh.n)
    np.add.at(out, mesh.tets.ravel(), np.repeat(vol / 4.0, 4))
    return out


def corner_block(mesh, ni, nj, nk=None):
    """Node ids of the ni x nj x nk corner block of a slab (nk=None: all z)."""
    nx, ny, nz = mesh.meta["shape"]
    nk = nz if nk is None else nk
    i, j, k = np.meshgrid(np.arange(ni), np.arange(nj), np.arange(nk), indexing="ij")
    return (i + nx * (j + ny * k)).ravel().astype(np.int32)


def pmj_sites(mesh, count=200, seed=0, radius=0.1):
    """PMJ stimulus sites drawn uniformly (by area) on the endocardium.

    Returns (site_nodes, site_ball) where site_ball[i] is the array of nodes
    within ``radius`` cm of site i (the stimulated volume of one PMJ)."""
    rng = np.random.default_rng(seed)
    endo = mesh.meta["endo_nodes"]
    w = lumped_volume(mesh)[endo]
    w = w / w.sum()
    sites = rng.choice(endo, size=count, replace=False, p=w)
    from scipy.spatial import cKDTree
    tree = cKDTree(mesh.xyz)
    balls = [np.sort(np.asarray(b, dtype=np.int32))
             for b in tree.query_ball_point(mesh.xyz[sites], r=radius)]
    return sites.astype(np.int32), balls


def fibonacci_sphere(count, radius, center):
    """``count`` near-uniform points on a sphere (golden-angle spiral)."""
    k = np.arange(count) + 0.5
    z = 1.0 - 2.0 * k / count
    r = np.sqrt(1.0 - z * z)
    t = np.pi * (1.0 + 5 ** 0.5) * k
    pts = np.stack([r * np.cos(t), r * np.sin(t), z], axis=1) * radius
    return pts + np.asarray(center)[None, :]
