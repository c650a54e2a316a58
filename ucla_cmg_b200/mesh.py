"""Synthetic linear-tet meshes, fibres, cell-type maps and stimulus sites.

The reference reads its geometry from ``.node/.ele/.fibers/.cell`` files
(voomEP/src/Mesh/Mesh.cc:142-483).  The workloads here are generated:

* :func:`slab` -- a box of ``nx*ny*nz`` nodes, every hexahedron split into 6
  tetrahedra along its main diagonal (Kuhn split, conforming), with the fibre
  angle rotating linearly through the thickness;
* :func:`shell` -- a truncated prolate-ellipsoid shell (a ventricle-like
  wall) built from a structured (phi, theta, rho) grid whose apex column is
  collapsed onto one node per transmural layer.

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


def shell(n_phi=480, n_theta=200, n_rho=20, a_in=2.5, c_in=5.0, wall=1.0, z_base=2.0,
          helix_deg=(60.0, -60.0)):
    """Truncated prolate-ellipsoid shell.

    Inner surface x^2/a^2 + y^2/a^2 + z^2/c^2 = 1 with (a, c) = (a_in, c_in),
    outer surface with (a_in + wall, c_in + wall); apex at z = -c, cut by the
    base plane z = ``z_base``.  Grid: ``n_phi`` nodes around, ``n_theta``
    intervals apex->base, ``n_rho`` intervals endo->epi; the apex column
    (theta = 0) is one node per layer and the degenerate tets there are
    dropped.  Fibres: helix angle rotating linearly endo->epi in the plane of
    the circumferential and longitudinal directions.
    meta["rho"] (per node, 0 endo .. 1 epi) and meta["height"] (0 apex .. 1
    base) feed the transmural and apicobasal parameter maps.
    """
    rho = np.linspace(0.0, 1.0, n_rho + 1)
    a = a_in + wall * rho
    c = c_in + wall * rho
    tmax = np.arccos(-z_base / c)                     # per layer
    u = np.linspace(0.0, 1.0, n_theta + 1)            # fraction apex->base
    phi = np.linspace(0.0, 2.0 * np.pi, n_phi, endpoint=False)
    # node numbering: apex node of layer k = k; ring nodes afterwards
    n_apex = n_rho + 1
    def nid(ip, jt, kr):
        ip = np.asarray(ip) % n_phi
        return np.where(jt == 0, kr, n_apex + ((kr * n_theta + (jt - 1)) * n_phi + ip))
    # coordinates
    xyz = np.zeros((n_apex + (n_rho + 1) * n_theta * n_phi, 3))
    xyz[:n_apex, 2] = -c
    K, J, I = np.meshgrid(np.arange(n_rho + 1), np.arange(1, n_theta + 1), np.arange(n_phi), indexing="ij")
    th = u[J] * tmax[K]
    ids = n_apex + (K * n_theta + (J - 1)) * n_phi + I
    xyz[ids.ravel(), 0] = (a[K] * np.sin(th) * np.cos(phi[I])).ravel()
    xyz[ids.ravel(), 1] = (a[K] * np.sin(th) * np.sin(phi[I])).ravel()
    xyz[ids.ravel(), 2] = (-c[K] * np.cos(th)).ravel()
    # hex cells (phi, theta, rho) -> Kuhn tets, collapsing theta=0
    ip, jt, kr = np.meshgrid(np.arange(n_phi), np.arange(n_theta), np.arange(n_rho), indexing="ij")
    ip, jt, kr = ip.ravel(), jt.ravel(), kr.ravel()
    tets = []
    for path in _kuhn_local():
        tets.append(np.stack([nid(ip + cc[0], jt + cc[1], kr + cc[2]) for cc in path], axis=1))
    tets = np.concatenate(tets, axis=0).astype(np.int64)
    # drop tets with repeated vertices (apex collapse)
    srt = np.sort(tets, axis=1)
    keep = np.all(srt[:, 1:] != srt[:, :-1], axis=1)
    tets = tets[keep].astype(np.int32)
    tets, vol = _orient(xyz, tets)
    good = vol > 1e-14
    tets = tets[good]
    # per-node transmural depth and height
    rho_n = np.zeros(len(xyz)); rho_n[:n_apex] = rho
    rho_n[ids.ravel()] = rho[K].ravel()
    zmin = -c[0]
    height = np.clip((xyz[:, 2] - zmin) / (z_base - zmin), 0.0, 1.0)
    fib = None
    if helix_deg is not None:
        cen = xyz[tets].mean(axis=1)
        rc = rho_n[tets].mean(axis=1)
        # circumferential direction (about z) and the local outward normal of
        # the ellipsoid family through the centroid
        r_xy = np.hypot(cen[:, 0], cen[:, 1])
        ec = np.stack([-cen[:, 1], cen[:, 0], np.zeros(len(cen))], axis=1)
        near_axis = r_xy < 1e-9
        ec[near_axis] = np.array([1.0, 0.0, 0.0])
        ec /= np.linalg.norm(ec, axis=1, keepdims=True)
        ae = a_in + wall * rc
        ce = c_in + wall * rc
        nrm = np.stack([cen[:, 0] / ae ** 2, cen[:, 1] / ae ** 2, cen[:, 2] / ce ** 2], axis=1)
        nrm -= np.einsum("ij,ij->i", nrm, ec)[:, None] * ec
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        el = np.cross(nrm, ec)                          # longitudinal (tangent)
        al = np.deg2rad(helix_deg[0] + (helix_deg[1] - helix_deg[0]) * rc)
        f = np.cos(al)[:, None] * ec + np.sin(al)[:, None] * el
        s = -np.sin(al)[:, None] * ec + np.cos(al)[:, None] * el
        fib = np.concatenate([f, s, nrm], axis=1)
    meta = dict(kind="shell", rho=rho_n, height=height, n_phi=n_phi, n_theta=n_theta,
                n_rho=n_rho, endo_nodes=np.where(rho_n == 0.0)[0], z_base=z_base)
    return TetMesh(xyz, tets, fib, meta)


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
    balls = []
    for s in sites:
        d = np.linalg.norm(mesh.xyz - mesh.xyz[s], axis=1)
        balls.append(np.where(d <= radius)[0].astype(np.int32))
    return sites.astype(np.int32), balls


def fibonacci_sphere(count, radius, center):
    """``count`` near-uniform points on a sphere (golden-angle spiral)."""
    k = np.arange(count) + 0.5
    z = 1.0 - 2.0 * k / count
    r = np.sqrt(1.0 - z * z)
    t = np.pi * (1.0 + 5 ** 0.5) * k
    pts = np.stack([r * np.cos(t), r * np.sin(t), z], axis=1) * radius
    return pts + np.asarray(center)[None, :]
