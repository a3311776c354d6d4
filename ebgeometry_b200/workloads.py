"""Seeded synthetic inputs of the mesh-SDF, nearest-neighbour and CSG-union workloads.

No dataset is read: every mesh, point set and query batch is generated from a seed with numpy's
PCG64 generator, so the same seed gives the same arrays in every process.

* ``displaced_icosphere(level, seed)`` -- an icosphere (12-vertex icosahedron, ``level`` rounds of
  4-to-1 midpoint subdivision, vertices projected to the sphere; 20 * 4**level triangles) whose
  vertices are moved radially by a seeded sum of 8 sinusoids of total amplitude <= 0.08.  The
  result is watertight, with counter-clockwise (outward) triangles.
* ``displaced_quad_sphere(n, seed)`` -- a cube subdivided into n x n quads per side, projected to
  the sphere and displaced the same way (6 n^2 outward quads, slightly non-planar);
  ``polygon_prism(k)`` -- a prism over a regular k-gon (two planar k-gon caps, k quads);
  ``mixed_polygon_sphere(n, seed)`` -- the quad sphere with every other quad split into two
  triangles.  Faces are (offsets, indices) pairs.
* ``uniform_points``, ``grid_points`` (cell centres, x fastest), ``band_points`` (within +-w of the
  surface along the face normal, triangles drawn by area).
* ``point_cloud`` -- half uniform in the unit cube, half from anisotropic Gaussian clusters.
* ``csg_scene`` -- spheres and posed displaced icospheres for the batched union.
"""
from __future__ import annotations

import numpy as np

_T = (1.0 + 5.0 ** 0.5) / 2.0
_ICO_V = np.array([[-1, _T, 0], [1, _T, 0], [-1, -_T, 0], [1, -_T, 0], [0, -1, _T], [0, 1, _T],
                   [0, -1, -_T], [0, 1, -_T], [_T, 0, -1], [_T, 0, 1], [-_T, 0, -1], [-_T, 0, 1]],
                  dtype=np.float64)
_ICO_F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                   [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                   [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)


def icosphere(level: int):
    """Unit icosphere: (vertices float64 (V,3), triangles int32 (20*4**level, 3))."""
    v = _ICO_V / np.linalg.norm(_ICO_V, axis=1, keepdims=True)
    f = _ICO_F.copy()
    for _ in range(level):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        key = np.minimum(e[:, 0], e[:, 1]) * nv + np.maximum(e[:, 0], e[:, 1])
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // nv, uk % nv
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1) + nv  # midpoint index of edges (0,1), (1,2), (2,0) per face
        ab, bc, ca = m[0], m[1], m[2]
        f = np.concatenate([np.stack([f[:, 0], ab, ca], 1), np.stack([f[:, 1], bc, ab], 1),
                            np.stack([f[:, 2], ca, bc], 1), np.stack([ab, bc, ca], 1)], axis=0)
        v = np.concatenate([v, mid], axis=0)
    return v, f.astype(np.int32)


def radial_field(seed: int, n_terms: int = 8, amplitude: float = 0.08):
    """Parameters of r(u) = 1 + sum_j a_j sin(w_j . u + phi_j), sum_j |a_j| = amplitude."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 1.0, n_terms)
    a *= amplitude / a.sum()
    a *= rng.choice([-1.0, 1.0], n_terms)
    d = rng.normal(size=(n_terms, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = d * rng.uniform(1.0, 6.0, (n_terms, 1))
    phi = rng.uniform(0.0, 2.0 * np.pi, n_terms)
    return a, w, phi


def displaced_icosphere(level: int, seed: int, radius: float = 1.0, amplitude: float = 0.08,
                        center=(0.0, 0.0, 0.0)):
    """Watertight icosphere with seeded radial displacement (see module docstring)."""
    v, f = icosphere(level)
    a, w, phi = radial_field(seed, 8, amplitude)
    r = 1.0 + (np.sin(v @ w.T + phi) * a).sum(axis=1)
    return (radius * r)[:, None] * v + np.asarray(center, np.float64), f


def _cube_quads(n: int):
    """Integer lattice points (coordinates in -n..n, step 2) and outward quads of a subdivided cube."""
    key, verts, quads = {}, [], []

    def vid(p):
        if p not in key:
            key[p] = len(verts)
            verts.append(p)
        return key[p]

    # (axis, sign) -> in-plane axes (b, c) with e_b x e_c = sign * e_axis (counter-clockwise outside)
    for a, s_, b, c in ((0, 1, 1, 2), (0, -1, 2, 1), (1, 1, 2, 0), (1, -1, 0, 2), (2, 1, 0, 1), (2, -1, 1, 0)):
        for i in range(n):
            for j in range(n):
                q = []
                for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                    p = [0, 0, 0]
                    p[a] = s_ * n
                    p[b] = 2 * (i + di) - n
                    p[c] = 2 * (j + dj) - n
                    q.append(vid(tuple(p)))
                quads.append(q)
    return np.array(verts, np.float64), np.array(quads, np.int64)


def displaced_quad_sphere(n: int, seed: int, radius: float = 1.0, amplitude: float = 0.08):
    """Quad sphere with seeded radial displacement: (vertices (V,3), (offsets, indices))."""
    v, q = _cube_quads(n)
    u = v / np.linalg.norm(v, axis=1, keepdims=True)
    a, w, phi = radial_field(seed, 8, amplitude)
    r = 1.0 + (np.sin(u @ w.T + phi) * a).sum(axis=1)
    off = np.arange(q.shape[0] + 1, dtype=np.int64) * 4
    return (radius * r)[:, None] * u, (off, q.ravel().astype(np.int32))


def mixed_polygon_sphere(n: int, seed: int):
    """The displaced quad sphere with every other quad split into two triangles."""
    v, (off, idx) = displaced_quad_sphere(n, seed)
    faces = []
    for k, qd in enumerate(idx.reshape(-1, 4)):
        if k % 2:
            faces += [[qd[0], qd[1], qd[2]], [qd[0], qd[2], qd[3]]]
        else:
            faces.append(list(qd))
    counts = np.array([len(f) for f in faces], np.int64)
    return v, (np.concatenate([[0], np.cumsum(counts)]).astype(np.int64),
               np.concatenate(faces).astype(np.int32))


def polygon_prism(k: int, radius: float = 1.0, height: float = 1.0):
    """A prism over a regular k-gon, centred at the origin: two k-gon caps and k side quads."""
    t = 2.0 * np.pi * np.arange(k) / k
    ring = np.stack([radius * np.cos(t), radius * np.sin(t)], 1)
    v = np.concatenate([np.c_[ring, np.full(k, -0.5 * height)], np.c_[ring, np.full(k, 0.5 * height)]])
    faces = [list(range(k - 1, -1, -1)), list(range(k, 2 * k))]
    faces += [[i, (i + 1) % k, k + (i + 1) % k, k + i] for i in range(k)]
    counts = np.array([len(f) for f in faces], np.int64)
    return v, (np.concatenate([[0], np.cumsum(counts)]).astype(np.int64), np.concatenate(faces).astype(np.int32))


def uniform_points(n: int, seed: int, lo=-1.5, hi=1.5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)


def grid_points(res: int, lo=-1.25, hi=1.25) -> np.ndarray:
    """Cell centres of a res^3 Cartesian grid over [lo, hi]^3, x fastest (float32 (res^3, 3))."""
    h = (hi - lo) / res
    c = (lo + h * (np.arange(res, dtype=np.float64) + 0.5)).astype(np.float32)
    out = np.empty((res, res, res, 3), np.float32)
    out[..., 0] = c[None, None, :]
    out[..., 1] = c[None, :, None]
    out[..., 2] = c[:, None, None]
    return out.reshape(-1, 3)


def band_points(v: np.ndarray, f: np.ndarray, n: int, seed: int, width: float = 1e-3) -> np.ndarray:
    """Points within +-width of the surface: triangle by area, uniform barycentric point, offset
    along the unit face normal by U(-width, width)."""
    rng = np.random.default_rng(seed)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    cr = np.cross(b - a, c - a)
    area = np.linalg.norm(cr, axis=1)
    nrm = cr / area[:, None]
    tri = rng.choice(f.shape[0], size=n, p=area / area.sum())
    r1, r2 = rng.random(n), rng.random(n)
    s = np.sqrt(r1)
    u, w = 1.0 - s, s * (1.0 - r2)
    p = u[:, None] * a[tri] + w[:, None] * b[tri] + (1.0 - u - w)[:, None] * c[tri]
    p += rng.uniform(-width, width, n)[:, None] * nrm[tri]
    return p.astype(np.float32)


def point_cloud(n: int, seed: int, n_clusters: int = 64) -> np.ndarray:
    """n float32 points in [0,1]^3: n//2 uniform, the rest from anisotropic Gaussian clusters
    (centres U[0,1]^3, per-axis sigma log-uniform in [0.002, 0.05], random rotation), clamped."""
    rng = np.random.default_rng(seed)
    nu = n // 2
    out = np.empty((n, 3), np.float32)
    out[:nu] = rng.random((nu, 3), dtype=np.float32)
    nc = n - nu
    lab = rng.integers(0, n_clusters, nc)
    cen = rng.random((n_clusters, 3))
    sig = np.exp(rng.uniform(np.log(0.002), np.log(0.05), (n_clusters, 3)))
    rot = np.linalg.qr(rng.normal(size=(n_clusters, 3, 3)))[0]
    z = rng.normal(size=(nc, 3)) * sig[lab]
    pts = np.einsum("nij,nj->ni", rot[lab], z) + cen[lab]
    out[nu:] = np.clip(pts, 0.0, 1.0).astype(np.float32)
    return out


def csg_scene(seed: int, n_spheres: int = 4096, n_meshes: int = 256, levels=(3, 7),
              mesh_radius=(0.03, 0.12)):
    """Spheres (centre U[-1,1]^3, radius log-uniform [0.001, 0.05]) and displaced icospheres of
    random level, radius, rotation (axis in {0,1,2}, angle U[0,360) degrees) and translation
    U[-1,1]^3.  Returns dict(spheres (S,4) float64, meshes [(V, F)], poses (M,5) float64 as
    (angle_deg, axis, tx, ty, tz))."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1, 1, (n_spheres, 3))
    r = np.exp(rng.uniform(np.log(0.001), np.log(0.05), n_spheres))
    spheres = np.concatenate([c, r[:, None]], axis=1)
    meshes, poses = [], []
    for m in range(n_meshes):
        lvl = int(rng.integers(levels[0], levels[1] + 1))
        rad = float(rng.uniform(*mesh_radius))
        v, f = displaced_icosphere(lvl, int(rng.integers(1 << 30)), radius=rad)
        meshes.append((v, f))
        poses.append([rng.uniform(0, 360), float(rng.integers(0, 3)), *rng.uniform(-1, 1, 3)])
    return dict(spheres=spheres, meshes=meshes, poses=np.asarray(poses, np.float64))


def rotate_points(p: np.ndarray, angle_deg: float, axis: int) -> np.ndarray:
    """RotateIF's point map (angle in degrees about one axis)."""
    th = angle_deg * np.pi / 180.0
    c, s = np.cos(th), np.sin(th)
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    out = p.copy()
    if axis == 0:
        out[..., 1], out[..., 2] = y * c + z * s, -y * s + z * c
    elif axis == 1:
        out[..., 0], out[..., 2] = x * c - z * s, x * s + z * c
    else:
        out[..., 0], out[..., 1] = x * c + y * s, -x * s + y * c
    return out
