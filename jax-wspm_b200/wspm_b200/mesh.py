"""Mesh input: the reference's CSV loader and structured generators.

``load_csv_mesh`` follows src/mesh/loader.py:11-108 (points as float64,
1-based connectivity converted to 0-based, shape and index validation with
the same errors).  The generators reproduce the reference's structured
meshes bit for bit (checked against digests of data/mesh/**):

* ``structured_triangles(n, L)``: (n+1)^2 nodes in x-fastest order; each cell
  with lower-left node a gives triangles (a, a+1, a+n+2), (a, a+n+2, a+n+1)
  (data/mesh/richards/t50.csv:1-2).
* ``kuhn_tetrahedra(n, L)``: (n+1)^3 nodes x-fastest; each hex is split into
  6 tetrahedra around its (0,0,0)-(1,1,1) diagonal, in the vertex order of
  data/mesh/richards/t_3D.csv:1-6 (all positively oriented).

Coordinates are the decimal values the reference files hold: i*L/n rounded
to 12 significant digits, then parsed as float64 (exactly what reading the
CSV gives).
"""
import os

import numpy as np


def _coords_1d(n, L):
    return np.array([float(f"{i * (L / n):.12g}") for i in range(n + 1)], dtype=np.float64)


def structured_triangles(n, L=1.0):
    """(points (N,2) float64, triangles (2n^2, 3) int64)."""
    c = _coords_1d(n, L)
    X, Y = np.meshgrid(c, c, indexing="xy")
    points = np.stack([X.ravel(), Y.ravel()], axis=1)
    j, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a = (j * (n + 1) + i).ravel()
    t1 = np.stack([a, a + 1, a + n + 2], axis=1)
    t2 = np.stack([a, a + n + 2, a + n + 1], axis=1)
    tri = np.stack([t1, t2], axis=1).reshape(-1, 3)
    return points, tri.astype(np.int64)


# corner (di, dj, dk) lists of the 6 tetrahedra of one hex (t_3D.csv:1-6)
_KUHN = [((0, 0, 1), (0, 0, 0), (0, 1, 1), (1, 1, 1)),
         ((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1)),
         ((1, 0, 0), (0, 0, 0), (1, 0, 1), (1, 1, 1)),
         ((0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1)),
         ((0, 1, 0), (0, 0, 0), (1, 1, 0), (1, 1, 1)),
         ((0, 0, 0), (0, 1, 0), (0, 1, 1), (1, 1, 1))]


def kuhn_tetrahedra(n, L=1.0):
    """(points (N,3) float64, tets (6n^3, 4) int64)."""
    c = _coords_1d(n, L)
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    n1 = n + 1
    k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = (k * n1 * n1 + j * n1 + i).ravel()
    tets = np.empty((base.size, 6, 4), dtype=np.int64)
    for t, corners in enumerate(_KUHN):
        for v, (di, dj, dk) in enumerate(corners):
            tets[:, t, v] = base + dk * n1 * n1 + dj * n1 + di
    return points, tets.reshape(-1, 4)


def load_csv_mesh(p_file, t_file, dim):
    """Points/elements from the reference's CSV format (loader.py:64-91)."""
    if not os.path.exists(p_file):
        raise FileNotFoundError(f"Points file not found: {p_file}")
    if not os.path.exists(t_file):
        raise FileNotFoundError(f"Elements file not found: {t_file}")
    points = np.loadtxt(p_file, delimiter=",", dtype=np.float64, ndmin=2)
    elements = np.loadtxt(t_file, delimiter=",", dtype=np.int64, ndmin=2) - 1
    if dim == 3:
        if points.ndim != 2 or points.shape[1] != 3:
            raise ValueError("Points array must have 3 columns (x, y, z coordinates) for 3D mesh")
        if elements.ndim != 2 or elements.shape[1] != 4:
            raise ValueError("Elements array must have 4 columns (vertex indices) for tetrahedral mesh")
    else:
        if points.ndim != 2 or points.shape[1] != 2:
            raise ValueError("Points array must have 2 columns (x, y coordinates) for 2D mesh")
        if elements.ndim != 2 or elements.shape[1] != 3:
            raise ValueError("Elements array must have 3 columns (vertex indices) for triangular mesh")
    if np.any(elements < 0) or np.any(elements >= len(points)):
        raise ValueError("Element indices out of bounds")
    return points, elements


def validate_elements(points, elements):
    """Host-side validation run before any device upload (index range, degeneracy)."""
    points = np.asarray(points)
    elements = np.asarray(elements)
    if elements.ndim != 2 or elements.shape[1] != points.shape[1] + 1:
        raise ValueError("elements must have dim+1 columns")
    if elements.size and (elements.min() < 0 or elements.max() >= points.shape[0]):
        raise ValueError("Element indices out of bounds")
    return True


KS_MEAN = 0.0922       # m/day, the van Genuchten unit-square soil's saturated conductivity


def lognormal_ks_square(n, seed, sigma_lnk=1.0, ks_mean=KS_MEAN):
    """The 1024^2-style Richards workload on an n x n unit square: (points, triangles, Ks per element, top nodes).

    Per-element saturated conductivity ln Ks ~ N(ln ks_mean, sigma_lnk^2), i.i.d., drawn with
    numpy.random.default_rng(seed); the top nodes (y == 1) carry the Dirichlet value."""
    pts, tri = structured_triangles(n, 1.0)
    rng = np.random.default_rng(seed)
    Ks = np.exp(np.log(ks_mean) + sigma_lnk * rng.standard_normal(len(tri)))
    top = np.where(pts[:, 1] == 1.0)[0]
    return pts, tri, Ks, top


def vg_parameter_ensemble(n_domains, seed, sides=tuple(range(32, 257, 16))):
    """Independent unit-square Richards domains of uneven size for the batched ensemble: side lengths drawn
    uniformly from {32, 48, ..., 256}; van Genuchten alpha, n, Ks log-uniform in [1, 10] 1/m, [1.3, 3],
    [0.01, 1] m/day, m = 1 - 1/n, theta_r .05, theta_s .40; Dirichlet -0.1 on the top edge (NaN = free).
    Returns [(points, triangles, phi, bc_val, None)] (the Ensemble's domain tuples); meshes of equal side are
    shared."""
    rng = np.random.default_rng(seed)
    lu = lambda lo, hi: float(np.exp(rng.uniform(np.log(lo), np.log(hi))))  # noqa: E731
    cache, doms = {}, []
    for _ in range(n_domains):
        s = int(rng.choice(sides))
        if s not in cache:
            pts, tri = structured_triangles(s, 1.0)
            bc = np.full(len(pts), np.nan)
            bc[np.abs(pts[:, 1] - 1.0) < 1e-12] = -0.1
            cache[s] = (pts, tri, bc)
        pts, tri, bc = cache[s]
        n = lu(1.3, 3.0)
        doms.append((pts, tri, (lu(1.0, 10.0), 0.40, 0.05, n, 1.0 - 1.0 / n, lu(0.01, 1.0)), bc, None))
    return doms
