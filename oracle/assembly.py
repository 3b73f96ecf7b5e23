"""Element and global assembly (oracle restatement, vectorised over elements).

Richards mixed form: src/numerics/assembly_re_v2.py:13-166 (triangles) and
src/numerics/assembly_re_3D.py:12-169 (tetrahedra).  The per-quadrature-point
accumulation order of the reference (``lax.scan`` over the rule) is kept;
the global matrix is a SciPy CSR matrix (duplicates summed, like
``BCOO.sum_duplicates``) and the right-hand side is scattered element by
element in element order (``lax.fori_loop`` at assembly_re_v2.py:156-164).
"""
import numpy as np
import scipy.sparse as sp

from .quadrature import TRI3_POINTS, TRI3_WEIGHTS, TET4_POINTS, TET4_WEIGHTS, TRI_DREF, TET_DREF


def _geometry(coords, dref):
    """Per element: (G = J^-1 dN/dref, det J).  coords (E, nv, d)."""
    J = np.einsum("ij,ejk->eik", dref, coords)           # (E, d, d)
    detJ = np.linalg.det(J)
    G = np.linalg.inv(J) @ dref                           # (E, d, nv)
    return G, detJ


def local_matrices_mixed_form(coords, theta_m, theta_0, h_m, K, C, dt, dim=2):
    """Element matrices and sources of the mass-lumped mixed form.

    coords (E, nv, dim); nodal fields (E, nv).  Returns (A_e (E,nv,nv), b_e (E,nv)).
    Restates compute_local_matrices_mixed_form (assembly_re_v2.py:13-60) and
    compute_local_matrices_3D_mixed_form (assembly_re_3D.py:12-70): gravity uses
    the last gradient component (G[1] in 2D, G[2] in 3D).
    """
    if dim == 2:
        Q, W, dref, shape = TRI3_POINTS, TRI3_WEIGHTS, TRI_DREF, lambda p: np.array([1 - p[0] - p[1], p[0], p[1]])
    else:
        Q, W, dref, shape = TET4_POINTS, TET4_WEIGHTS, TET_DREF, \
            lambda p: np.array([1.0 - p[0] - p[1] - p[2], p[0], p[1], p[2]])
    E, nv = theta_m.shape
    G, detJ = _geometry(coords, dref)
    GtG = np.einsum("eki,ekj->eij", G, G)
    stiff = np.zeros((E, nv, nv))
    mass = np.zeros((E, nv, nv))
    src = np.zeros((E, nv))
    for q in range(len(W)):
        N = shape(Q[q])
        w = W[q]
        NK = K @ N
        stiff += w * NK[:, None, None] * GtG * detJ[:, None, None]
        mass += w * np.outer(N, N)[None] * detJ[:, None, None]
        src -= w * NK[:, None] * G[:, dim - 1, :] * detJ[:, None]
    Ml = mass.sum(axis=2)
    A = stiff.copy()
    idx = np.arange(nv)
    A[:, idx, idx] = (1 / dt) * (Ml * C) + stiff[:, idx, idx]
    b = src - (1 / dt) * (Ml * (theta_m - theta_0 - C * h_m))
    return A, b


def scatter_global(elements, nnt, A_e, b_e):
    """COO fill + sum_duplicates (assembly_re_v2.py:114-152) and ordered RHS scatter (:156-164)."""
    E, nv = elements.shape
    rows = np.repeat(elements, nv, axis=1).ravel()
    cols = np.tile(elements, (1, nv)).ravel()
    A = sp.coo_matrix((A_e.ravel(), (rows, cols)), shape=(nnt, nnt)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    b = np.zeros(nnt)
    np.add.at(b, elements.ravel(), b_e.ravel())
    return A, b


def assemble_richards(elements, nnt, points, theta_m, theta_n, h_m, K_node, C, dt, Ks_elem=None):
    """Global (A, b) for Richards; assemble_global_matrices_sparse_re / _3D.

    ``K_node`` is the nodal conductivity.  With ``Ks_elem`` given, element e
    uses ``Ks_elem[e] * K_node[nodes]`` (per-element saturated conductivity;
    ``K_node`` then holds the relative conductivity K/Ks).
    """
    elements = np.asarray(elements)
    dim = points.shape[1]
    coords = points[elements]
    Ke = K_node[elements]
    if Ks_elem is not None:
        Ke = Ks_elem[:, None] * Ke
    A_e, b_e = local_matrices_mixed_form(coords, theta_m[elements], theta_n[elements],
                                         h_m[elements], Ke, C[elements], dt, dim=dim)
    return scatter_global(elements, nnt, A_e, b_e)


def apply_dirichlet_rows(A, b, nodes, values):
    """Row replacement A[i,:] = e_i, b[i] = g (boundary.py:38-53; sparse twin :603-648).

    Columns are left untouched (the reference zeroes rows only), so the
    system stays non-symmetric exactly like the reference's.
    """
    A = A.tocsr(copy=True)
    b = b.copy()
    nodes = np.asarray(nodes, dtype=np.int64)
    if nodes.size == 0:
        return A, b
    mask = np.zeros(A.shape[0], dtype=bool)
    mask[nodes] = True
    row_of = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    sel = mask[row_of]
    A.data[sel] = 0.0
    A.data[sel & (A.indices == row_of)] = 1.0
    b[nodes] = values
    return A, b
