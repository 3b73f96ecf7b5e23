"""Richards assembly on triangles (drop-in for src/numerics/assembly_re_v2.py:62-166).

``assemble_global_matrices_sparse_re`` keeps the reference's signature and
returns ``(A, b)``: A is a ``wspm_b200.device.SparseMatrix`` (SELL-32 on the
GPU; ``A @ x``, ``A.todense()``, ``A.to_scipy()``), b a CUDA float64 tensor.
The whole assembly is one kernel (libwspm.so ``wspm_assemble_richards``):
element matrices, the fixed-pattern scatter and the Jacobi diagonal; the
reference's sequential COO fill and ``sum_duplicates`` are not needed because
the pattern is built once per mesh.
"""
import numpy as np

from wspm_b200 import context
from wspm_b200.device import SparseMatrix, assemble_richards


def assemble_global_matrices_sparse_re(triangles, nnt, points, theta_m, theta_n, pressure_head_m,
                                       conductivity_m, capacity_m, quad_points, weights, dt):
    dm = context.mesh_for(points, triangles)
    if int(nnt) != dm.n_nodes:
        raise ValueError(f"nnt={nnt} does not match the mesh ({dm.n_nodes} nodes)")
    vals, rhs, dinv, _ = assemble_richards(
        dm, context.as_cuda_f64(theta_m), context.as_cuda_f64(theta_n), context.as_cuda_f64(pressure_head_m),
        context.as_cuda_f64(conductivity_m), context.as_cuda_f64(capacity_m),
        np.asarray(context.as_host(quad_points), dtype=np.float64),
        np.asarray(context.as_host(weights), dtype=np.float64), float(dt))
    A = SparseMatrix(dm, vals)
    A.dinv = dinv
    return A, rhs


def compute_local_matrices_mixed_form(local_coordinates, local_theta_m, local_theta_0, local_pressure_head,
                                      local_conductivity, local_capacity, quad_points, weights, dt):
    """Element matrix and source of one triangle (host; for inspection and tests)."""
    X = np.asarray(local_coordinates, dtype=np.float64)
    B = np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]])
    J = B @ X
    G = np.linalg.inv(J) @ B
    det = np.linalg.det(J)
    K = np.asarray(local_conductivity, dtype=np.float64)
    stiff, mass, src = np.zeros((3, 3)), np.zeros((3, 3)), np.zeros(3)
    for (ks, et), w in zip(np.asarray(quad_points), np.asarray(weights)):
        N = np.array([1 - ks - et, ks, et])
        nk = N @ K
        stiff += w * nk * (G.T @ G) * det
        mass += w * np.outer(N, N) * det
        src -= w * nk * G[1] * det
    Ml = mass.sum(axis=1)
    C = np.asarray(local_capacity, dtype=np.float64)
    A = (1 / dt) * np.diag(Ml * C) + stiff
    b = src - (1 / dt) * (Ml * (np.asarray(local_theta_m) - np.asarray(local_theta_0) - C * np.asarray(local_pressure_head)))
    return A, b
