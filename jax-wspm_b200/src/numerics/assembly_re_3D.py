"""Richards assembly on tetrahedra (drop-in for src/numerics/assembly_re_3D.py:72-169).

Same kernel as the triangle path (``wspm_assemble_richards`` with dim 3):
4x4 element matrices, gravity on z, fixed-pattern scatter.
"""
import numpy as np

from wspm_b200 import context
from wspm_b200.device import SparseMatrix, assemble_richards


def assemble_global_matrices_sparse_3D(tetrahedra, nnt, points, theta_m, theta_n, pressure_head_m,
                                       conductivity_m, capacity_m, quad_points, weights, dt):
    dm = context.mesh_for(points, tetrahedra)
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
