"""Linear-solver dispatch (drop-in for src/solvers/solver_types.py:7-67).

``solve_system(matrix, rhs, x0, solver_config) -> (x, convergence)``.  The
second value is a CUDA int32 tensor [status, iterations, 0, 0] (the reference
returns JAX's ignored ``info``); status 1 means the iteration cap was hit,
which the reference silently ignores.  ``direct`` densifies like the
reference (solver_types.py:60-63) and is limited to small systems.
"""
import torch

from wspm_b200 import context

from .jax_linear_solver import JAXSparseSolver

DIRECT_MAX_ROWS = 20000


def solve_system(matrix, rhs, x0, solver_config):
    solver = JAXSparseSolver(matrix)
    precond = solver_config.precond_type if solver_config.precond_type != "none" else None
    kw = dict(solver_config.precond_params or {})
    st = solver_config.solver_type
    if st == "gmres":
        return solver.solve_gmres(rhs, x0=x0, tol=solver_config.tol, restart=solver_config.restart,
                                  maxiter=solver_config.maxiter, precond_type=precond, **kw)
    if st == "bicgstab":
        return solver.solve_bicgstab(rhs, x0=x0, tol=solver_config.tol, maxiter=solver_config.maxiter,
                                     precond_type=precond, **kw)
    if st == "cg":
        return solver.solve_cg(rhs, x0=x0, tol=solver_config.tol, maxiter=solver_config.maxiter,
                               precond_type=precond, **kw)
    if st == "direct":
        if matrix.shape[0] > DIRECT_MAX_ROWS:
            raise NotImplementedError(f"direct solve is dense (O(N^3)); limited to {DIRECT_MAX_ROWS} rows")
        dense = matrix.todense().to(device=context.device())
        x = torch.linalg.solve(dense, context.as_cuda_f64(rhs))
        return x, torch.zeros(4, dtype=torch.int32, device=x.device)
    raise ValueError(f"Unsupported solver type: {st}")
