"""Transport time steps on the device: solute (coupled_solver_v2.py) and nitrogen species (nitrogen_solver.py).

Each step assembles A = M/dt + K and b = M c_n/dt + F with the ADR row kernel
(``wspm_assemble_adr_2d``), adds the boundary-edge terms (``wspm_apply_edge_terms``)
and solves on the device with the Krylov kernels.  The Jacobi diagonal, when
asked for, is taken from the final matrix (after the edge terms), as the
reference builds its preconditioner from the matrix it solves.

  * ``solute_step``: consistent mass, Cauchy inflow
    (coupled_solver_v2.py:148-197);
  * ``nitrogen_species_step``: row-lumped mass, first-order decay, sorption,
    source from the upstream species, Cauchy inflow, free-drainage outflow
    (nitrogen_solver.py:151-305, assembly_nitrogen.py:33-606).
"""
import numpy as np
import torch

from .device import BoundaryEdges, SparseMatrix, apply_edge_terms, assemble_adr, jacobi_dinv, krylov_solve

EDGE_NEUMANN, EDGE_FREEDRAINAGE_WATER, EDGE_CAUCHY, EDGE_FREEDRAINAGE_NITROGEN = 0, 1, 2, 3
KRYLOV = ("cg", "bicgstab", "gmres")


def edges_or_none(dm, nodes):
    nodes = np.asarray(nodes if nodes is not None else [], dtype=np.int64)
    return BoundaryEdges(dm, nodes) if nodes.size > 1 else None


def _solve(dm, vals, rhs, x0, solver, precond, tol, maxiter, restart, workspace):
    if precond not in ("none", None, "jacobi"):
        raise NotImplementedError(f"preconditioner {precond!r} is not available on the device path")
    if solver == "direct":
        # dense solve, like the reference's jnp.linalg.solve (small systems only)
        A = SparseMatrix(dm, vals).todense().to(rhs.device)
        return torch.linalg.solve(A, rhs), None
    if solver not in KRYLOV:
        raise ValueError(f"Unsupported solver type: {solver}")
    dinv = jacobi_dinv(dm, vals) if precond == "jacobi" else None
    return krylov_solve(dm, vals, rhs, x0, solver, dinv=dinv, tol=tol, maxiter=maxiter, restart=restart,
                        workspace=workspace)


def solute_step(dm, c_n, theta, qx, qz, Dxx, Dxz, Dzz, dt, quad, cauchy_edges=None, cauchy_flux=0.0, c_in=0.0,
                solver="gmres", precond="none", tol=1e-10, maxiter=100, restart=30, workspace=None):
    """c^{n+1} of the solute equation; returns (c, krylov status tensor or None)."""
    Q, W = quad
    vals, rhs, _ = assemble_adr(dm, theta, qx, qz, Dxx, Dxz, Dzz, c_n, dt, Q, W, want_dinv=False)
    if cauchy_edges is not None:
        apply_edge_terms(dm, cauchy_edges, EDGE_CAUCHY, rhs, vals=vals, flux=cauchy_flux, c_in=c_in)
    return _solve(dm, vals, rhs, c_n, solver, precond, tol, maxiter, restart, workspace)


def nitrogen_species_step(dm, c_n, theta, qx, qz, Dxx, Dxz, Dzz, K_node, dt, quad, mu=0.0, sorption=0.0,
                          mu_up=0.0, c_up=None, cauchy_edges=None, cauchy_flux=0.0, c_in=0.0, fd_edges=None,
                          solver="gmres", precond="none", tol=1e-10, maxiter=100, restart=30, workspace=None):
    """c^{n+1} of one nitrogen species; returns (c, krylov status tensor or None)."""
    Q, W = quad
    vals, rhs, _ = assemble_adr(dm, theta, qx, qz, Dxx, Dxz, Dzz, c_n, dt, Q, W, mu=mu, sorption=sorption,
                                mu_up=mu_up, c_up=c_up, lumped=True, want_dinv=False)
    if cauchy_edges is not None:
        apply_edge_terms(dm, cauchy_edges, EDGE_CAUCHY, rhs, vals=vals, flux=cauchy_flux, c_in=c_in)
    if fd_edges is not None:
        apply_edge_terms(dm, fd_edges, EDGE_FREEDRAINAGE_NITROGEN, rhs, vals=vals, K=K_node, theta=theta)
    return _solve(dm, vals, rhs, c_n, solver, precond, tol, maxiter, restart, workspace)
