"""Preconditioners and Krylov solvers (drop-in for src/solvers/jax_linear_solver.py:8-329).

Same class and method names.  With no preconditioner or Jacobi the solves
run as CUDA graphs in libwspm.so (``wspm_krylov_solve``): the whole Krylov
loop, including its convergence test, stays on the device.  ``ilu``, ``ssor``
and ``block_jacobi`` are the reference's own operators as its code computes
them (jax_linear_solver.py:38-252: ilu is the symmetric Gauss-Seidel form,
ssor a scaled forward sweep), applied on the device with level-scheduled
triangular sweeps (``wspm_b200.precond``); their Krylov loops are driven from
the host.
"""
from typing import Optional, Tuple

import torch

from wspm_b200 import context
from wspm_b200 import precond as _pre
from wspm_b200.device import KrylovWorkspace, SparseMatrix, jacobi_dinv, krylov_solve


class Preconditioner:
    @staticmethod
    def create_jacobi(A: SparseMatrix):
        """x -> x / diag(A), zero diagonals replaced by 1 (jax_linear_solver.py:11-36)."""
        dinv = getattr(A, "dinv", None)
        if dinv is None:
            dinv = jacobi_dinv(A.dmesh, A.vals)
        fn = lambda x: dinv * x  # noqa: E731
        fn.dinv = dinv
        return fn

    @staticmethod
    def create_block_jacobi(A, block_size: int = 2):
        """Inverses of the diagonal blocks (+ 1e-12 I), jax_linear_solver.py:38-89."""
        return _pre.ReferencePreconditioner(A.dmesh, A.vals, "block_jacobi", block_size=block_size)

    @staticmethod
    def create_ssor(A, omega: float = 1.0):
        """omega (D/omega + L)^-1, what jax_linear_solver.py:91-169 computes."""
        return _pre.ReferencePreconditioner(A.dmesh, A.vals, "ssor", omega=omega)

    @staticmethod
    def create_ilu0(A):
        """(D' + U)^-1 (I + L D'^-1)^-1, what jax_linear_solver.py:171-252 computes."""
        return _pre.ReferencePreconditioner(A.dmesh, A.vals, "ilu")


def _workspace(A):
    ws = getattr(A.dmesh, "_krylov_ws", None)
    if ws is None:
        ws = KrylovWorkspace(A.dmesh)
        A.dmesh._krylov_ws = ws
    return ws


class JAXSparseSolver:
    """Same interface as the reference's class; returns (x, info) with info = (status, iterations)."""

    def __init__(self, A: SparseMatrix):
        if not isinstance(A, SparseMatrix):
            raise TypeError("A must be a wspm_b200 SparseMatrix")
        self.A = A

    def _dinv(self, precond_type, **kw):
        if precond_type in (None, "none"):
            return None
        if precond_type == "jacobi":
            return Preconditioner.create_jacobi(self.A).dinv
        raise ValueError(f"Unsupported preconditioner: {precond_type}")

    def _solve(self, solver, b, x0, tol, atol, maxiter, restart, precond_type, **kw):
        b = context.as_cuda_f64(b)
        x0 = b.new_zeros(b.shape) if x0 is None else context.as_cuda_f64(x0)
        if maxiter is None:
            maxiter = 10 * b.numel()
        if precond_type in ("ilu", "ssor", "block_jacobi"):
            x, k = _pre.solve(self.A.dmesh, self.A.vals, b, x0, solver, precond_type, tol=tol, atol=atol,
                              maxiter=maxiter, restart=restart, omega=kw.get("omega", 1.0),
                              block_size=kw.get("block_size", 2))
            status = 3 if k < 0 else (1 if k >= maxiter else 0)
            return x, torch.tensor([status, max(k, 0), 0, 0], dtype=torch.int32, device=b.device)
        x, res = krylov_solve(self.A.dmesh, self.A.vals, b, x0, solver=solver, dinv=self._dinv(precond_type, **kw),
                              tol=tol, atol=atol, maxiter=maxiter, restart=restart, workspace=_workspace(self.A))
        return x, res

    def solve_cg(self, b, x0=None, tol: float = 1e-5, atol: float = 0.0, maxiter: Optional[int] = None,
                 precond_type: Optional[str] = None, **precond_kwargs) -> Tuple[torch.Tensor, torch.Tensor]:
        return self._solve("cg", b, x0, tol, atol, maxiter, 0, precond_type, **precond_kwargs)

    def solve_bicgstab(self, b, x0=None, tol: float = 1e-5, atol: float = 0.0, maxiter: Optional[int] = None,
                       precond_type: Optional[str] = None, **precond_kwargs):
        return self._solve("bicgstab", b, x0, tol, atol, maxiter, 0, precond_type, **precond_kwargs)

    def solve_gmres(self, b, x0=None, tol: float = 1e-5, atol: float = 0.0, restart: int = 20,
                    maxiter: Optional[int] = None, precond_type: Optional[str] = None, **precond_kwargs):
        return self._solve("gmres", b, x0, tol, atol, maxiter, restart, precond_type, **precond_kwargs)
