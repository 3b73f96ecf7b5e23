"""Preconditioners and Krylov solvers (drop-in for src/solvers/jax_linear_solver.py:8-329).

Same class and method names.  The solves run as CUDA graphs in libwspm.so
(``wspm_krylov_solve``): the whole Krylov loop, including its convergence
test, stays on the device.  Jacobi is the only preconditioner of the hot
path; ``block_jacobi``, ``ssor`` and ``ilu`` raise NotImplementedError (the
reference builds them with sequential scans over the nonzeros, see
jax_linear_solver.py:38-252; they are the next items to port).
"""
from typing import Optional, Tuple

import torch

from wspm_b200 import context
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
    def _unsupported(name):
        raise NotImplementedError(f"preconditioner {name!r} is not implemented on the GPU path "
                                  "(supported: 'none', 'jacobi')")

    @staticmethod
    def create_block_jacobi(A, block_size: int = 2):
        Preconditioner._unsupported("block_jacobi")

    @staticmethod
    def create_ssor(A, omega: float = 1.0):
        Preconditioner._unsupported("ssor")

    @staticmethod
    def create_ilu0(A):
        Preconditioner._unsupported("ilu")


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
        if precond_type == "block_jacobi":
            return Preconditioner.create_block_jacobi(self.A, kw.get("block_size", 2))
        if precond_type == "ssor":
            return Preconditioner.create_ssor(self.A, kw.get("omega", 1.0))
        if precond_type == "ilu":
            return Preconditioner.create_ilu0(self.A)
        raise ValueError(f"Unsupported preconditioner: {precond_type}")

    def _solve(self, solver, b, x0, tol, atol, maxiter, restart, precond_type, **kw):
        b = context.as_cuda_f64(b)
        x0 = b.new_zeros(b.shape) if x0 is None else context.as_cuda_f64(x0)
        if maxiter is None:
            maxiter = 10 * b.numel()
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
