"""The reference's ILU / SSOR / block-Jacobi preconditioners and Krylov solvers that accept them.

``ReferencePreconditioner`` applies create_ilu0 / create_ssor / create_block_jacobi
(src/solvers/jax_linear_solver.py:38-252) as their code computes them, on the
device (``wspm_precond_apply``; triangular sweeps level scheduled); kind
``"ilu0"`` is a true ILU(0) on A's pattern (``wspm_ilu0_factor``), which the
reference's ``ilu`` is not.  The
solvers below follow jax.scipy.sparse.linalg's cg / bicgstab / gmres with a
general preconditioner -- the same recurrences and stopping rules as the
device-resident Jacobi path (JAX: with a preconditioner CG tests r.r; GMRES is
left preconditioned and tests ||M r||) -- driven from the host on device
vectors: each iteration reads its scalars back, so this path is for the
preconditioners whose sweeps are sequential anyway, not for throughput.
"""
import ctypes

import torch

from . import _lib
from ._lib import check, dptr, lib
from .device import spmv


class ReferencePreconditioner:
    def __init__(self, dm, vals, kind, omega=1.0, block_size=2):
        if kind not in _lib.PRECOND_KIND:
            raise ValueError(f"unknown preconditioner {kind!r}")
        self.dm, self.vals, self.kind = dm, vals, _lib.PRECOND_KIND[kind]
        self.omega, self.block_size = float(omega), int(block_size)
        if kind == "block_jacobi" and self.block_size not in (1, 2):
            raise NotImplementedError("block_jacobi: block_size 1 or 2 on the device path")
        self.lower = self.upper = None
        if kind in ("ilu", "ssor", "ilu0"):
            self.lower = self._levels(True)
        if kind in ("ilu", "ilu0"):
            self.upper = self._levels(False)
        self.tmp = dm.vec()
        if kind == "ilu0":
            # true ILU(0): factor once on the device, then apply the two sweeps with the factors
            self.vals = dm.empty_vals()
            check("ilu0_factor", lib.wspm_ilu0_factor(ctypes.byref(dm.c_pat), dptr(vals), ctypes.byref(self.lower),
                                                      dptr(self.vals),
                                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def _levels(self, lower):
        cache = self.dm.__dict__.setdefault("_tri_levels", {})
        if lower not in cache:
            ptr, rows = self.dm.pattern.tri_levels(lower)
            t_ptr = torch.as_tensor(ptr, device=self.dm.device)
            t_rows = torch.as_tensor(rows, device=self.dm.device)
            c = _lib.WspmLevels(len(ptr) - 1, t_ptr.data_ptr(), t_rows.data_ptr())
            cache[lower] = (c, t_ptr, t_rows)
        return cache[lower][0]

    def __call__(self, v):
        y = torch.empty_like(v)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        check("precond_apply", lib.wspm_precond_apply(
            ctypes.byref(self.dm.c_pat), dptr(self.vals), self.kind, self.omega, self.block_size,
            ctypes.byref(self.lower) if self.lower is not None else None,
            ctypes.byref(self.upper) if self.upper is not None else None, dptr(v), dptr(y), dptr(self.tmp), st))
        return y


def _dot(a, b):
    return float(torch.dot(a, b))


def cg(A, b, x0, M, tol=1e-10, atol=0.0, maxiter=100):
    bs = _dot(b, b)
    atol2 = max(tol * tol * bs, atol * atol)
    x = x0.clone()
    r = b - A(x)
    z = M(r)
    p = z.clone()
    gamma = _dot(r, z)
    k = 0
    while _dot(r, r) > atol2 and k < maxiter:
        Ap = A(p)
        alpha = gamma / _dot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = M(r)
        gamma_new = _dot(r, z)
        beta = gamma_new / gamma
        gamma = gamma_new
        p = z + beta * p
        k += 1
    return x, k


def bicgstab(A, b, x0, M, tol=1e-10, atol=0.0, maxiter=100):
    bs = _dot(b, b)
    atol2 = max(tol * tol * bs, atol * atol)
    x = x0.clone()
    r = b - A(x)
    rhat, p, q = r.clone(), r.clone(), r.clone()
    rho = alpha = omega = 1.0
    k = 0
    while _dot(r, r) > atol2 and k < maxiter and k >= 0:
        rho_new = _dot(rhat, r)
        beta = rho_new / rho * alpha / omega
        p = r + beta * (p - omega * q)
        phat = M(p)
        q = A(phat)
        alpha_new = rho_new / _dot(rhat, q)
        s = r - alpha_new * q
        exit_early = _dot(s, s) < atol2
        shat = M(s)
        t = A(shat)
        tt = _dot(t, t)
        omega_new = _dot(t, s) / tt if tt != 0 else float("nan")
        if exit_early:
            x = x + alpha_new * phat
            r = s
        else:
            x = x + (alpha_new * phat + omega_new * shat)
            r = s - omega_new * t
        k = -11 if (omega_new == 0 or alpha_new == 0) else k + 1
        if rho_new == 0:
            k = -10
        rho, alpha, omega = rho_new, alpha_new, omega_new
    return x, k


def _normalize(v, thresh):
    nrm = float(torch.linalg.norm(v))
    if nrm > thresh:
        return v / nrm, nrm
    return torch.zeros_like(v), 0.0


def gmres(A, b, x0, M, tol=1e-10, atol=0.0, restart=30, maxiter=100):
    n = b.numel()
    m = min(restart, n)
    eps = torch.finfo(torch.float64).eps
    b_norm = float(torch.linalg.norm(b))
    atol_eff = max(tol * b_norm, atol)
    Mb_norm = float(torch.linalg.norm(M(b)))
    ptol = Mb_norm * min(1.0, atol_eff / b_norm) if b_norm > 0 else float("nan")
    x = x0.clone()
    unit, rnorm = _normalize(M(b - A(x)), eps)
    k = 0
    while k < maxiter and rnorm > ptol:
        V = torch.zeros((m + 1, n), dtype=b.dtype, device=b.device)
        H = torch.zeros((m + 1, m), dtype=b.dtype, device=b.device)
        V[0] = unit
        steps = 0
        for j in range(m):
            w = M(A(V[j]))
            w_norm0 = float(torch.linalg.norm(w))
            h = torch.zeros(m + 1, dtype=b.dtype, device=b.device)
            for _ in range(2):
                c = V[: j + 1] @ w
                w = w - c @ V[: j + 1]
                h[: j + 1] += c
            unit_w, w_norm = _normalize(w, eps * w_norm0)
            h[j + 1] = w_norm
            H[:, j] = h
            V[j + 1] = unit_w
            steps = j + 1
            if w_norm == 0.0:
                break
        beta_vec = torch.zeros(steps + 1, dtype=b.dtype, device=b.device)
        beta_vec[0] = rnorm
        y = torch.linalg.lstsq(H[: steps + 1, :steps].cpu(), beta_vec.cpu().unsqueeze(1)).solution.squeeze(1)
        x = x + y.to(b.device) @ V[:steps]
        unit, rnorm = _normalize(M(b - A(x)), eps)
        k += 1
    return x, k


def solve(dm, vals, b, x0, solver, precond, tol=1e-10, atol=0.0, maxiter=100, restart=30, omega=1.0, block_size=2):
    """(x, iterations) of A x = b with the preconditioner ``precond``: the reference's ilu / ssor / block_jacobi,
    the true ILU(0) (``"ilu0"``) or Jacobi (host-driven loop; the device-resident Jacobi solvers are
    ``device.krylov_solve``)."""
    if precond == "jacobi":
        from .device import jacobi_dinv
        dinv = jacobi_dinv(dm, vals)
        M = lambda v: dinv * v  # noqa: E731
    else:
        M = ReferencePreconditioner(dm, vals, precond, omega=omega, block_size=block_size)
    A = lambda v: spmv(dm, vals, v)  # noqa: E731
    if solver == "cg":
        return cg(A, b, x0, M, tol, atol, maxiter)
    if solver == "bicgstab":
        return bicgstab(A, b, x0, M, tol, atol, maxiter)
    if solver == "gmres":
        return gmres(A, b, x0, M, tol, atol, restart, maxiter)
    raise ValueError(f"Unsupported solver type: {solver}")
