"""Krylov solvers and preconditioners (oracle restatement).

The reference calls ``jax.scipy.sparse.linalg.{cg, bicgstab, gmres}``
(src/solvers/jax_linear_solver.py:255-329) with ``tol=1e-10, atol=0,
maxiter=100, restart=30`` (config/settings.py:104-106) and x0 = the current
Picard iterate.  jax/jaxlib are third-party and unpinned
(requirements.txt:1-2) and absent here, so these are restatements of the
published algorithms with JAX's documented stopping semantics:

* CG: preconditioned Hestenes-Stiefel; stop when ``r.r <= max(tol^2 b.b, atol^2)``
  (recursive residual) or after ``maxiter`` iterations.
* BiCGSTAB: van der Vorst (1992), right preconditioned, shadow residual
  r_hat = r0, rho0 = alpha0 = omega0 = 1, early exit on ``s.s < atol2``,
  breakdown exit when rho, alpha or omega is exactly zero.
* GMRES(m): Saad-Schultz, left preconditioned; ``maxiter`` counts restart
  cycles; each cycle runs all m Arnoldi steps (classical Gram-Schmidt with one
  re-orthogonalisation pass) unless the new basis vector vanishes, solves the
  (m+1) x m least-squares problem, and tests the preconditioned residual
  ``||M(b - A x)||`` against ``||M b|| * min(1, max(tol*||b||, atol)/||b||)``.

Jacobi: ``Preconditioner.create_jacobi`` (jax_linear_solver.py:11-36):
``M x = x / d`` with d = diag(A), zeros replaced by 1.

The reference's other preconditioners, restated from what their code computes
(``reference_preconditioner``; d = diag(A), L / U = strict lower / upper parts):
* ``ilu`` (create_ilu0, jax_linear_solver.py:171-252): L scaled by 1/d of its
  column, U unscaled, no pivot update -- M = (D + L) D^-1 (D' + U) with
  D' = D with zeros replaced by 1, i.e. symmetric Gauss-Seidel, not a true ILU(0);
* ``ssor`` (create_ssor, :91-169): forward sweep y = (D/omega + L)^-1 x; the
  backward sweep reads entries of z that are not computed yet (zeros), so it
  returns z = omega y;
* ``block_jacobi`` (create_block_jacobi, :38-89): inverses of the diagonal
  blocks of size block_size (last block smaller), each + 1e-12 I before inversion.
The solvers take either a Jacobi diagonal (``dinv`` array) or any such
callable; with any preconditioner CG tests r.r (JAX's rule for M != identity).
"""
import numpy as np


def jacobi_inverse_diagonal(A):
    d = A.diagonal().astype(np.float64)
    return 1.0 / np.where(d != 0, d, 1.0)


def _precond(dinv):
    if callable(dinv):
        return dinv
    if dinv is None:
        return lambda v: v
    return lambda v: dinv * v


def cg(A, b, x0, tol=1e-10, atol=0.0, maxiter=100, dinv=None):
    """Returns (x, iterations)."""
    M = _precond(dinv)
    matvec = A.__matmul__ if not callable(A) else A
    bs = float(b @ b)
    atol2 = max(tol * tol * bs, atol * atol)
    x = np.array(x0, dtype=np.float64, copy=True)
    r = b - matvec(x)
    z = M(r)
    p = z.copy()
    gamma = float(r @ z)
    k = 0
    while True:
        rs = gamma if dinv is None else float(r @ r)
        if not (rs > atol2 and k < maxiter):
            break
        Ap = matvec(p)
        alpha = gamma / float(p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = M(r)
        gamma_new = float(r @ z)
        beta = gamma_new / gamma
        gamma = gamma_new
        p = z + beta * p
        k += 1
    return x, k



def pipelined_cg(A, b, x0, tol=1e-10, atol=0.0, maxiter=100, dinv=None, dtype=np.float64):
    """Pipelined Jacobi-CG as the device's inner solver computes it (not a reference function: the mixed
    path's FP32 inner solve).  Ghysels & Vanroose, Parallel Computing 40 (2014) 224-238, Alg. 4, with the
    recurrences of u = M r, q = M s, m = M w collapsed into products with the diagonal d (M = diag(d)):
    gamma = (r, u), delta = (w, u), rho = (r, r) are read after n = A M w; the stopping rule tests rho
    (gamma without a preconditioner) before the update.  Equals CG in exact arithmetic; the recurrence for
    w = A M r drifts by rounding.  Returns (x, iterations)."""
    d = np.ones(len(b)) if dinv is None else np.asarray(dinv)
    A = A.astype(dtype)
    d = d.astype(dtype)
    b = np.asarray(b).astype(dtype)
    x = np.array(x0, dtype=dtype, copy=True)
    r = b - A @ x
    u = d * r
    w = A @ u
    z, s, p = (np.zeros_like(r) for _ in range(3))
    bs = float(b @ b)
    atol2 = max(tol * tol * bs, atol * atol)
    gamma_old = alpha = 0.0
    k = 0
    while True:
        gamma, delta, rho = float(r @ u), float(w @ u), float(r @ r)
        n_ = A @ (d * w)
        rs = gamma if dinv is None else rho
        if not (rs > atol2) or k >= maxiter:
            break
        if k == 0:
            beta, alpha = 0.0, gamma / delta
        else:
            beta = gamma / gamma_old
            alpha = gamma / (delta - beta * gamma / alpha)
        z = n_ + dtype(beta) * z
        s = w + dtype(beta) * s
        p = u + dtype(beta) * p
        x = x + dtype(alpha) * p
        r = r - dtype(alpha) * s
        w = w - dtype(alpha) * z
        u = d * r
        gamma_old = gamma
        k += 1
    return x, k

def bicgstab(A, b, x0, tol=1e-10, atol=0.0, maxiter=100, dinv=None):
    """Returns (x, iterations); iterations < 0 flags a breakdown exit."""
    M = _precond(dinv)
    matvec = A.__matmul__ if not callable(A) else A
    bs = float(b @ b)
    atol2 = max(tol * tol * bs, atol * atol)
    x = np.array(x0, dtype=np.float64, copy=True)
    r = b - matvec(x)
    rhat = r.copy()
    rho = alpha = omega = 1.0
    p = r.copy()
    q = r.copy()
    k = 0
    while float(r @ r) > atol2 and k < maxiter and k >= 0:
        rho_new = float(rhat @ r)
        beta = rho_new / rho * alpha / omega
        p = r + beta * (p - omega * q)
        phat = M(p)
        q = matvec(phat)
        alpha_new = rho_new / float(rhat @ q)
        s = r - alpha_new * q
        exit_early = float(s @ s) < atol2
        shat = M(s)
        t = matvec(shat)
        with np.errstate(all="ignore"):
            omega_new = float(t @ s) / float(t @ t)
        if exit_early:
            x = x + alpha_new * phat
            r = s
        else:
            x = x + (alpha_new * phat + omega_new * shat)
            r = s - omega_new * t
        if omega_new == 0 or alpha_new == 0:
            k = -11
        else:
            k = k + 1
        if rho_new == 0:
            k = -10
        rho, alpha, omega = rho_new, alpha_new, omega_new
    return x, k


def _safe_normalize(v, thresh=None):
    n = float(np.sqrt(v @ v))
    if thresh is None:
        thresh = np.finfo(np.float64).eps
    if n > thresh:
        return v / n, n
    return np.zeros_like(v), 0.0


def gmres(A, b, x0, tol=1e-10, atol=0.0, restart=30, maxiter=100, dinv=None):
    """Returns (x, restart_cycles)."""
    M = _precond(dinv)
    matvec = A.__matmul__ if not callable(A) else A
    n = b.shape[0]
    m = min(restart, n)
    b_norm = float(np.sqrt(b @ b))
    atol_eff = max(tol * b_norm, atol)
    Mb_norm = float(np.sqrt(M(b) @ M(b)))
    # jnp.minimum propagates NaN: b == 0 gives a NaN tolerance and no iterations
    ptol = Mb_norm * min(1.0, atol_eff / b_norm) if b_norm > 0 else float('nan')
    x = np.array(x0, dtype=np.float64, copy=True)
    unit, rnorm = _safe_normalize(M(b - matvec(x)))
    eps = np.finfo(np.float64).eps
    k = 0
    while k < maxiter and rnorm > ptol:
        V = np.zeros((m + 1, n))
        H = np.zeros((m + 1, m))
        V[0] = unit
        steps = 0
        for j in range(m):
            w = M(matvec(V[j]))
            w_norm0 = float(np.sqrt(w @ w))
            h = np.zeros(m + 1)
            for _ in range(2):                       # CGS2: project twice
                c = V[: j + 1] @ w
                w = w - c @ V[: j + 1]
                h[: j + 1] += c
            unit_w, w_norm = _safe_normalize(w, thresh=eps * w_norm0)
            h[j + 1] = w_norm
            H[:, j] = h
            V[j + 1] = unit_w
            steps = j + 1
            if w_norm == 0.0:
                break
        beta_vec = np.zeros(m + 1)
        beta_vec[0] = rnorm
        y = np.linalg.lstsq(H[: steps + 1, :steps], beta_vec[: steps + 1], rcond=None)[0]
        x = x + y @ V[:steps]
        unit, rnorm = _safe_normalize(M(b - matvec(x)))
        k += 1
    return x, k


def reference_preconditioner(A, precond_type, omega=1.0, block_size=2):
    """Callable M(v) of the reference's preconditioner of A (see the module docstring)."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import spsolve_triangular
    A = sp.csr_matrix(A)
    n = A.shape[0]
    d = A.diagonal().astype(np.float64)
    if precond_type == "jacobi":
        dinv = jacobi_inverse_diagonal(A)
        return lambda v: dinv * v
    if precond_type == "ilu":
        dz = np.where(d == 0, 1.0, d)
        L = sp.tril(A, -1).tocsr() @ sp.diags(1.0 / dz)
        Lw = (L + sp.identity(n)).tocsr()
        Uw = (sp.triu(A, 1) + sp.diags(dz)).tocsr()
        return lambda v: spsolve_triangular(Uw, spsolve_triangular(Lw, v, lower=True, unit_diagonal=True),
                                            lower=False)
    if precond_type == "ssor":
        Lw = (sp.tril(A, -1) + sp.diags(d / omega)).tocsr()
        return lambda v: omega * spsolve_triangular(Lw, v, lower=True)
    if precond_type == "block_jacobi":
        Ad = A.toarray() if n <= 4096 else None
        invs = []
        for s0 in range(0, n, block_size):
            s1 = min(s0 + block_size, n)
            blk = (Ad[s0:s1, s0:s1] if Ad is not None else A[s0:s1, s0:s1].toarray()) + 1e-12 * np.eye(s1 - s0)
            invs.append((s0, s1, np.linalg.inv(blk)))

        def apply(v):
            out = np.empty_like(v)
            for s0, s1, inv in invs:
                out[s0:s1] = inv @ v[s0:s1]
            return out
        return apply
    raise ValueError(f"unknown preconditioner {precond_type!r}")


def solve_system(A, b, x0, solver_type="gmres", precond_type="none", tol=1e-10,
                 maxiter=100, restart=30, omega=1.0, block_size=2):
    """Dispatch of src/solvers/solver_types.py:7-67 with the reference's preconditioners.

    Returns (x, iterations).  ``direct`` solves exactly (the reference densifies
    and calls jnp.linalg.solve; a sparse LU gives the same solution).
    """
    if precond_type in ("none", None):
        M = None
    elif precond_type == "jacobi":
        M = jacobi_inverse_diagonal(A)
    else:
        M = reference_preconditioner(A, precond_type, omega=omega, block_size=block_size)
    if solver_type == "cg":
        return cg(A, b, x0, tol=tol, maxiter=maxiter, dinv=M)
    if solver_type == "bicgstab":
        return bicgstab(A, b, x0, tol=tol, maxiter=maxiter, dinv=M)
    if solver_type == "gmres":
        return gmres(A, b, x0, tol=tol, restart=restart, maxiter=maxiter, dinv=M)
    if solver_type == "direct":
        import scipy.sparse.linalg as spla
        return spla.spsolve(A.tocsc(), b), 0
    raise ValueError(f"Unsupported solver type: {solver_type}")


def true_ilu0(A):
    """Incomplete LU with zero fill on A's own pattern (Saad, Iterative Methods for Sparse Linear Systems,
    Alg. 10.4, IKJ form) -- not a reference function (the reference's `ilu` is `reference_preconditioner`'s
    symmetric Gauss-Seidel form); the factorization the device's wspm_ilu0_factor computes.  Returns a CSR matrix
    holding L (strict lower part, unit diagonal implied) and U; zero pivots are taken as 1."""
    import scipy.sparse as sp
    LU = sp.csr_matrix(A, dtype=np.float64, copy=True)
    LU.sort_indices()
    ip, ix, d = LU.indptr, LU.indices, LU.data
    n = LU.shape[0]
    diag = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        for q in range(ip[i], ip[i + 1]):
            if ix[q] == i:
                diag[i] = q
    for i in range(n):
        pos = {int(ix[q]): q for q in range(ip[i], ip[i + 1])}
        for q in range(ip[i], ip[i + 1]):
            k = int(ix[q])
            if k >= i:
                break
            if d[q] == 0.0:
                continue
            ukk = d[diag[k]] if diag[k] >= 0 else 0.0
            lik = d[q] / (ukk if ukk != 0.0 else 1.0)
            d[q] = lik
            for q2 in range(ip[k], ip[k + 1]):
                j = int(ix[q2])
                if j > k and j in pos and pos[j] > q:
                    d[pos[j]] -= lik * d[q2]
    return LU


def true_ilu0_apply(LU, x):
    """y = (L U)^-1 x with the factors of true_ilu0 (forward sweep with unit L, backward with U)."""
    ip, ix, d = LU.indptr, LU.indices, LU.data
    n = LU.shape[0]
    y = np.array(x, dtype=np.float64, copy=True)
    for i in range(n):
        s = y[i]
        for q in range(ip[i], ip[i + 1]):
            if ix[q] < i:
                s -= d[q] * y[ix[q]]
        y[i] = s
    z = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s, di = y[i], 0.0
        for q in range(ip[i], ip[i + 1]):
            if ix[q] > i:
                s -= d[q] * z[ix[q]]
            elif ix[q] == i:
                di = d[q]
        z[i] = s / (di if di != 0.0 else 1.0)
    return z
