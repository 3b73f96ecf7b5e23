"""Coupled water + solute / nitrogen transport (oracle restatement, parity-unpinned).

The reference has no numeric goldens for these paths (only figures), so this
part of the oracle is a literal restatement without pinning.  Sources:
  * nodal Darcy flux + dispersion tensor: src/models/transport_utilities.py:118-192
  * solute ADR element matrices / assembly: src/numerics/assembly_solute.py:10-186
  * nitrogen species assembly: src/numerics/assembly_nitrogen.py:33-606
  * boundary edges: src/models/boundary.py:108-173 (Neumann, free drainage water),
    :217-277 (Cauchy, sparse), :336-421 (free drainage nitrogen, sparse)
  * drivers: src/solvers/coupled_solver_v2.py:80-331, src/solvers/nitrogen_solver.py:36-412
"""
import numpy as np
import scipy.sparse as sp

from .assembly import assemble_richards, scatter_global
from .krylov import solve_system
from .quadrature import EDGE_POINTS, EDGE_WEIGHTS, TRI3_POINTS, TRI3_WEIGHTS, TRI_DREF
from .soil import van_genuchten_model


# ------------------------------------------------------------------ a13: flux + dispersion
def fluxes_and_dispersion(points, triangles, h, phi, DL, DT, Dm):
    """(qx, qz, |q|, Dxx, Dxz, Dzz, theta) per node (transport_utilities.py:118-192).

    Node gradient = unweighted mean of the constant P1 gradients of the
    triangles containing the node (summed in element order).
    """
    t = np.asarray(triangles)
    P = np.asarray(points)
    x0, y0 = P[t[:, 0], 0], P[t[:, 0], 1]
    x1, y1 = P[t[:, 1], 0], P[t[:, 1], 1]
    x2, y2 = P[t[:, 2], 0], P[t[:, 2], 1]
    b1, b2, b3 = y1 - y2, y2 - y0, y0 - y1
    c1, c2, c3 = x2 - x1, x0 - x2, x1 - x0
    aire = np.abs(c3 * b2 - c2 * b3) / 2
    hl = h[t]
    dhdx = (b1 * hl[:, 0] + b2 * hl[:, 1] + b3 * hl[:, 2]) / (2 * aire)
    dhdz = (c1 * hl[:, 0] + c2 * hl[:, 1] + c3 * hl[:, 2]) / (2 * aire)
    n = P.shape[0]
    sx, sz, cnt = np.zeros(n), np.zeros(n), np.zeros(n)
    # every element adds its gradient to each of its nodes, element by element (np.add.at is ordered)
    rows = t.ravel()
    np.add.at(sx, rows, np.repeat(dhdx, 3))
    np.add.at(sz, rows, np.repeat(dhdz, 3))
    np.add.at(cnt, rows, 1.0)
    gx, gz = sx / cnt, sz / cnt
    _, K, theta = van_genuchten_model(h, phi)
    qx = -K * gx
    qz = -K * (gz + 1)
    aq = np.sqrt(qx ** 2 + qz ** 2)
    theta_s = float(phi[1])
    tau = (theta ** (7 / 3)) / theta_s ** 2
    with np.errstate(all="ignore"):
        Dxx = (DL * qx ** 2 + DT * qz ** 2) / aq + theta * Dm * tau
        Dzz = (DL * qz ** 2 + DT * qx ** 2) / aq + theta * Dm * tau
        Dxz = (DL - DT) * qx * qz / aq
    return qx, qz, aq, Dxx, Dxz, Dzz, theta


# ------------------------------------------------------------------ a14/a15: ADR element matrices
def adr_element_matrices(coords, theta, qx, qz, Dxx, Dxz, Dzz, mu=0.0, sorption=0.0, mu_up=0.0, c_up=None):
    """(K_e, M_e, F_e) per element (assembly_solute.py:39-85, assembly_nitrogen.py:67-133,166-218).

    K = -dispersion - advection + mu*theta*N N^T; M = -(theta + sorption) N N^T;
    F = -mu_up * theta * c_up * N.  All nodal fields are (E, 3).
    """
    E = coords.shape[0]
    J = np.einsum("ij,ejk->eik", TRI_DREF, coords)
    detJ = np.linalg.det(J)
    G = np.linalg.inv(J) @ TRI_DREF
    G0, G1 = G[:, 0, :], G[:, 1, :]
    K = np.zeros((E, 3, 3))
    M = np.zeros((E, 3, 3))
    F = np.zeros((E, 3))
    for q in range(3):
        ks, et = TRI3_POINTS[q]
        w = TRI3_WEIGHTS[q]
        N = np.array([1 - ks - et, ks, et])
        dxx, dxz, dzz = Dxx @ N, Dxz @ N, Dzz @ N
        vx, vz, th = qx @ N, qz @ N, theta @ N
        o = lambda a, b: np.einsum("ei,ej->eij", a, b)  # noqa: E731
        disp = w * (-(dxx[:, None, None] * o(G0, G0)) - dxz[:, None, None] * o(G0, G1)
                    - dxz[:, None, None] * o(G1, G0) - dzz[:, None, None] * o(G1, G1)) * detJ[:, None, None]
        NN = np.outer(N, N)[None]
        adv = w * (-(vx[:, None, None] * np.einsum("i,ej->eij", N, G0))
                   - vz[:, None, None] * np.einsum("i,ej->eij", N, G1)) * detJ[:, None, None]
        react = w * (mu * th)[:, None, None] * NN * detJ[:, None, None]
        K += disp + adv + (react if mu != 0.0 else 0.0)
        M += w * (-th - sorption)[:, None, None] * NN * detJ[:, None, None]
        if c_up is not None:
            cq = c_up @ N
            F += -w * mu_up * th[:, None] * cq[:, None] * N[None] * detJ[:, None]
    return K, M, F


def assemble_adr(triangles, n, points, theta, qx, qz, Dxx, Dxz, Dzz, mu=0.0, sorption=0.0, mu_up=0.0, c_up=None):
    t = np.asarray(triangles)
    coords = points[t]
    K_e, M_e, F_e = adr_element_matrices(coords, theta[t], qx[t], qz[t], Dxx[t], Dxz[t], Dzz[t], mu, sorption,
                                         mu_up, None if c_up is None else c_up[t])
    K, F = scatter_global(t, n, K_e, F_e)
    M, _ = scatter_global(t, n, M_e, np.zeros_like(F_e))
    return K, M, F


def lump(M):
    """Row-sum lumping (nitrogen_solver.py:36-66)."""
    return sp.diags(np.asarray(M.sum(axis=1)).ravel()).tocsr()


# ------------------------------------------------------------------ a7: boundary edges
def edges(nodes):
    """Consecutive boundary-node pairs in the given order (boundary.py loops i -> (n[i], n[i+1]))."""
    nodes = np.asarray(nodes)
    return list(zip(nodes[:-1], nodes[1:]))


def neumann_rhs(b, flux, nodes, points):
    """boundary.py:108-128: b[I,J] -= Jac * w * flux * N (2-point Gauss)."""
    b = b.copy()
    Nm = np.stack([(1 - EDGE_POINTS) / 2, (1 + EDGE_POINTS) / 2])
    for I, J in edges(nodes):
        jac = (points[J, 0] - points[I, 0]) / 2
        loc = np.zeros(2)
        for j in range(2):
            loc = loc - jac * EDGE_WEIGHTS[j] * flux * Nm[:, j]
        b[I] += loc[0]
        b[J] += loc[1]
    return b


def freedrainage_water_rhs(b, K, nodes, points):
    """boundary.py:132-173: b[I,J] += -Jac * w * (N.K) * N."""
    b = b.copy()
    Nm = np.stack([(1 - EDGE_POINTS) / 2, (1 + EDGE_POINTS) / 2])
    for I, J in edges(nodes):
        jac = (points[J, 0] - points[I, 0]) / 2
        loc = np.zeros(2)
        for j in range(2):
            kav = Nm[:, j] @ K[[I, J]]
            loc = loc + (-jac * EDGE_WEIGHTS[j] * kav * Nm[:, j])
        b[I] += loc[0]
        b[J] += loc[1]
    return b


def cauchy(A, b, flux, c_in, nodes, points):
    """boundary.py:217-277 (sparse): A[IJ block] += Jac w flux N N^T ; b += Jac c_in flux sum_w N."""
    n = A.shape[0]
    Nm = np.stack([(1 - EDGE_POINTS) / 2, (1 + EDGE_POINTS) / 2])
    rows, cols, vals = [], [], []
    b = b.copy()
    sI, sJ, II, JJ = [], [], [], []
    for I, J in edges(nodes):
        jac = (points[J, 0] - points[I, 0]) / 2
        loc = np.zeros(4)
        for j in range(2):
            wgt = jac * EDGE_WEIGHTS[j] * flux
            Nv = Nm[:, j]
            loc += wgt * np.array([Nv[0] * Nv[0], Nv[0] * Nv[1], Nv[1] * Nv[0], Nv[1] * Nv[1]])
        rows += [I, I, J, J]
        cols += [I, J, I, J]
        vals += list(loc)
        sI.append(jac * c_in * flux * (EDGE_WEIGHTS[0] * Nm[0, 0] + EDGE_WEIGHTS[1] * Nm[0, 1]))
        sJ.append(jac * c_in * flux * (EDGE_WEIGHTS[0] * Nm[1, 0] + EDGE_WEIGHTS[1] * Nm[1, 1]))
        II.append(I)
        JJ.append(J)
    B = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    np.add.at(b, II, sI)
    np.add.at(b, JJ, sJ)
    return (A + B).tocsr(), b


def freedrainage_nitrogen(A, b, K, theta, nodes, points):
    """boundary.py:336-421 (sparse): A[IJ block] += Jac w (-(N.K)/(N.theta)) N N^T."""
    n = A.shape[0]
    Nm = np.stack([(1 - EDGE_POINTS) / 2, (1 + EDGE_POINTS) / 2])
    rows, cols, vals = [], [], []
    for I, J in edges(nodes):
        jac = (points[J, 0] - points[I, 0]) / 2.0
        loc = np.zeros(4)
        for j in range(2):
            Nv = Nm[:, j]
            vel = -(Nv @ K[[I, J]]) / (Nv @ theta[[I, J]])
            wgt = jac * EDGE_WEIGHTS[j] * vel
            loc += wgt * np.array([Nv[0] * Nv[0], Nv[0] * Nv[1], Nv[1] * Nv[0], Nv[1] * Nv[1]])
        rows += [I, I, J, J]
        cols += [I, J, I, J]
        vals += list(loc)
    B = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    return (A + B).tocsr(), b


# ------------------------------------------------------------------ a12/a16: drivers
def richards_neumann_step(points, tri, h_n, theta_n, dt, phi, neumann_nodes, flux, fd_nodes=None,
                          solver="gmres", precond="none", tol=1e-10, maxiter=100, restart=30,
                          picard_tol=1e-4, picard_max=100):
    """coupled_solver_v2.py:80-140 / nitrogen_solver.py:100-149 (absolute Picard error)."""
    n = points.shape[0]
    h_m = h_n.copy()
    err, it = np.inf, 0
    while err >= picard_tol and it < picard_max:
        C, K, th = van_genuchten_model(h_m, phi)
        A, b = assemble_richards(tri, n, points, th, theta_n, h_m, K, C, dt)
        b = neumann_rhs(b, flux, neumann_nodes, points)
        if fd_nodes is not None and len(fd_nodes) > 0:
            b = freedrainage_water_rhs(b, K, fd_nodes, points)
        h_new, _ = solve_system(A, b, h_m, solver, precond, tol=tol, maxiter=maxiter, restart=restart)
        err = np.linalg.norm(h_new - h_m)
        h_m = h_new
        it += 1
    return h_m, err, it


def solute_step(points, tri, c_n, theta, theta_n, qx, qz, Dxx, Dxz, Dzz, dt, cauchy_nodes, cauchy_flux, c_in,
                solver="gmres", precond="none", tol=1e-10, maxiter=100, restart=30):
    """coupled_solver_v2.py:147-197: b = M c_n / dt (+Cauchy), A = M/dt + K."""
    n = points.shape[0]
    K, M, _ = assemble_adr(tri, n, points, theta, qx, qz, Dxx, Dxz, Dzz)
    b = (1 / dt) * (M @ c_n)
    K, b = cauchy(K, b, cauchy_flux, c_in, cauchy_nodes, points)
    A = ((1 / dt) * M + K).tocsr()
    c, _ = solve_system(A, b, c_n, solver, precond, tol=tol, maxiter=maxiter, restart=restart)
    return c


def nitrogen_species_step(points, tri, c_n, theta, qx, qz, Dxx, Dxz, Dzz, K_node, dt, mu, sorption, mu_up, c_up,
                          cauchy_nodes, cauchy_flux, c_in, fd_nodes, solver="gmres", precond="none", tol=1e-10,
                          maxiter=100, restart=30):
    """One species of nitrogen_solver.py:151-235: lumped mass, Cauchy inflow, free-drainage outflow."""
    n = points.shape[0]
    K, M, F = assemble_adr(tri, n, points, theta, qx, qz, Dxx, Dxz, Dzz, mu=mu, sorption=sorption, mu_up=mu_up,
                           c_up=c_up)
    Ml = lump(M)
    b = (1.0 / dt) * (Ml @ c_n) + F
    if len(cauchy_nodes):
        K, b = cauchy(K, b, cauchy_flux, c_in, cauchy_nodes, points)
    if len(fd_nodes):
        K, b = freedrainage_nitrogen(K, b, K_node, theta, fd_nodes, points)
    A = ((1.0 / dt) * Ml + K).tocsr()
    c, _ = solve_system(A, b, c_n, solver, precond, tol=tol, maxiter=maxiter, restart=restart)
    return c


# ------------------------------------------------------------------ mass balance, Peclet / Courant
def integrate_2d_domain(f, points, triangles):
    """richards_mass_balance-checkpoint.py:25-69: sum_e |det J| sum_q (1/3) f(x_q) (twice the integral)."""
    t = np.asarray(triangles)
    P = np.asarray(points)
    J00 = P[t[:, 1], 0] - P[t[:, 0], 0]
    J01 = P[t[:, 2], 0] - P[t[:, 0], 0]
    J10 = P[t[:, 1], 1] - P[t[:, 0], 1]
    J11 = P[t[:, 2], 1] - P[t[:, 0], 1]
    det = np.abs(J00 * J11 - J01 * J10)
    fl = np.asarray(f)[t]
    total = np.zeros(len(t))
    for a, b in ((1 / 6, 1 / 6), (2 / 3, 1 / 6), (1 / 6, 2 / 3)):
        total += (1 / 3) * (fl[:, 0] * (1 - a - b) + fl[:, 1] * a + fl[:, 2] * b)
    return float(np.sum(total * det))


def element_size(points, triangles):
    """transport_utilities.py:196-203: shortest edge per triangle."""
    v = np.asarray(points)[np.asarray(triangles)]
    e = v - np.roll(v, 1, axis=1)
    return np.min(np.sqrt(np.sum(e ** 2, axis=2)), axis=1)


def peclet_courant(points, triangles, qx, qz, theta, Dxx, Dzz, dt):
    """transport_utilities.py:205-242: max over elements and nodes of |v| h / (2D) and |v| dt / h."""
    t = np.asarray(triangles)
    h = element_size(points, triangles)[:, None]
    vx, vz = np.abs(qx[t] / theta[t]), np.abs(qz[t] / theta[t])
    pe = np.maximum(vx * h / (2 * Dxx[t]), vz * h / (2 * Dzz[t])).max()
    cr = np.maximum(vx * dt / h, vz * dt / h).max()
    return float(pe), float(cr)


def coupled_time_loop(points, tri, phi, neumann_nodes, cauchy_nodes, dt0, tmax, DL=0.5, DT=0.1, Dm=0.0,
                      c_init=0.1, c_inlet=1.0, neumann_flux=-0.1, cauchy_flux=-0.1, h0=-1.3, solver="gmres",
                      precond="none", tol=1e-10, maxiter=100, restart=30, m_it=5, M_it=7, lambda_amp=2.0,
                      lambda_red=0.5, max_steps=None):
    """CoupledSolver.solve, src/solvers/coupled_solver_v2.py:223-300, on the oracle's step functions.

    Per step: theta_n at the previous head; the Richards step with the Neumann inflow and the absolute
    Picard error (< 1e-4, at most 100 iterations, :80-140); fluxes and dispersion at the new head; the
    solute step (:147-197); dt_new from the iteration count with the floor max(dt_new, 1e-6) (:200-221;
    the reference's upper clamp to 0.5 is overwritten by that line and has no effect); the clock advances
    by the step's own dt, then dt = dt_new (:291-292).  Returns per-step lists: time after the step,
    Picard error, iterations, dt_new, and the heads and concentrations."""
    n = points.shape[0]
    h_n = float(h0) * np.ones(n)
    c_n = float(c_init) * np.ones(n)
    kw = dict(solver=solver, precond=precond, tol=tol, maxiter=maxiter, restart=restart)
    out = {k: [] for k in ("time", "error", "iterations", "dt", "pressure_head", "solute")}
    t, dt, steps = 0.0, float(dt0), 0
    while t < tmax and (max_steps is None or steps < max_steps):
        _, _, th_n = van_genuchten_model(h_n, phi)
        h, err, it = richards_neumann_step(points, tri, h_n, th_n, dt, phi, neumann_nodes, neumann_flux,
                                           picard_tol=1e-4, picard_max=100, **kw)
        qx, qz, aq, Dxx, Dxz, Dzz, th = fluxes_and_dispersion(points, tri, h, phi, DL, DT, Dm)
        c = solute_step(points, tri, c_n, th, th_n, qx, qz, Dxx, Dxz, Dzz, dt, cauchy_nodes, cauchy_flux, c_inlet,
                        **kw)
        dt_r = lambda_amp * dt if it <= m_it else (dt if it <= M_it else lambda_red * dt)
        dt_new = max(dt_r, 1e-6)
        h_n, c_n = h, c
        t += dt
        dt = dt_new
        steps += 1
        for k, v in (("time", t), ("error", float(err)), ("iterations", it), ("dt", dt_new),
                     ("pressure_head", h), ("solute", c)):
            out[k].append(v)
    return out
