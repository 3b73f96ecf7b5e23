"""Picard time steppers for Richards' equation (oracle restatement).

* 2D tests Test1/2/3 (Gardner soil, Dirichlet top/bottom):
  src/solvers/richards_solver_v2.py:75-168 (set-up, Picard body) and
  :272-352 (time loop, dt adaptation :91-105).
* 3D Test3D: src/solvers/richards_solver_3D_v2.py:72-302 (absolute Picard
  error, <= 30 iterations, start-of-step theta recorded).
* VG Dirichlet case (van Genuchten soil with the same Picard/Dirichlet
  mechanism) used for the unit-square workloads.

Quirks reproduced: the bottom Dirichlet value is ``-15`` (``jnp.full_like`` on
an int64 index array truncates -15.24, richards_solver_v2.py:141 and
boundary.py:678); top is applied before bottom; the recorded time is the
start time of the step and the clock advances by the *new* dt
(richards_solver_v2.py:316,323).

Two Picard profiles exist in the reference tree and both are supported:
  * the current source (richards_solver_v2.py:155-162): relative error
    ``||h-h_m||/||h|| < 1e-6``, at most 100 iterations, end-of-step theta;
  * the driver that produced the published resultsRE2D CSVs
    (src/solvers/.ipynb_checkpoints/richards_solver-checkpoint.py:157-164,214):
    absolute error ``< 1e-4``, at most 30 iterations, start-of-step theta
    recorded, run with dt0 = 1e-3 (the CSV runs' first dt_new is 2e-3 in
    logs/40064505.err).  With this profile the oracle reproduces the CSV
    iteration totals and all six error metrics to 5 significant digits.
"""
import numpy as np

from .soil import exponential_model, van_genuchten_model
from .assembly import assemble_richards, apply_dirichlet_rows
from .krylov import solve_system

L_DOMAIN = 15.24
EXP_PHI = (0.164, 0.45, 0.15, 0.1)          # [alpha0, thetas, thetar, Ks] (config/settings.py:40-48)


def upper_bc(test_case, x, alpha0, eps0, y=None, L=L_DOMAIN):
    """Top boundary functions (boundary.py:17-33, 3D :423-442)."""
    if test_case == "Test1":
        return (1 / alpha0) * np.log(eps0 + (1 - eps0) * ((3 / 4) * np.sin(np.pi * x / L) - (1 / 4) * np.sin(3 * np.pi * x / L)))
    if test_case == "Test2":
        return (1 / alpha0) * np.log(eps0 + (1 - eps0) * np.sin(np.pi * x / L))
    if test_case == "Test3":
        return (1 / alpha0) * np.log(eps0 + 0.5 * (1 - eps0) * (1 - np.cos(2 * np.pi * x / L)))
    if test_case == "Test3D":
        return (1 / alpha0) * np.log(eps0 + (1 - eps0) * np.sin(np.pi * x / L) * np.sin(np.pi * y / L))
    raise ValueError(test_case)


def boundary_nodes_2d(points, test_case):
    """(top, bottom) index sets by exact coordinate compares (boundary.py:482-547)."""
    x, y = points[:, 0], points[:, 1]
    if test_case == "Test3":
        bottom = np.where(y == 0)[0]
    else:
        bottom = np.where((y == 0) | (x == 0) | (x == 15.24))[0]
    top = np.where(y == 15.24)[0]
    return top, bottom


def boundary_nodes_3d(points, L=L_DOMAIN, tol=1e-10):
    """(top, bottom) for the cube (boundary.py:444-480)."""
    x, y, z = points[:, 0], points[:, 1], points[:, 2]
    top = np.where(np.abs(z - L) < tol)[0]
    bottom = np.where((np.abs(z) < tol) | (np.abs(x) < tol) | (np.abs(x - L) < tol)
                      | (np.abs(y) < tol) | (np.abs(y - L) < tol))[0]
    return top, bottom


def dirichlet_arrays(n, sets):
    """Merge Dirichlet sets applied in order (later sets overwrite earlier ones)."""
    nodes = []
    vals = np.zeros(n)
    mask = np.zeros(n, dtype=bool)
    for idx, v in sets:
        mask[idx] = True
        vals[idx] = v
    nodes = np.where(mask)[0]
    return nodes, vals[nodes]


def adapt_dt(dt, it, m_it=5, M_it=7, amp=2.0, red=0.5):
    """richards_solver_v2.py:91-105."""
    if it <= m_it:
        return amp * dt
    if it <= M_it:
        return dt
    return red * dt


class RichardsProblem:
    """One Richards problem: mesh, soil model, Dirichlet data and solver knobs."""

    def __init__(self, points, elements, soil="exp", phi=EXP_PHI, dirichlet=((), ()),
                 solver="cg", precond="jacobi", tol=1e-10, maxiter=100, restart=30,
                 picard_tol=1e-6, picard_max=100, picard_relative=True, Ks_elem=None):
        self.points = np.asarray(points, dtype=np.float64)
        self.elements = np.asarray(elements, dtype=np.int64)
        self.n = self.points.shape[0]
        self.soil = soil
        self.phi = tuple(float(v) for v in phi)
        self.bc_nodes, self.bc_vals = dirichlet
        self.solver, self.precond = solver, precond
        self.tol, self.maxiter, self.restart = tol, maxiter, restart
        self.picard_tol, self.picard_max, self.picard_relative = picard_tol, picard_max, picard_relative
        self.Ks_elem = Ks_elem

    def model(self, h):
        if self.soil == "exp":
            return exponential_model(h, self.phi)
        return van_genuchten_model(h, self.phi)

    def linear_system(self, h_m, theta_n, dt):
        C, K, th_m = self.model(h_m)
        A, b = assemble_richards(self.elements, self.n, self.points, th_m, theta_n, h_m, K, C, dt,
                                 Ks_elem=self.Ks_elem)
        A, b = apply_dirichlet_rows(A, b, self.bc_nodes, self.bc_vals)
        return A, b

    def timestep(self, h_n, theta_n, dt, stats=None):
        """Picard loop: returns (h, err, iterations) (richards_solver_v2.py:107-168)."""
        h_m = h_n.copy()
        err = np.inf
        it = 0
        while err >= self.picard_tol and it < self.picard_max:
            A, b = self.linear_system(h_m, theta_n, dt)
            h_new, kits = solve_system(A, b, h_m, self.solver, self.precond, tol=self.tol,
                                       maxiter=self.maxiter, restart=self.restart)
            if stats is not None:
                stats.append(kits)
            d = np.linalg.norm(h_new - h_m)
            err = d / np.linalg.norm(h_new) if self.picard_relative else d
            h_m = h_new
            it += 1
        return h_m, err, it


def run_time_loop(prob, h0, dt0, tmax, theta_at_end=True, fixed_dt=False, max_steps=None):
    """Host time loop (richards_solver_v2.py:272-352; 3D records start-of-step theta)."""
    out = {"pressure_head": [], "theta": [], "times": [], "iterations": [], "errors": [], "dt_values": []}
    h_n = np.array(h0, dtype=np.float64)
    t = 0.0
    dt = float(dt0)
    steps = 0
    while t < tmax and (max_steps is None or steps < max_steps):
        _, _, theta_n = prob.model(h_n)
        h, err, it = prob.timestep(h_n, theta_n, dt)
        dt_new = dt if fixed_dt else float(adapt_dt(dt, it))
        theta = prob.model(h)[2] if theta_at_end else theta_n
        out["pressure_head"].append(h)
        out["theta"].append(theta)
        out["times"].append(t)
        out["iterations"].append(it)
        out["errors"].append(err)
        out["dt_values"].append(dt_new)
        h_n = h
        t += dt_new
        dt = dt_new
        steps += 1
    return {k: np.array(v) for k, v in out.items()}


def test_case_2d(points, triangles, test_case, solver="cg", precond="jacobi", **kw):
    """Set-up of RichardsSolver for Test1/2/3 (richards_solver_v2.py:50-89)."""
    alpha0 = EXP_PHI[0]
    top, bottom = boundary_nodes_2d(points, test_case)
    h0 = -15.24 * np.ones(points.shape[0])
    hupper = upper_bc(test_case, points[top, 0], alpha0, np.exp(alpha0 * h0[top]))
    nodes, vals = dirichlet_arrays(points.shape[0], [(top, hupper), (bottom, float(int(-15.24)))])
    prob = RichardsProblem(points, triangles, soil="exp", phi=EXP_PHI, dirichlet=(nodes, vals),
                           solver=solver, precond=precond, **kw)
    return prob, h0


def test_case_3d(points, tets, solver="bicgstab", precond="none", **kw):
    """Set-up of RichardsSolver3D (richards_solver_3D_v2.py:49-88); absolute err < 1e-4, <= 30 its."""
    alpha0 = EXP_PHI[0]
    top, bottom = boundary_nodes_3d(points)
    h0 = -15.24 * np.ones(points.shape[0])
    hupper = upper_bc("Test3D", points[top, 0], alpha0, np.exp(alpha0 * h0[top]), y=points[top, 1])
    nodes, vals = dirichlet_arrays(points.shape[0], [(top, hupper), (bottom, float(int(-15.24)))])
    kw.setdefault("picard_tol", 1e-4)
    kw.setdefault("picard_max", 30)
    kw.setdefault("picard_relative", False)
    prob = RichardsProblem(points, tets, soil="exp", phi=EXP_PHI, dirichlet=(nodes, vals),
                           solver=solver, precond=precond, **kw)
    return prob, h0


# van Genuchten unit-domain workload: theta_r .102, theta_s .368, alpha 3.35, n 2, m .5, Ks .0922
VG_UNIT_PHI = (3.35, 0.368, 0.102, 2.0, 0.5, 0.0922)


def vg_dirichlet_case(points, elements, top_nodes, h_top=-0.1, h0=-1.0, phi=VG_UNIT_PHI,
                      solver="cg", precond="jacobi", Ks_elem=None, **kw):
    """VG soil, uniform h0, Dirichlet h_top on the top nodes, natural no-flux elsewhere."""
    n = points.shape[0]
    nodes, vals = dirichlet_arrays(n, [(np.asarray(top_nodes), h_top)])
    if Ks_elem is not None:
        phi = tuple(phi[:5]) + (1.0,)
    prob = RichardsProblem(points, elements, soil="vg", phi=phi, dirichlet=(nodes, vals),
                           solver=solver, precond=precond, Ks_elem=Ks_elem, **kw)
    return prob, h0 * np.ones(n)
