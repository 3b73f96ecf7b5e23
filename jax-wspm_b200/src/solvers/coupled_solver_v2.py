"""Coupled water flow + solute transport (drop-in for src/solvers/coupled_solver_v2.py:42-331).

``CoupledSolver(config).solve()`` returns the reference's result dictionary.
Per time step: theta_n from the soil model at the previous head; the Richards
step on the device (``PicardEngine``: van Genuchten soil, Neumann flux on the
inlet nodes, no Dirichlet rows, absolute Picard error < 1e-4, at most 100
iterations -- coupled_solver_v2.py:81-140); nodal Darcy fluxes and the
dispersion tensor (``wspm_flux_dispersion_2d``); the solute step (consistent
mass, Cauchy inflow, A = M/dt + K -- :148-197); dt adaptation with the
configured thresholds and the reference's 1e-6 floor (:200-221).
"""
import time
from typing import Any, Dict

import numpy as np
import torch

from wspm_b200 import context
from wspm_b200.device import KrylovWorkspace, flux_dispersion, soil
from wspm_b200.engine import PicardEngine, adapt_time_step as _adapt
from wspm_b200.transport import edges_or_none, solute_step

from ..mesh.loader import load_and_validate_mesh
from ..models.boundary import extract_boundary_nodes, get_boundary_condition
from ..numerics.gauss import gauss_triangle

PICARD_TOL, PICARD_MAXITER = 1e-4, 100


class CoupledSolver:
    """Solver for coupled water flow and solute transport equations."""

    def __init__(self, config):
        self.config = config
        self.setup_solver()

    def setup_solver(self):
        cfg = self.config
        self.points, self.triangles, self.mesh_info = load_and_validate_mesh(cfg.mesh.mesh_size, cfg.mesh.mesh_dir,
                                                                             cfg.test_case)
        self.boundary_nodes = extract_boundary_nodes(self.points, cfg.test_case)
        self.quad_points, self.weights = gauss_triangle(3)
        self.bc_info = get_boundary_condition(cfg.test_case)
        self.nnt = len(self.points)
        self.dm = context.mesh_for(self.points, self.triangles)
        self.phi = tuple(float(v) for v in cfg.van_genuchten.to_array())
        s = cfg.solver
        self.krylov = dict(solver=s.solver_type, precond=s.precond_type, tol=s.tol, maxiter=s.maxiter,
                           restart=s.restart, workspace=KrylovWorkspace(self.dm))
        neumann = np.asarray(self.boundary_nodes.neumann, dtype=np.int64)
        self.engine = PicardEngine(self.dm, "vg", self.phi, solver=s.solver_type, precond=s.precond_type,
                                   krylov_tol=s.tol, krylov_maxiter=s.maxiter, restart=s.restart,
                                   picard_tol=PICARD_TOL, picard_maxiter=PICARD_MAXITER, picard_relative=False,
                                   quad=(self.quad_points, self.weights),
                                   neumann_nodes=neumann if self.bc_info["type"] == "coupled" else None,
                                   neumann_flux=self.bc_info.get("water_flux", {}).get("neumann_flux", 0.0))
        self.cauchy_edges = edges_or_none(self.dm, self.boundary_nodes.cauchy)
        self.initialize_problem()

    def initialize_problem(self):
        self.pressure_head = -1.3 * np.ones(self.nnt)
        self.solute = np.ones(self.nnt) * self.config.solute.c_init

    def solve_richards_step(self, pressure_head_n, thetan_0=None, dt=1e-3):
        """(h, err, iterations) of one Picard-converged step (theta_n is recomputed from h_n on the device)."""
        self.engine.set_state(pressure_head_n)
        res = self.engine.step(dt)
        return self.engine.h_n.clone(), res["error"], res["iterations"]

    def solve_transport_step(self, solute_n, pressure_head, theta, theta_n, water_flux_x, water_flux_z, abs_q,
                             D_xx, D_xz, D_zz, dt):
        sol = self.config.solute
        bc = self.bc_info.get("solute", {})
        c, _ = solute_step(self.dm, solute_n, theta, water_flux_x, water_flux_z, D_xx, D_xz, D_zz, dt,
                           (self.quad_points, self.weights), self.cauchy_edges, bc.get("cauchy_flux", 0.0),
                           bc.get("inlet_conc", sol.c_inlet), **self.krylov)
        return c

    def adapt_time_step(self, dt, iter_count):
        t = self.config.time
        dt_new = _adapt(dt, iter_count, t.m_it, t.M_it, t.lambda_amp, t.lambda_red)
        return max(dt_new, 1e-6)          # the reference's min(., 0.5) is overwritten by this line

    def solve(self, max_steps=None) -> Dict[str, Any]:
        t0 = time.perf_counter()
        cfg = self.config
        dev = self.dm.device
        keys = ("pressure_head", "theta", "solute", "times", "iterations", "errors", "dt_values")
        out = {k: [] for k in keys}
        h_n = torch.as_tensor(self.pressure_head, dtype=torch.float64, device=dev)
        c_n = torch.as_tensor(self.solute, dtype=torch.float64, device=dev)
        sol = cfg.solute
        current_time, dt, steps = 0.0, float(cfg.time.dt_init), 0
        h = theta = c = h_n
        while current_time < cfg.time.Tmax and (max_steps is None or steps < max_steps):
            theta_n = soil("vg", h_n, self.phi)[2]
            h, error, iter_count = self.solve_richards_step(h_n, theta_n, dt)
            qx, qz, aq, Dxx, Dxz, Dzz, theta = flux_dispersion(self.dm, h, self.phi, sol.DL, sol.DT, sol.Dm)
            c = self.solve_transport_step(c_n, h, theta, theta_n, qx, qz, aq, Dxx, Dxz, Dzz, dt)
            dt_new = self.adapt_time_step(dt, iter_count)
            out["pressure_head"].append(h)
            out["theta"].append(theta)
            out["solute"].append(c)
            out["times"].append(current_time)
            out["iterations"].append(iter_count)
            out["errors"].append(error)
            out["dt_values"].append(dt_new)
            h_n, c_n = h, c
            current_time += float(dt)
            dt = dt_new
            steps += 1
        simulation_time = time.perf_counter() - t0
        stack = lambda v: torch.stack(v).cpu().numpy() if v else np.zeros((0, self.nnt))  # noqa: E731
        return {
            "pressure_head": stack(out["pressure_head"]), "theta": stack(out["theta"]),
            "solute": stack(out["solute"]), "times": np.array(out["times"]),
            "iterations": np.array(out["iterations"]), "errors": np.array(out["errors"]),
            "dt_values": np.array(out["dt_values"]), "Pe_values": np.array([]), "Cr_values": np.array([]),
            "points": self.points, "triangles": self.triangles,
            "final_pressure": h.cpu().numpy(), "final_theta": theta.cpu().numpy(), "final_solute": c.cpu().numpy(),
            "simulation_time": simulation_time, "mesh_info": self.mesh_info, "config": cfg,
        }
