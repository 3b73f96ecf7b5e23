"""Coupled water flow + nitrogen transport (drop-in for src/solvers/nitrogen_solver.py:36-412).

``NitrogenSolver(config).solve()`` returns the reference's result dictionary.
Per time step: the Richards step on the device (van Genuchten soil, Neumann
infiltration on the top nodes, free drainage at the bottom, absolute Picard
error < 1e-6, at most 100 iterations -- :100-149); fluxes and dispersion with
the nitrogen dispersivities; K at the new head; then the species chain
NH4+ -> NO2- -> NO3- (:151-235), each with row-lumped mass, first-order decay,
the upstream species as source, Cauchy inflow and free-drainage outflow, solved
on the device; dt adaptation of :401-412.
"""
import time
from typing import Any, Dict

import numpy as np
import torch

from wspm_b200 import context
from wspm_b200.device import KrylovWorkspace, flux_dispersion, soil
from wspm_b200.engine import PicardEngine
from wspm_b200.transport import edges_or_none, nitrogen_species_step

from ..mesh.loader import load_and_validate_mesh
from ..models.boundary import extract_boundary_nodes, get_boundary_condition
from ..numerics.gauss import gauss_triangle

PICARD_TOL, PICARD_MAXITER = 1e-6, 100


def lump_sparse_mass_matrix(mass_matrix):
    """Row-sum lumping (nitrogen_solver.py:37-66); the device path lumps inside the ADR kernel."""
    import scipy.sparse as sp
    m = mass_matrix.to_scipy() if hasattr(mass_matrix, "to_scipy") else sp.csr_matrix(mass_matrix)
    return sp.diags(np.asarray(m.sum(axis=1)).ravel()).tocsr()


class NitrogenSolver:
    """Solver for coupled water flow and nitrogen transport equations."""

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
        coupled = self.bc_info["type"] == "coupled"
        fd = np.asarray(self.boundary_nodes.freedrainage, dtype=np.int64)
        self.engine = PicardEngine(self.dm, "vg", self.phi, solver=s.solver_type, precond=s.precond_type,
                                   krylov_tol=s.tol, krylov_maxiter=s.maxiter, restart=s.restart,
                                   picard_tol=PICARD_TOL, picard_maxiter=PICARD_MAXITER, picard_relative=False,
                                   quad=(self.quad_points, self.weights),
                                   neumann_nodes=np.asarray(self.boundary_nodes.neumann, dtype=np.int64)
                                   if coupled else None,
                                   neumann_flux=self.bc_info.get("water_flux", {}).get("neumann_flux", 0.0),
                                   drainage_nodes=fd if (coupled and fd.size) else None)
        self.cauchy_edges = edges_or_none(self.dm, self.boundary_nodes.cauchy)
        self.fd_edges = edges_or_none(self.dm, self.boundary_nodes.freedrainage)
        self.initialize_problem()

    def initialize_problem(self):
        n = self.config.nitrogen
        self.pressure_head = -1.0 * np.ones(self.nnt)
        self.NH4_concentration = np.ones(self.nnt) * n.c_init_NH4
        self.NO2_concentration = np.ones(self.nnt) * n.c_init_NO2
        self.NO3_concentration = np.ones(self.nnt) * n.c_init_NO3

    def solve_richards_step(self, pressure_head_n, theta_n=None, dt=1e-3):
        self.engine.set_state(pressure_head_n)
        res = self.engine.step(dt)
        return self.engine.h_n.clone(), res["error"], res["iterations"]

    def solve_nitrogen_transport_step(self, pressure_head, theta, water_flux_x, water_flux_z, D_xx, D_xz, D_zz,
                                      NH4_n, NO2_n, NO3_n, dt, Konduc):
        n = self.config.nitrogen
        sf = self.bc_info.get("solute_flux", {})
        flux = sf.get("cauchy_flux", 0.0)
        common = dict(quad=(self.quad_points, self.weights), cauchy_edges=self.cauchy_edges, cauchy_flux=flux,
                      fd_edges=self.fd_edges, **self.krylov)
        args = (theta, water_flux_x, water_flux_z, D_xx, D_xz, D_zz, Konduc, dt)
        NH4, _ = nitrogen_species_step(self.dm, NH4_n, *args, mu=n.mu1, sorption=n.rho * n.Kd,
                                       c_in=n.c_inlet_NH4, **common)
        NO2, _ = nitrogen_species_step(self.dm, NO2_n, *args, mu=n.mu2, mu_up=n.mu1, c_up=NH4,
                                       c_in=n.c_inlet_NO2, **common)
        NO3, _ = nitrogen_species_step(self.dm, NO3_n, *args, mu=n.mu3, mu_up=n.mu2, c_up=NO2,
                                       c_in=n.c_inlet_NO3, **common)
        return NH4, NO2, NO3

    @staticmethod
    def adapt_time_step(dt, iter_count):
        if iter_count <= 5:
            return min(1.2 * dt, 0.01)
        if iter_count <= 15:
            return dt
        return max(0.5 * dt, 1e-6)

    def solve(self, max_steps=None) -> Dict[str, Any]:
        t0 = time.perf_counter()
        cfg = self.config
        dev = self.dm.device
        keys = ("pressure_head", "theta", "NH4", "NO2", "NO3", "times", "iterations", "errors", "dt_values")
        out = {k: [] for k in keys}
        f64 = dict(dtype=torch.float64, device=dev)
        h_n = torch.as_tensor(self.pressure_head, **f64)
        NH4_n = torch.as_tensor(self.NH4_concentration, **f64)
        NO2_n = torch.as_tensor(self.NO2_concentration, **f64)
        NO3_n = torch.as_tensor(self.NO3_concentration, **f64)
        n = cfg.nitrogen
        current_time, dt, steps = 0.0, float(cfg.time.dt_init), 0
        while current_time < cfg.time.Tmax and (max_steps is None or steps < max_steps):
            theta_n = soil("vg", h_n, self.phi)[2]
            h, error, iter_count = self.solve_richards_step(h_n, theta_n, dt)
            qx, qz, aq, Dxx, Dxz, Dzz, theta = flux_dispersion(self.dm, h, self.phi, n.DL, n.DT, n.Dm)
            Konduc = soil("vg", h, self.phi)[1]
            NH4, NO2, NO3 = self.solve_nitrogen_transport_step(h, theta, qx, qz, Dxx, Dxz, Dzz, NH4_n, NO2_n, NO3_n,
                                                               dt, Konduc)
            dt_new = self.adapt_time_step(dt, iter_count)
            for k, v in (("pressure_head", h), ("theta", theta), ("NH4", NH4), ("NO2", NO2), ("NO3", NO3)):
                out[k].append(v)
            out["times"].append(current_time)
            out["iterations"].append(iter_count)
            out["errors"].append(error)
            out["dt_values"].append(dt)          # the reference records the step's own dt here
            h_n, NH4_n, NO2_n, NO3_n = h, NH4, NO2, NO3
            current_time += dt
            dt = dt_new
            steps += 1
        simulation_time = time.perf_counter() - t0
        stack = lambda v: torch.stack(v).cpu().numpy() if v else np.zeros((0, self.nnt))  # noqa: E731
        return {
            "pressure_head": stack(out["pressure_head"]), "theta": stack(out["theta"]),
            "NH4_concentration": stack(out["NH4"]), "NO2_concentration": stack(out["NO2"]),
            "NO3_concentration": stack(out["NO3"]), "times": np.array(out["times"]),
            "iterations": np.array(out["iterations"]), "errors": np.array(out["errors"]),
            "dt_values": np.array(out["dt_values"]), "points": self.points, "triangles": self.triangles,
            "simulation_time": simulation_time, "mesh_info": self.mesh_info, "config": cfg,
        }
