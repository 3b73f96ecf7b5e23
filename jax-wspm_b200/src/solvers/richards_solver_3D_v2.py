"""3D Richards solver (drop-in for src/solvers/richards_solver_3D_v2.py:41-302).

Test3D: Gardner soil on the 15.24 m cube, Kuhn-split hexahedra, top
boundary (1/a0) log(eps0 + (1-eps0) sin(pi x/L) sin(pi y/L)), other faces -15.
The reference's Picard loop is a host loop with an absolute error < 1e-4 and
at most 30 iterations (:177-222), and the recorded theta is the step-start
theta (:261); the engine runs the same loop on the device.
"""
import numpy as np

from wspm_b200.device import merge_dirichlet

from ..mesh.loader import load_and_validate_mesh
from ..models.boundary import BOTTOM_VALUE, extract_boundary_nodes, get_boundary_condition
from ..numerics.gauss_3D import gauss_tetrahedron
from .richards_solver_v2 import RichardsSolver

PROFILE_3D = {"tol": 1e-4, "maxiter": 30, "relative": False, "theta_at_end": False}


class RichardsSolver3D(RichardsSolver):
    dimension = 3

    def __init__(self, config, picard_profile: str = None):
        self.config = config
        self.picard = dict(PROFILE_3D)
        self.setup_solver()

    def setup_solver(self):
        self.points, self.tetrahedra, self.mesh_info = load_and_validate_mesh(
            self.config.mesh.mesh_size, self.config.mesh.mesh_dir, "Test3D", prefix=("p_3D", "t_3D"))
        self.triangles = self.tetrahedra            # element array used by the shared engine code
        self.boundary_nodes = extract_boundary_nodes(self.points, "Test3D")
        self.quad_points, self.weights = gauss_tetrahedron(4)
        self.bc_info = get_boundary_condition("Test3D")
        self.nnt = len(self.points)
        self.initialize_problem()
        self._engine = None

    def soil(self):
        return "exp", self.config.exponential.to_array()

    def initialize_problem(self):
        self.pressure_head = -15.24 * np.ones(self.nnt)
        self.L = 15.24
        top = self.boundary_nodes.top
        eps0_top = np.exp(self.config.exponential.alpha0 * self.pressure_head[top])
        self.hupper = self.bc_info["upper_bc"](self.points[top][:, 0], self.points[top][:, 1], self.L,
                                               self.config.exponential.alpha0, eps0_top)
        self.bc_val = merge_dirichlet(self.nnt, [(top, self.hupper), (self.boundary_nodes.bottom, BOTTOM_VALUE)])

    def solve(self):
        res = super().solve()
        res["tetrahedra"] = res.pop("triangles")
        res["final_theta"] = res["theta"][-1]
        return res
