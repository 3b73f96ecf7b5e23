"""Picard time-stepping engine: one CUDA graph per implicit time step.

``PicardEngine`` owns every device buffer of a Richards problem and a
``wspm_picard`` plan whose graph runs the whole Picard loop (soil model,
assembly, Dirichlet rows, preconditioned Krylov solve, Picard norm and
convergence test) on the device.  The host time loop mirrors
RichardsSolver.solve (src/solvers/richards_solver_v2.py:272-352): record the
step-start time, adapt dt from the Picard iteration count
(richards_solver_v2.py:91-105) and advance the clock by the new dt.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .device import BoundaryEdges, DeviceMesh, soil

TRI3_POINTS = np.array([[0.166666666666667, 0.166666666666667],
                        [0.166666666666667, 0.666666666666667],
                        [0.666666666666667, 0.166666666666667]])
TRI3_WEIGHTS = np.array([0.166666666666667, 0.166666666666667, 0.166666666666667])
_A, _B = 0.585410196624969, 0.138196601125011
TET4_POINTS = np.array([[_A, _B, _B], [_B, _A, _B], [_B, _B, _A], [_B, _B, _B]])
TET4_WEIGHTS = np.array([0.25, 0.25, 0.25, 0.25])


def default_rule(dim):
    """The reference's quadrature rules: gauss_triangle(3) (gauss.py:31-37), gauss_tetrahedron(4) (gauss_3D.py:29-39)."""
    return (TRI3_POINTS, TRI3_WEIGHTS) if dim == 2 else (TET4_POINTS, TET4_WEIGHTS)


def adapt_time_step(dt, it, m_it=5, M_it=7, lambda_amp=2.0, lambda_red=0.5):
    """richards_solver_v2.py:91-105."""
    if it <= m_it:
        return lambda_amp * dt
    if it <= M_it:
        return dt
    return lambda_red * dt


class PicardEngine:
    def __init__(self, dmesh, soil_model="vg", phi=(), Ks_elem=None, bc_val=None, solver="cg", precond="jacobi",
                 krylov_tol=1e-10, krylov_maxiter=100, restart=30, mixed=False, inner_tol=1e-4,
                 inner_maxiter=2000, refine_maxiter=20, picard_tol=1e-6, picard_maxiter=100, picard_relative=True,
                 quad=None, neumann_nodes=None, neumann_flux=0.0, drainage_nodes=None, element_shapes=True):
        """``element_shapes``: give the plan a buffer in which it records the mesh's distinct element Jacobians;
        with few of them (structured grids) the assembly reads each element-row's geometric factors from a table
        instead of recomputing them, with bitwise identical results."""
        if not isinstance(dmesh, DeviceMesh):
            raise TypeError("dmesh must be a DeviceMesh")
        self.dm = dm = dmesh
        n = dm.n_nodes
        dev = dm.device
        self.soil_model = soil_model
        self.phi = tuple(float(v) for v in phi)
        f64 = dict(dtype=torch.float64, device=dev)
        self.h_n = torch.empty(n, **f64)
        self.theta_n = torch.empty(n, **f64)
        self.h_m = torch.empty(n, **f64)
        self.x = torch.empty(n, **f64)
        self.K = torch.empty(n, **f64)
        self.C = torch.empty(n, **f64)
        self.theta_m = torch.empty(n, **f64)
        self.vals = dm.empty_vals()
        self.vals32 = dm.empty_vals(torch.float32) if mixed else None
        self.rhs = torch.empty(n, **f64)
        self.dinv = torch.empty(n, **f64)
        self.work = torch.empty(int(lib.wspm_picard_workspace_doubles(n, 1 if mixed else 0)), **f64)
        self.dt_dev = torch.zeros(1, **f64)
        self.result = torch.zeros(8, dtype=torch.int32, device=dev)
        self.result_f64 = torch.zeros(4, **f64)
        self.Ks_elem = None if Ks_elem is None else torch.as_tensor(np.asarray(Ks_elem, dtype=np.float64)).to(dev)
        self.bc_val = None if bc_val is None else torch.as_tensor(np.asarray(bc_val, dtype=np.float64)).to(dev)
        Q, W = default_rule(dm.dim) if quad is None else quad
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        d = _lib.WspmPicardDesc()
        d.mesh = ctypes.pointer(dm.c_mesh)
        d.pat = ctypes.pointer(dm.c_pat)
        d.soil_model = _lib.SOIL_VG if soil_model == "vg" else _lib.SOIL_EXP
        for j, v in enumerate(self.phi[:6]):
            d.phi[j] = v
        d.Ks_elem = self.Ks_elem.data_ptr() if self.Ks_elem is not None else None
        d.bc_val = self.bc_val.data_ptr() if self.bc_val is not None else None
        for j, v in enumerate(Q.ravel()):
            d.quad_points[j] = v
        for j, v in enumerate(W):
            d.weights[j] = v
        d.nq = len(W)
        d.solver = _lib.SOLVERS[solver]
        d.precond = _lib.PRECONDS[precond]
        d.krylov_tol, d.krylov_maxiter, d.restart = float(krylov_tol), int(krylov_maxiter), int(restart)
        d.mixed, d.inner_tol = int(bool(mixed)), float(inner_tol)
        d.inner_maxiter, d.refine_maxiter = int(inner_maxiter), int(refine_maxiter)
        d.picard_tol, d.picard_maxiter, d.picard_relative = float(picard_tol), int(picard_maxiter), int(picard_relative)
        for name in ("h_n", "theta_n", "h_m", "x", "K", "C", "theta_m", "vals", "rhs", "dinv", "work", "dt_dev",
                     "result", "result_f64"):
            setattr(d, name, getattr(self, name).data_ptr())
        d.vals32 = self.vals32.data_ptr() if self.vals32 is not None else None
        d.work_doubles = self.work.numel()
        self.Ks_inc = None
        if self.Ks_elem is not None:        # Ks_elem in incidence order, refreshed by the step graph
            self.Ks_inc = torch.empty(int(lib.wspm_picard_ks_inc_doubles(ctypes.byref(dm.c_pat))), **f64)
            d.Ks_inc = self.Ks_inc.data_ptr()
        # element shapes: the plan tags the incidence words with them when the mesh has few distinct Jacobians
        self.shape_buf = None
        if element_shapes:
            nbytes = int(lib.wspm_picard_shape_bytes(ctypes.byref(dm.c_mesh), ctypes.byref(dm.c_pat)))
            if nbytes > 0:
                self.shape_buf = torch.empty(nbytes, dtype=torch.uint8, device=dm.device)
                d.shapes = self.shape_buf.data_ptr()
        # boundary-edge rhs terms (Neumann flux, free drainage of water), applied after assembly
        self.neumann = BoundaryEdges(dm, neumann_nodes) if neumann_nodes is not None else None
        self.drainage = BoundaryEdges(dm, drainage_nodes) if drainage_nodes is not None else None
        d.neumann = ctypes.pointer(self.neumann.c) if self.neumann is not None else None
        d.neumann_flux = float(neumann_flux)
        d.drainage = ctypes.pointer(self.drainage.c) if self.drainage is not None else None
        self._edge_kernels = sum(1 for e in (self.neumann, self.drainage) if e is not None and e.n_bnodes > 0)
        self.desc = d
        self.plan = ctypes.c_void_p()
        torch.cuda.synchronize(dev)
        check("picard_create", lib.wspm_picard_create(ctypes.byref(d), ctypes.byref(self.plan)))
        self.config = dict(solver=solver, precond=precond, krylov_tol=krylov_tol, krylov_maxiter=krylov_maxiter,
                           restart=restart, mixed=mixed, picard_tol=picard_tol, picard_maxiter=picard_maxiter,
                           picard_relative=picard_relative)

    def __del__(self):
        plan = getattr(self, "plan", None)
        if plan is not None and plan.value:
            try:
                lib.wspm_picard_destroy(plan)
            except Exception:
                pass
            self.plan = None

    def assemble(self):
        """One assembly of the current system (vals, rhs, dinv; vals32 on a mixed plan) with the step's kernel."""
        st = torch.cuda.current_stream()
        check("picard_assemble", lib.wspm_picard_assemble(self.plan, ctypes.c_void_p(st.cuda_stream)))

    def element_shape_count(self):
        """Distinct element Jacobians the plan's assembly takes from its shape table (0: it recomputes every
        element's geometry)."""
        return int(lib.wspm_picard_shapes(self.plan))

    @property
    def live_diagonals(self):
        """DIA plans: bit mask of the diagonals that can hold nonzeros (the others are structural zeros whose
        loads the step skips); None for SELL patterns."""
        m = int(lib.wspm_picard_dia_live(self.plan))
        return None if m < 0 else m

    # -- device-side step -----------------------------------------------------
    def set_state(self, h):
        self.h_n.copy_(torch.as_tensor(h, dtype=torch.float64).to(self.dm.device).reshape(-1))

    host_loop = False     # True: loops driven from the host (profiling tools); same kernels

    def launch_step(self, dt, stream=None):
        """Enqueue one time step (no host synchronisation in the default device-loop mode)."""
        st = stream if stream is not None else torch.cuda.current_stream()
        if getattr(self, "_dt_set", None) != float(dt):
            self.dt_dev.fill_(float(dt))
            self._dt_set = float(dt)
        fn = lib.wspm_picard_step_host if self.host_loop else lib.wspm_picard_step
        check("picard_step", fn(self.plan, ctypes.c_void_p(st.cuda_stream)))

    def kernel_launches(self, its, refinements, krylov_launches):
        """Kernels the step graph launched (device counters; graph structure in picard.cu).

        Per step: state resets, step_init, step_finish.  Per Picard iteration: assembly, edge-term
        kernels, the x0 copy, the Krylov init kernels, picard_update (which also evaluates the soil
        law at the new iterate).  The Krylov
        loop itself is counted on the device (one persistent kernel per CG solve, 4 kernels per
        BiCGSTAB iteration, 4m+4 per GMRES cycle); each refinement adds correction + residual.
        The mixed path's refinement start is one kernel either way (the stand-alone residual, or
        the one-block decision after an assembly that computed the residual of its rows).
        """
        cfg = self.config
        e = self._edge_kernels
        if cfg["mixed"]:
            return 5 + (4 + e) * its + 2 * refinements + krylov_launches
        if cfg["solver"] == "gmres":
            return 4 + (5 + e) * its + krylov_launches
        if cfg["solver"] == "bicgstab":
            return 4 + (4 + e) * its + krylov_launches
        return 4 + (3 + e) * its + krylov_launches

    def read_result(self):
        r = self.result.cpu().numpy()
        f = self.result_f64.cpu().numpy()
        out = {"status": int(r[0]), "iterations": int(r[1]), "krylov_iterations": int(r[2]),
               "refinements": int(r[3]), "krylov_cap_hits": int(r[4]), "krylov_status": int(r[5]),
               "krylov_launches": int(r[6]), "error": float(f[0]), "krylov_kernel_seconds": float(f[1])}
        out["launches"] = self.kernel_launches(out["iterations"], out["refinements"], out["krylov_launches"])
        return out

    def step(self, dt):
        self.launch_step(dt)
        return self.read_result()

    def theta(self, h=None):
        h = self.h_n if h is None else h
        return soil(self.soil_model, h, self.phi)[2]

    # -- host time loop (reference semantics) ---------------------------------
    def run(self, h0, dt0, tmax, theta_at_end=True, fixed_dt=False, max_steps=None, keep_fields=True,
            time_params=None):
        tp = time_params or {}
        self.set_state(h0)
        out = {k: [] for k in ("pressure_head", "theta", "times", "iterations", "errors", "dt_values",
                               "krylov_iterations", "status")}
        t = 0.0
        dt = float(dt0)
        steps = 0
        t0 = time.perf_counter()
        while t < tmax and (max_steps is None or steps < max_steps):
            theta_start = self.theta().clone() if (keep_fields and not theta_at_end) else None
            res = self.step(dt)
            dt_new = dt if fixed_dt else float(adapt_time_step(dt, res["iterations"], **tp))
            if keep_fields:
                out["pressure_head"].append(self.h_n.clone())
                out["theta"].append(self.theta().clone() if theta_at_end else theta_start)
            out["times"].append(t)
            out["iterations"].append(res["iterations"])
            out["errors"].append(res["error"])
            out["dt_values"].append(dt_new)
            out["krylov_iterations"].append(res["krylov_iterations"])
            out["status"].append(res["status"])
            t += dt_new
            dt = dt_new
            steps += 1
        out["simulation_time"] = time.perf_counter() - t0
        if keep_fields:
            out["pressure_head"] = torch.stack(out["pressure_head"]).cpu().numpy() if out["pressure_head"] else np.zeros((0, self.dm.n_nodes))
            out["theta"] = torch.stack(out["theta"]).cpu().numpy() if out["theta"] else np.zeros((0, self.dm.n_nodes))
        for k in ("times", "iterations", "errors", "dt_values", "krylov_iterations", "status"):
            out[k] = np.array(out[k])
        return out
