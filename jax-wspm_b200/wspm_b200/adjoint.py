"""Implicit Richards time stepping with per-element soil parameters, and its discrete adjoint.

Parameters: ``params[e] = (ln Ks_e, ln alpha_e, ln n_e)`` per triangle,
theta_r / theta_s shared.  Forward: per step a Picard loop on the device
(``wspm_elem_assemble_richards`` + Jacobi-CG), host-driven convergence test.
Loss: sum over steps n = 1..N and sensor nodes s of
(theta_node_s(h^n) - target[n-1, s])^2, with theta_node the lumped-mass average
of the element water contents at the node.

Backward (discrete adjoint of the implicit stepper, FP64): states are
checkpointed every ``checkpoint_every`` steps during the forward run and each
segment is recomputed (bitwise, the kernels are deterministic) before it is
swept backwards.  Per step n = N..1, one transpose solve with the exact
Jacobian of the converged-step residual,
    J(h^n)^T lam^n = dL/dh^n + (sum_e Ml C(h^n) / dt) lam^{n+1}   (free rows)
then grad += -(dR^n/dp)^T lam^n + dL_n/dp (direct sensor term).
``ElementRichardsLoss`` wraps forward and backward as a torch.autograd.Function.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._lib import check, dptr, lib
from .device import KrylovWorkspace, krylov_solve
from .engine import default_rule


class ElementParamRichards:
    def __init__(self, dm, theta_r, theta_s, bc_val, dt, n_steps, quad=None, picard_tol=1e-10, picard_maxiter=200,
                 krylov_tol=1e-12, krylov_maxiter=5000, adjoint_tol=1e-12, adjoint_restart=30,
                 adjoint_maxiter=200, checkpoint_every=10):
        if dm.dim != 2:
            raise ValueError("per-element soil parameters are implemented for 2D triangles")
        self.dm = dm
        self.thr, self.ths = float(theta_r), float(theta_s)
        dev = dm.device
        self.bc_val = torch.as_tensor(np.asarray(bc_val, dtype=np.float64), device=dev)
        self.dt, self.n_steps = float(dt), int(n_steps)
        Q, W = default_rule(2) if quad is None else quad
        self.Q = _lib.dbl_array(np.ascontiguousarray(Q, dtype=np.float64).ravel())
        self.W = _lib.dbl_array(np.ascontiguousarray(W, dtype=np.float64).ravel())
        self.nq = len(np.asarray(W).ravel())
        self.picard_tol, self.picard_maxiter = float(picard_tol), int(picard_maxiter)
        self.krylov_tol, self.krylov_maxiter = float(krylov_tol), int(krylov_maxiter)
        self.adjoint_tol, self.adjoint_restart = float(adjoint_tol), int(adjoint_restart)
        self.adjoint_maxiter = int(adjoint_maxiter)
        self.checkpoint_every = max(1, int(checkpoint_every))
        self.ws = KrylovWorkspace(dm)
        n = dm.n_nodes
        f64 = dict(dtype=torch.float64, device=dev)
        self.vals, self.rhs, self.dinv = dm.empty_vals(), torch.empty(n, **f64), torch.empty(n, **f64)
        self.theta_node, self.dtheta, self.mass = (torch.empty(n, **f64) for _ in range(3))
        self.picard_its = []

    # -- C-ABI wrappers -------------------------------------------------------------------
    def _common(self, params):
        return (ctypes.byref(self.dm.c_mesh), ctypes.byref(self.dm.c_pat), dptr(params), self.thr, self.ths,
                self.Q, self.W, self.nq)

    def _st(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def assemble(self, params, h_m, h_n):
        check("elem_assemble_richards", lib.wspm_elem_assemble_richards(
            *self._common(params), self.dt, dptr(self.bc_val), dptr(h_m), dptr(h_n), dptr(self.vals),
            dptr(self.rhs), dptr(self.dinv), self._st()))

    def theta_nodes(self, params, h):
        check("elem_theta_node", lib.wspm_elem_theta_node(*self._common(params), dptr(h), dptr(self.theta_node),
                                                          dptr(self.dtheta), dptr(self.mass), self._st()))
        return self.theta_node, self.dtheta, self.mass

    # -- forward ---------------------------------------------------------------------------
    def step(self, params, h_n):
        """One implicit step: Picard iterations (relative error) to picard_tol; returns h^{n+1}."""
        h_m = h_n.clone()
        for it in range(self.picard_maxiter):
            self.assemble(params, h_m, h_n)
            x, _ = krylov_solve(self.dm, self.vals, self.rhs, h_m, "cg", dinv=self.dinv, tol=self.krylov_tol,
                                maxiter=self.krylov_maxiter, workspace=self.ws)
            err = float(torch.linalg.norm(x - h_m) / torch.linalg.norm(x))
            h_m = x
            if err < self.picard_tol:
                break
        self.picard_its.append(it + 1)
        return h_m

    def forward(self, params, h0, sensors, target):
        """Loss of the run; keeps the checkpoints for backward()."""
        self.params = params
        self.sensors = torch.as_tensor(sensors, dtype=torch.int64, device=self.dm.device)
        self.target = torch.as_tensor(target, dtype=torch.float64, device=self.dm.device)
        h = torch.as_tensor(h0, dtype=torch.float64, device=self.dm.device).clone()
        self.checkpoints = {0: h.clone()}
        self.picard_its = []
        loss = torch.zeros((), dtype=torch.float64, device=self.dm.device)
        for n in range(1, self.n_steps + 1):
            h = self.step(params, h)
            th = self.theta_nodes(params, h)[0]
            loss = loss + torch.sum((th[self.sensors] - self.target[n - 1]) ** 2)
            if n % self.checkpoint_every == 0 and n < self.n_steps:
                self.checkpoints[n] = h.clone()
        self.final = h
        return loss

    def simulate_theta(self, params, h0, sensors):
        """theta at the sensors after every step (the synthetic target of a second parameter draw)."""
        s = torch.as_tensor(sensors, dtype=torch.int64, device=self.dm.device)
        h = torch.as_tensor(h0, dtype=torch.float64, device=self.dm.device).clone()
        out = []
        for _ in range(self.n_steps):
            h = self.step(params, h)
            out.append(self.theta_nodes(params, h)[0][s].clone())
        return torch.stack(out)

    # -- backward --------------------------------------------------------------------------
    def backward(self):
        """dL/dparams, shape (E, 3), by the discrete adjoint."""
        params = self.params
        dm = self.dm
        n_e = dm.n_elems
        grad = torch.zeros(3 * n_e, dtype=torch.float64, device=dm.device)
        nn = dm.n_nodes
        f64 = dict(dtype=torch.float64, device=dm.device)
        g = torch.zeros(nn, **f64)
        wl = torch.zeros(nn, **f64)
        rhs = torch.zeros(nn, **f64)
        jt_vals, jt_dinv = dm.empty_vals(), torch.empty(nn, **f64)
        lam_next = None
        starts = sorted(self.checkpoints)
        ends = starts[1:] + [self.n_steps]
        for c0, c1 in reversed(list(zip(starts, ends))):
            # recompute the states of this segment from its checkpoint
            states = {c0: self.checkpoints[c0]}
            h = states[c0]
            for n in range(c0 + 1, c1 + 1):
                h = self.step(params, h)
                states[n] = h
            for n in range(c1, c0, -1):
                h, h_old = states[n], states[n - 1]
                th, dth, mass = self.theta_nodes(params, h)
                res = th[self.sensors] - self.target[n - 1]
                g.zero_()
                wl.zero_()
                g[self.sensors] = 2.0 * res * dth[self.sensors]
                wl[self.sensors] = 2.0 * res
                check("elem_adjoint_rhs", lib.wspm_elem_adjoint_rhs(
                    *self._common(params), self.dt, dptr(self.bc_val), dptr(h), dptr(lam_next), dptr(g),
                    dptr(rhs), self._st()))
                check("elem_assemble_jt", lib.wspm_elem_assemble_jt(
                    *self._common(params), self.dt, dptr(self.bc_val), dptr(h), dptr(h_old), dptr(jt_vals),
                    dptr(jt_dinv), self._st()))
                x0 = lam_next if lam_next is not None else torch.zeros(nn, **f64)
                lam, _ = krylov_solve(dm, jt_vals, rhs, x0, "gmres", dinv=jt_dinv, tol=self.adjoint_tol,
                                      maxiter=self.adjoint_maxiter, restart=self.adjoint_restart, workspace=self.ws)
                check("elem_param_grad", lib.wspm_elem_param_grad(
                    *self._common(params), self.dt, dptr(self.bc_val), dptr(h), dptr(h_old), dptr(lam), dptr(wl),
                    dptr(mass), dptr(grad), self._st()))
                lam_next = lam
        return grad.view(n_e, 3)


class ElementRichardsLoss(torch.autograd.Function):
    """loss = ElementRichardsLoss.apply(params, problem, h0, sensors, target); d loss / d params by the adjoint."""

    @staticmethod
    def forward(ctx, params, problem, h0, sensors, target):
        p = params.detach().contiguous().to(torch.float64)
        loss = problem.forward(p.view(-1), h0, sensors, target)
        ctx.problem = problem
        return loss

    @staticmethod
    def backward(ctx, grad_out):
        grad = ctx.problem.backward()
        return grad_out * grad, None, None, None, None


def timed(fn):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0
