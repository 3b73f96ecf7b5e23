"""Device-resident mesh + pattern and thin tensor wrappers of the C ABI.

``DeviceMesh`` uploads a mesh and its SELL-32 pattern once (torch tensors on
the current CUDA device) and keeps the ``wspm_mesh`` / ``wspm_pattern``
structs that the C ABI reads.  The functions below take and return torch
tensors and call libwspm.so on the current torch stream; they never copy
data to the host.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, dptr, lib
from .pattern import Pattern


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _require_cuda(t, dtype, name, numel=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"{name} must have {numel} elements, got {t.numel()}")
    return t


class DeviceMesh:
    """Mesh + pattern on the GPU.  ``points`` (N, dim) float64, ``elements`` (E, dim+1)."""

    def __init__(self, points, elements, device=None, pattern=None, layout="auto", extra_pairs=None,
                 builder="native"):
        points = np.ascontiguousarray(points, dtype=np.float64)
        elements = np.ascontiguousarray(elements, dtype=np.int64)
        if elements.ndim != 2 or elements.shape[1] != points.shape[1] + 1:
            raise ValueError("elements must have dim+1 columns")
        if elements.size and (elements.min() < 0 or elements.max() >= points.shape[0]):
            raise ValueError("Element indices out of bounds")
        self.device = torch.device(device if device is not None else "cuda")
        self.points_host, self.elements_host = points, elements
        self.n_nodes, self.dim = points.shape
        self.n_elems, self.nv = elements.shape
        self.pattern = pattern if pattern is not None else Pattern(elements, self.n_nodes, layout=layout,
                                                                   extra_pairs=extra_pairs, builder=builder)
        pat = self.pattern
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.conn = t(elements.astype(np.int32))
        self.coords = t(points)
        dev_arrays = getattr(pat, "device_arrays", None)
        if dev_arrays is not None and dev_arrays["cols"].device == self.device:
            # built on this GPU (Pattern(builder="device")): use the arrays where they are
            for k in ("slice_ptr", "slice_width", "cols", "diag_pos", "inc_ptr", "inc_width", "inc_elem",
                      "inc_slots", "sell_index", "diag_offsets"):
                setattr(self, k, dev_arrays[k])
        else:
            self.slice_ptr = t(pat.slice_ptr)
            self.slice_width = t(pat.slice_width)
            self.cols = t(pat.cols)
            self.diag_pos = t(pat.diag_pos)
            self.inc_ptr = t(pat.inc_ptr)
            self.inc_width = t(pat.inc_width)
            self.inc_elem = t(pat.inc_elem)
            self.inc_slots = t(pat.inc_slots.view(np.int32))
            self.sell_index = t(pat.sell_index)
            self.diag_offsets = t(pat.diag_offsets if pat.n_diags else np.zeros(1, dtype=np.int32))
        self.c_mesh = _lib.WspmMesh(self.n_nodes, self.n_elems, self.dim, self.nv, self.conn.data_ptr(),
                                    self.coords.data_ptr())
        self.c_pat = _lib.WspmPattern(pat.n_rows, pat.n_slices, pat.max_width, pat.max_inc, pat.nnz_padded,
                                      self.slice_ptr.data_ptr(), self.slice_width.data_ptr(), self.cols.data_ptr(),
                                      self.diag_pos.data_ptr(), self.inc_ptr.data_ptr(),
                                      self.inc_width.data_ptr(), self.inc_elem.data_ptr(),
                                      self.inc_slots.data_ptr(), pat.n_diags, 0,
                                      self.diag_offsets.data_ptr() if pat.n_diags else None)

    @property
    def nnz_padded(self):
        return self.pattern.nnz_padded

    def empty_vals(self, dtype=torch.float64):
        return torch.empty(self.pattern.nnz_padded, dtype=dtype, device=self.device)

    def vec(self, fill=None, dtype=torch.float64):
        if fill is None:
            return torch.empty(self.n_nodes, dtype=dtype, device=self.device)
        return torch.full((self.n_nodes,), float(fill), dtype=dtype, device=self.device)


class SparseMatrix:
    """Global matrix in SELL-32 form on the GPU (drop-in for the reference's BCOO)."""

    def __init__(self, dmesh, vals):
        self.dmesh = dmesh
        self.vals = vals
        self.shape = (dmesh.n_nodes, dmesh.n_nodes)

    @property
    def nse(self):
        return self.dmesh.pattern.nnz

    # CSR view (the fields a CSR matrix object has; the storage stays DIA / SELL-32 on the device)
    @property
    def indptr(self):
        return self.dmesh.pattern.csr_indptr

    @property
    def indices(self):
        return self.dmesh.pattern.csr_indices

    @property
    def data(self):
        return self.csr_values()

    def __matmul__(self, x):
        return spmv(self.dmesh, self.vals, x)

    def csr_values(self):
        return self.vals[self.dmesh.sell_index]

    def to_scipy(self):
        return self.dmesh.pattern.to_scipy(self.vals.detach().cpu().numpy())

    def todense(self):
        return torch.from_numpy(self.to_scipy().toarray())

    def diagonal(self):
        return jacobi_dinv(self.dmesh, self.vals).reciprocal()


CSRMatrix = SparseMatrix   # the name under which the C-ABI shims describe the matrix object


# ---------------------------------------------------------------- soil
def soil(model, h, phi):
    """(C, K, theta) on the device; model "vg" (6 params) or "exp" (4 params)."""
    _require_cuda(h, torch.float64, "h")
    C, K, th = torch.empty_like(h), torch.empty_like(h), torch.empty_like(h)
    arr = _lib.dbl_array(phi)
    if model == "vg":
        fn = lib.wspm_soil_van_genuchten
    elif model == "exp":
        fn = lib.wspm_soil_exponential
    else:
        raise ValueError(f"unknown soil model {model!r}")
    check("soil", fn(dptr(h), h.numel(), arr, dptr(C), dptr(K), dptr(th), _stream()))
    return C, K, th


# ---------------------------------------------------------------- assembly
def assemble_richards(dm, theta_m, theta_n, h_m, K, C, quad_points, weights, dt, bc_val=None, Ks_elem=None,
                      want_f32=False, want_dinv=True):
    """(vals, rhs, dinv, vals32) of the Richards system (Dirichlet rows fused when bc_val is given)."""
    n = dm.n_nodes
    for name, t in (("theta_m", theta_m), ("theta_n", theta_n), ("h_m", h_m), ("K", K), ("C", C)):
        _require_cuda(t, torch.float64, name, n)
    if bc_val is not None:
        _require_cuda(bc_val, torch.float64, "bc_val", n)
    if Ks_elem is not None:
        _require_cuda(Ks_elem, torch.float64, "Ks_elem", dm.n_elems)
    q = np.ascontiguousarray(quad_points, dtype=np.float64).ravel()
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    vals = dm.empty_vals()
    vals32 = dm.empty_vals(torch.float32) if want_f32 else None
    rhs = dm.vec()
    dinv = dm.vec() if want_dinv else None
    check("assemble_richards", lib.wspm_assemble_richards(
        ctypes.byref(dm.c_mesh), ctypes.byref(dm.c_pat), dptr(theta_m), dptr(theta_n), dptr(h_m), dptr(K), dptr(C),
        dptr(Ks_elem), _lib.dbl_array(q), _lib.dbl_array(w), len(w), float(dt), dptr(bc_val), dptr(vals),
        dptr(vals32), dptr(rhs), dptr(dinv), _stream()))
    return vals, rhs, dinv, vals32


def spmv(dm, vals, x):
    if vals.dtype == torch.float64:
        _require_cuda(x, torch.float64, "x", dm.n_nodes)
        y = torch.empty_like(x)
        check("spmv_f64", lib.wspm_spmv_f64(ctypes.byref(dm.c_pat), dptr(vals), dptr(x), dptr(y), _stream()))
    else:
        _require_cuda(x, torch.float32, "x", dm.n_nodes)
        y = torch.empty_like(x)
        check("spmv_f32", lib.wspm_spmv_f32(ctypes.byref(dm.c_pat), dptr(vals), dptr(x), dptr(y), _stream()))
    return y


def jacobi_dinv(dm, vals):
    dinv = dm.vec()
    check("jacobi_dinv", lib.wspm_jacobi_dinv(ctypes.byref(dm.c_pat), dptr(vals), dptr(dinv), _stream()))
    return dinv


def merge_dirichlet(n, sets):
    """Merge (nodes, values) sets applied in order; later sets win (boundary.py:38-53 order)."""
    val = np.full(n, np.nan)
    for nodes, v in sets:
        nodes = np.asarray(nodes, dtype=np.int64)
        val[nodes] = np.broadcast_to(np.asarray(v, dtype=np.float64), nodes.shape)
    return val


def apply_dirichlet(dm, nodes, values, vals, rhs):
    """In place: rows ``nodes`` -> e_i, rhs[nodes] = values (nodes unique)."""
    nodes_t = torch.as_tensor(np.asarray(nodes, dtype=np.int32), device=dm.device)
    vals_t = torch.as_tensor(np.asarray(values, dtype=np.float64), device=dm.device)
    if torch.unique(nodes_t).numel() != nodes_t.numel():
        raise ValueError("Dirichlet nodes must be unique; merge overlapping sets first")
    check("apply_dirichlet", lib.wspm_apply_dirichlet(ctypes.byref(dm.c_pat), dptr(nodes_t), dptr(vals_t),
                                                      nodes_t.numel(), dptr(vals), dptr(rhs), _stream()))
    return vals, rhs


class KrylovWorkspace:
    """Reusable device workspace for stand-alone solves (keeps solve graphs cached)."""

    def __init__(self, dm):
        self.dm = dm
        self.buffers = {}
        self.result = torch.zeros(4, dtype=torch.int32, device=dm.device)

    def get(self, solver, restart):
        key = (solver, restart if solver == "gmres" else 0)
        if key not in self.buffers:
            need = lib.wspm_krylov_workspace_doubles(self.dm.n_nodes, _lib.SOLVERS[solver], int(restart))
            if need < 0:
                raise ValueError(f"unsupported Krylov configuration {solver} restart={restart}")
            self.buffers[key] = torch.empty(int(need), dtype=torch.float64, device=self.dm.device)
        return self.buffers[key]


def krylov_solve(dm, vals, b, x0, solver="cg", dinv=None, tol=1e-10, atol=0.0, maxiter=100, restart=30,
                 workspace=None, x_out=None):
    """Solve A x = b from x0 on the device; returns (x, status_tensor[4] on device)."""
    if solver not in _lib.SOLVERS:
        raise ValueError(f"Unsupported solver type: {solver}")
    _require_cuda(b, torch.float64, "b", dm.n_nodes)
    ws = workspace if workspace is not None else KrylovWorkspace(dm)
    work = ws.get(solver, restart)
    x = x_out if x_out is not None else torch.empty_like(b)
    x.copy_(x0)
    check("krylov_solve", lib.wspm_krylov_solve(
        ctypes.byref(dm.c_pat), dptr(vals), dptr(b), dptr(x), dptr(dinv), _lib.SOLVERS[solver], float(tol),
        float(atol), int(maxiter), int(restart), dptr(work), work.numel(), dptr(ws.result), _stream()))
    return x, ws.result


def krylov_solve_mixed(dm, vals, b, x0, dinv=None, tol=1e-8, inner_tol=1e-5, inner_maxiter=20000,
                       refine_maxiter=20, vals32=None, workspace=None, x_out=None, result=None, solver="cg",
                       restart=30):
    """A x = b with FP32 Krylov corrections (``solver``: cg, bicgstab or gmres with ``restart``) inside FP64
    iterative refinement (``wspm_krylov_solve_mixed``): the FP64 residual ||b - A x|| reaches tol ||b||.  Returns
    (x, status tensor[4] on the device: status, FP32 iterations (GMRES: restart cycles), corrections, 0).
    ``workspace`` (float64, wspm_krylov_mixed_workspace_doubles entries), ``x_out`` and ``result`` (int32[4]) may
    be kept across calls: the captured graph is cached per argument set, so repeated solves with the same buffers
    replay it."""
    if solver not in _lib.SOLVERS:
        raise ValueError(f"Unsupported solver type: {solver}")
    _require_cuda(b, torch.float64, "b", dm.n_nodes)
    sid = _lib.SOLVERS[solver]
    need = int(lib.wspm_krylov_mixed_workspace_doubles(dm.n_nodes, dm.nnz_padded, sid, int(restart)))
    if need <= 0:
        raise ValueError(f"unsupported mixed solve ({solver}, restart {restart})")
    work = workspace if workspace is not None else torch.empty(need, dtype=torch.float64, device=b.device)
    if work.numel() < need:
        raise ValueError("workspace too small")
    if result is None:
        result = torch.zeros(4, dtype=torch.int32, device=b.device)
    x = x_out if x_out is not None else torch.empty_like(b)
    x.copy_(x0)
    check("krylov_solve_mixed", lib.wspm_krylov_solve_mixed(
        ctypes.byref(dm.c_pat), dptr(vals), dptr(vals32), dptr(b), dptr(x), dptr(dinv), sid, int(restart), float(tol),
        float(inner_tol), int(inner_maxiter), int(refine_maxiter), dptr(work), work.numel(), dptr(result),
        _stream()))
    return x, result


# ---------------------------------------------------------------- transport
def edge_pairs(nodes):
    """Consecutive pairs of a boundary-node list (the reference's edges: boundary.py loops i -> (n[i], n[i+1]))."""
    nodes = np.asarray(nodes, dtype=np.int64)
    return np.stack([nodes[:-1], nodes[1:]], axis=1) if nodes.size > 1 else np.zeros((0, 2), dtype=np.int64)


class BoundaryEdges:
    """Boundary edges of a node list, grouped per boundary node for ``wspm_apply_edge_terms``.

    The edges are the consecutive pairs of ``nodes`` in the given order (the
    reference sorts node sets by id, boundary.py:482-547); the edge Jacobian is
    (x_J - x_I) / 2 as in the reference (horizontal edges).
    """

    def __init__(self, dm, nodes):
        nodes = np.asarray(nodes, dtype=np.int64)
        nb = nodes.size if nodes.size > 1 else 0
        self.nodes = nodes
        x = dm.points_host[:, 0]
        cnt = np.zeros(max(nb, 1), dtype=np.int32)
        loc = np.zeros(2 * max(nb, 1), dtype=np.int32)
        oth = np.zeros(2 * max(nb, 1), dtype=np.int32)
        kot = np.zeros(2 * max(nb, 1), dtype=np.int32)
        jac = np.zeros(2 * max(nb, 1), dtype=np.float64)
        for t in range(nb):
            c = 0
            if t > 0:                                  # edge t-1 = (nodes[t-1], nodes[t]): this node is J
                I, J = nodes[t - 1], nodes[t]
                loc[2 * t + c], oth[2 * t + c], jac[2 * t + c] = 1, I, (x[J] - x[I]) / 2
                kot[2 * t + c] = dm.pattern.slot([J], [I])[0]
                c += 1
            if t < nb - 1:                             # edge t = (nodes[t], nodes[t+1]): this node is I
                I, J = nodes[t], nodes[t + 1]
                loc[2 * t + c], oth[2 * t + c], jac[2 * t + c] = 0, J, (x[J] - x[I]) / 2
                kot[2 * t + c] = dm.pattern.slot([I], [J])[0]
                c += 1
            cnt[t] = c
        t_ = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dm.device)  # noqa: E731
        self._keep = [t_(nodes[:max(nb, 1)].astype(np.int32) if nb else np.zeros(1, np.int32)), t_(cnt), t_(loc),
                      t_(oth), t_(kot), t_(jac)]
        node_t, cnt_t, loc_t, oth_t, kot_t, jac_t = self._keep
        self.c = _lib.WspmEdges(nb, 0, node_t.data_ptr(), cnt_t.data_ptr(), loc_t.data_ptr(), oth_t.data_ptr(),
                                kot_t.data_ptr(), jac_t.data_ptr())
        self.n_bnodes = nb


EDGE_NEUMANN, EDGE_DRAINAGE_WATER, EDGE_CAUCHY, EDGE_DRAINAGE_SOLUTE = 0, 1, 2, 3


def apply_edge_terms(dm, edges, mode, rhs, vals=None, flux=0.0, c_in=0.0, K=None, theta=None):
    """In place: boundary-edge contributions to rhs (and to vals for the matrix modes)."""
    check("apply_edge_terms", lib.wspm_apply_edge_terms(ctypes.byref(dm.c_pat), ctypes.byref(edges.c), int(mode),
                                                        float(flux), float(c_in), dptr(K), dptr(theta), dptr(vals),
                                                        dptr(rhs), _stream()))
    return vals, rhs


def flux_dispersion(dm, h, phi, DL, DT, Dm):
    """(qx, qz, |q|, Dxx, Dxz, Dzz, theta) per node (transport_utilities.py:118-192)."""
    _require_cuda(h, torch.float64, "h", dm.n_nodes)
    out = [torch.empty_like(h) for _ in range(7)]
    check("flux_dispersion_2d", lib.wspm_flux_dispersion_2d(
        ctypes.byref(dm.c_mesh), ctypes.byref(dm.c_pat), dptr(h), _lib.dbl_array(phi), float(DL), float(DT),
        float(Dm), *[dptr(t) for t in out], _stream()))
    return tuple(out)


def assemble_adr(dm, theta, qx, qz, Dxx, Dxz, Dzz, c_n, dt, quad_points, weights, mu=0.0, sorption=0.0,
                 mu_up=0.0, c_up=None, lumped=False, want_dinv=True):
    """(vals, rhs, dinv): A = M/dt + K and b = M c_n/dt + F (consistent or row-lumped mass)."""
    n = dm.n_nodes
    for name, t in (("theta", theta), ("qx", qx), ("qz", qz), ("Dxx", Dxx), ("Dxz", Dxz), ("Dzz", Dzz),
                    ("c_n", c_n)):
        _require_cuda(t, torch.float64, name, n)
    if c_up is not None:
        _require_cuda(c_up, torch.float64, "c_up", n)
    q = np.ascontiguousarray(quad_points, dtype=np.float64).ravel()
    w = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    vals, rhs = dm.empty_vals(), dm.vec()
    dinv = dm.vec() if want_dinv else None
    check("assemble_adr_2d", lib.wspm_assemble_adr_2d(
        ctypes.byref(dm.c_mesh), ctypes.byref(dm.c_pat), dptr(theta), dptr(qx), dptr(qz), dptr(Dxx), dptr(Dxz),
        dptr(Dzz), dptr(c_n), dptr(c_up), float(mu), float(sorption), float(mu_up), int(bool(lumped)),
        _lib.dbl_array(q), _lib.dbl_array(w), len(w), float(dt), dptr(vals), dptr(rhs), dptr(dinv), _stream()))
    return vals, rhs, dinv


# ---------------------------------------------------------------- mass balance, Peclet / Courant
def integrate_2d(dm, f):
    """The reference's integrate_2d_domain of a nodal field (device scalar tensor)."""
    _require_cuda(f, torch.float64, "f", dm.n_nodes)
    work = torch.empty(int(lib.wspm_balance_workspace_doubles()), dtype=torch.float64, device=dm.device)
    out = torch.empty(1, dtype=torch.float64, device=dm.device)
    check("integrate_2d", lib.wspm_integrate_2d(ctypes.byref(dm.c_mesh), dptr(f), dptr(out), dptr(work), _stream()))
    return out[0]


def peclet_courant(dm, qx, qz, theta, Dxx, Dzz, dt):
    """(Pe, Cr) maxima over the mesh (transport_utilities.py:193-242), device tensor [2]."""
    work = torch.empty(int(lib.wspm_balance_workspace_doubles()), dtype=torch.float64, device=dm.device)
    out = torch.empty(2, dtype=torch.float64, device=dm.device)
    check("peclet_courant", lib.wspm_peclet_courant(ctypes.byref(dm.c_mesh), dptr(qx), dptr(qz), dptr(theta),
                                                    dptr(Dxx), dptr(Dzz), float(dt), dptr(out), dptr(work),
                                                    _stream()))
    return out
