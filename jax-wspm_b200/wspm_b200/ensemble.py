"""Batched ensemble of independent 2D Richards domains (one persistent launch per step).

The reference runs one ``RichardsSolver`` per domain (richards_solver_v2.py);
an ensemble there is a Python loop over solver instances.  ``Ensemble`` puts
the domains on the diagonal of one mesh (node and element ids offset per
domain, SELL-32 pattern over the union) and ``wspm_ensemble_step`` advances
every domain still below ``tmax`` by one implicit step in a single launch:
each CTA -- or each thread-block cluster of ``cluster_size`` CTAs, which spreads
a domain over that many SMs -- takes the next domain (largest first), runs its
Picard loop with its own soil parameters, Dirichlet values and dt, and adapts
that dt.  Domains that reached ``tmax`` are masked out of later launches.

``autotune()`` times one step at each (CTA size, cluster size) the kernel
supports on a copy of the state and keeps the fastest.  ``run_device()`` runs
the time loop itself on the device: one CUDA graph whose WHILE node repeats the
step launch until every domain reached ``tmax`` (or a step cap).
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._lib import check, dptr, lib
from .device import DeviceMesh
from .engine import default_rule

BLOCK_SIZES = (128, 256, 512)
CLUSTER_SIZES = (1, 2, 4, 8, 16)
LAUNCH_SHAPES = tuple((tb, cs) for cs in CLUSTER_SIZES for tb in ((128, 256, 512) if cs == 1 else (512,)))


def partition_domains(work, world):
    """Split domain ids over `world` ranks, balancing the summed work (e.g. nnz): largest first, each to the
    least-loaded rank (ties: lowest rank).  Deterministic; every domain goes to exactly one rank."""
    work = np.asarray(work, dtype=np.float64)
    load = np.zeros(int(world))
    parts = [[] for _ in range(int(world))]
    for d in np.argsort(-work, kind="stable"):
        r = int(np.argmin(load))
        parts[r].append(int(d))
        load[r] += work[d]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def gather_domain_results(local_ids, local_values, n_domains, world):
    """Rank 0 receives every rank's (ids, values) once, at the end of a run (host objects over the process
    group); returns the values in domain order on rank 0, None elsewhere."""
    if world == 1:
        out = np.zeros(n_domains, dtype=np.asarray(local_values).dtype)
        out[np.asarray(local_ids)] = local_values
        return out
    import torch.distributed as dist
    got = [None] * world
    dist.all_gather_object(got, (np.asarray(local_ids).tolist(), np.asarray(local_values).tolist()))
    if dist.get_rank() != 0:
        return None
    out = np.zeros(n_domains, dtype=np.asarray(local_values).dtype)
    for ids, vals in got:
        out[np.asarray(ids, dtype=np.int64)] = vals
    return out


class Ensemble:
    """Independent domains d = 0..D-1, each ``(points, triangles, phi[6], bc_val or None, Ks_elem or None)``."""

    def __init__(self, domains, dt0, tmax, krylov_tol=1e-10, krylov_maxiter=1000, picard_tol=1e-6,
                 picard_maxiter=100, picard_relative=True, time_params=None, quad=None, device=None):
        dev = torch.device(device or "cuda")
        D = len(domains)
        if D == 0:
            raise ValueError("empty ensemble")
        sizes = np.array([len(d[0]) for d in domains], dtype=np.int64)
        node_off = np.zeros(D + 1, dtype=np.int64)
        np.cumsum(sizes, out=node_off[1:])
        pts = np.concatenate([np.asarray(d[0], dtype=np.float64) for d in domains])
        tri = np.concatenate([np.asarray(d[1], dtype=np.int64) + node_off[i] for i, d in enumerate(domains)])
        phi = np.stack([np.asarray(d[2], dtype=np.float64).reshape(6) for d in domains])
        N = int(node_off[-1])
        bc = np.full(N, np.nan)
        ks = np.ones(len(tri))
        has_ks = False
        e0 = 0
        for i, d in enumerate(domains):
            ne = len(d[1])
            if d[3] is not None:
                bc[node_off[i]:node_off[i + 1]] = np.asarray(d[3], dtype=np.float64)
            if len(d) > 4 and d[4] is not None:
                ks[e0:e0 + ne] = np.asarray(d[4], dtype=np.float64)
                has_ks = True
            e0 += ne
        self.n_domains, self.sizes, self.node_off_host = D, sizes, node_off
        self.dm = DeviceMesh(pts, tri, layout="sell", device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        self.node_off = torch.as_tensor(node_off, device=dev)
        self.order = torch.as_tensor(np.argsort(-sizes, kind="stable").astype(np.int32), device=dev)
        self.phi = torch.as_tensor(phi.ravel(), **f64)
        self.bc_val = torch.as_tensor(bc, **f64)
        self.Ks_elem = torch.as_tensor(ks, **f64) if has_ks else None
        self.h_n = torch.empty(N, **f64)
        wd = int(lib.wspm_ensemble_workspace_doubles(N, self.dm.nnz_padded))
        self.work = torch.empty(wd, **f64)
        self.dt = torch.full((D,), float(dt0), **f64)
        self.t = torch.zeros(D, **f64)
        self.its, self.kits, self.status = (torch.zeros(D, **i32) for _ in range(3))
        self.err = torch.zeros(D, **f64)
        self.queue = torch.zeros(1, **i32)
        tp = dict(m_it=5, M_it=7, lambda_amp=2.0, lambda_red=0.5)
        tp.update(time_params or {})
        Q, W = default_rule(2) if quad is None else quad
        Q, W = np.ascontiguousarray(Q, dtype=np.float64).ravel(), np.ascontiguousarray(W, dtype=np.float64)
        e = _lib.WspmEnsemble()
        e.n_domains = D
        e.node_off, e.order, e.phi = self.node_off.data_ptr(), self.order.data_ptr(), self.phi.data_ptr()
        e.Ks_elem = self.Ks_elem.data_ptr() if self.Ks_elem is not None else None
        e.bc_val = self.bc_val.data_ptr()
        for j, v in enumerate(Q):
            e.quad_points[j] = v
        for j, v in enumerate(W):
            e.weights[j] = v
        e.nq = len(W)
        e.krylov_tol, e.krylov_maxiter = float(krylov_tol), int(krylov_maxiter)
        e.picard_tol, e.picard_maxiter, e.picard_relative = float(picard_tol), int(picard_maxiter), int(picard_relative)
        e.tmax = float(tmax)
        e.m_it, e.M_it = int(tp["m_it"]), int(tp["M_it"])
        e.lambda_amp, e.lambda_red = float(tp["lambda_amp"]), float(tp["lambda_red"])
        e.h_n, e.work, e.work_doubles = self.h_n.data_ptr(), self.work.data_ptr(), self.work.numel()
        e.dt, e.t = self.dt.data_ptr(), self.t.data_ptr()
        e.its, e.kits, e.status, e.err = (x.data_ptr() for x in (self.its, self.kits, self.status, self.err))
        e.queue = self.queue.data_ptr()
        self.c = e
        self.tmax = float(tmax)
        self.block_threads = 512
        self.cluster_size = 1

    def set_state(self, h0):
        """Initial head: one array over all nodes, or a scalar."""
        if np.isscalar(h0):
            self.h_n.fill_(float(h0))
        else:
            self.h_n.copy_(torch.as_tensor(np.asarray(h0, dtype=np.float64)).to(self.h_n.device))

    def domain(self, d, x=None):
        x = self.h_n if x is None else x
        return x[int(self.node_off_host[d]):int(self.node_off_host[d + 1])]

    def launch(self, stream=None):
        st = stream if stream is not None else torch.cuda.current_stream()
        self.c.cluster_size = int(self.cluster_size)
        check("ensemble_step", lib.wspm_ensemble_step(ctypes.byref(self.dm.c_mesh), ctypes.byref(self.dm.c_pat),
                                                       ctypes.byref(self.c), int(self.block_threads),
                                                       ctypes.c_void_p(st.cuda_stream)))

    def run_device(self, max_steps, stream=None):
        """Up to ``max_steps`` steps of every active domain in one CUDA graph (``wspm_ensemble_run``: the time
        loop runs on the device, no host round trip between steps).  Returns device tensors (Picard iterations
        summed per domain, int32[2] = steps launched, domains still active); nothing is synchronised."""
        st = stream if stream is not None else torch.cuda.current_stream()
        dev = self.h_n.device
        if not hasattr(self, "_run_bufs"):
            self._run_bufs = (torch.zeros(self.n_domains, dtype=torch.int32, device=dev),
                              torch.zeros(self.n_domains, dtype=torch.int64, device=dev),
                              torch.zeros(2, dtype=torch.int32, device=dev))
        act, its, run = self._run_bufs
        self.c.cluster_size = int(self.cluster_size)
        check("ensemble_run", lib.wspm_ensemble_run(ctypes.byref(self.dm.c_mesh), ctypes.byref(self.dm.c_pat),
                                                     ctypes.byref(self.c), int(self.block_threads), int(max_steps),
                                                     dptr(act), dptr(its), dptr(run), ctypes.c_void_p(st.cuda_stream)))
        return its, run

    def active(self):
        return int((self.t < self.tmax).sum().item())

    def step(self):
        """One implicit step of every active domain; returns per-domain (its, krylov its, status, err) on the host."""
        active = (self.t < self.tmax).cpu().numpy()
        self.launch()
        return {"active": active, "iterations": self.its.cpu().numpy(), "krylov_iterations": self.kits.cpu().numpy(),
                "status": self.status.cpu().numpy(), "error": self.err.cpu().numpy()}

    def autotune(self, shapes=LAUNCH_SHAPES):
        """Pick the (CTA size, cluster size) with the fastest step on a copy of the current state (state
        restored); returns the CTA size and sets ``block_threads`` and ``cluster_size``."""
        saved = [x.clone() for x in (self.h_n, self.dt, self.t, self.its, self.kits, self.status, self.err)]
        timing = {}
        for tb, cs in shapes:
            for x, s in zip((self.h_n, self.dt, self.t, self.its, self.kits, self.status, self.err), saved):
                x.copy_(s)
            self.block_threads, self.cluster_size = tb, cs
            try:
                self.launch()                   # warm
            except _lib.WspmError:
                continue                        # shape not available on this GPU (e.g. 16-CTA clusters)
            for x, s in zip((self.h_n, self.dt, self.t, self.its, self.kits, self.status, self.err), saved):
                x.copy_(s)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.launch()
            e1.record()
            torch.cuda.synchronize()
            timing[(tb, cs)] = e0.elapsed_time(e1)
        for x, s in zip((self.h_n, self.dt, self.t, self.its, self.kits, self.status, self.err), saved):
            x.copy_(s)
        self.block_threads, self.cluster_size = min(timing, key=timing.get)
        self.timing = {f"{tb}x{cs}": t for (tb, cs), t in timing.items()}
        return self.block_threads

    def run(self, max_steps=None):
        """Steps until every domain reached tmax (or max_steps launches); per-launch host records."""
        out = {"iterations": [], "krylov_iterations": [], "active": [], "status": []}
        t0 = time.perf_counter()
        n = 0
        while self.active() and (max_steps is None or n < max_steps):
            r = self.step()
            for k in out:
                out[k].append(r[k])
            n += 1
        out = {k: np.array(v) for k, v in out.items()}
        out["wall_time"] = time.perf_counter() - t0
        return out
