"""One Richards domain split over ranks: row strips with one ghost layer.

The reference has no multi-device path; its Picard step (src/solvers/richards_solver_v2.py:107-168) and Krylov
solve (src/solvers/jax_linear_solver.py:262-283) run on one device.  Here the rows are cut into contiguous strips
(balanced by nonzeros, ``StripPartition``); a rank owns its rows and keeps, as ghosts, the other columns of those
rows.  Every owned row is assembled completely on its owner (the elements incident to owned rows, with ghost nodes
as extra vertices: owner-computes, no communication in the assembly), so a step needs:

* per Krylov iteration one halo exchange (owners send the ghost values of the preconditioned residual to the ranks
  that read them; point-to-point, before the SpMV) and one allreduce of three sums: the CG is the single-reduction
  form (Chronopoulos & Gear), whose (w, z), (r, z), (r, r) give both alpha and beta -- the same iteration as the
  single-GPU resident kernel;
* per Picard iteration one halo exchange of the new head (the ghosts' soil values for the next assembly) and one
  allreduce of the Picard norm's two sums.

The ranks' local compute sits behind a back end: ``DeviceBackend`` runs libwspm's soil, assembly and SpMV kernels
on the rank's extended mesh (owned nodes first, then ghosts) on its GPU; any object with the same four members
(``n_owned``, ``theta``, ``assemble``, ``spmv``) works.  Communication sits behind ``ProcessGroupComm`` (one rank
per process, ``torch.distributed``: NCCL between GPUs, gloo between CPU processes) or ``EmulatedComm`` (every rank
in this process, the exchange as copies between the ranks' vectors and the reductions as sums -- host-driven, so
no launch waits on another).
"""
import numpy as np
import torch


class StripPartition:
    """Contiguous row ranges per rank (balanced by nonzeros) of a CSR pattern, with each rank's ghost columns.

    ``indptr``/``indices``: the global pattern; ``elements`` (E, nv): the mesh.  For rank r: ``rows[r]`` = (r0, r1);
    ``ext[r]`` = global ids of its extended nodes (owned ascending, then ghosts ascending); ``elems[r]`` = the
    elements incident to its owned rows (ascending ids, so every owned row sums its element contributions in the
    order the single-domain assembly does)."""

    def __init__(self, indptr, indices, elements, world):
        indptr = np.asarray(indptr, dtype=np.int64)
        indices = np.asarray(indices, dtype=np.int64)
        elements = np.asarray(elements, dtype=np.int64)
        n = indptr.size - 1
        world = int(world)
        if world < 1 or world > n:
            raise ValueError(f"cannot cut {n} rows into {world} strips")
        self.n, self.world = n, world
        target = np.arange(1, world) * (indptr[-1] / world)
        cuts = np.searchsorted(indptr[1:], target, side="left") + 1
        bounds = np.zeros(world + 1, dtype=np.int64)
        bounds[world] = n
        for k in range(1, world):   # every strip keeps at least one row
            bounds[k] = min(max(int(cuts[k - 1]), bounds[k - 1] + 1), n - (world - k))
        self.rows = [(int(bounds[r]), int(bounds[r + 1])) for r in range(world)]
        self.owner = np.repeat(np.arange(world), np.diff(bounds))
        self.ext, self.elems = [], []
        elem_owner = self.owner[elements]
        for r, (r0, r1) in enumerate(self.rows):
            cols = indices[indptr[r0]:indptr[r1]]
            ghosts = np.unique(cols[(cols < r0) | (cols >= r1)])
            self.ext.append(np.concatenate([np.arange(r0, r1, dtype=np.int64), ghosts]))
            self.elems.append(np.where(np.any(elem_owner == r, axis=1))[0])

    def n_owned(self, r):
        return self.rows[r][1] - self.rows[r][0]

    def local_mesh(self, r, points, elements):
        """(points, elements renumbered to rank r's extended nodes)."""
        ext = self.ext[r]
        glob_to_loc = -np.ones(self.n, dtype=np.int64)
        glob_to_loc[ext] = np.arange(ext.size)
        loc = glob_to_loc[np.asarray(elements, dtype=np.int64)[self.elems[r]]]
        if np.any(loc < 0):
            raise ValueError("an element of an owned row has a vertex outside the rank's extended nodes")
        return np.asarray(points)[ext], loc

    def scatter(self, r, v):
        """Rank r's extended slice of a global nodal vector (NumPy or torch)."""
        return v[self.ext[r]] if isinstance(v, np.ndarray) else v[torch.as_tensor(self.ext[r], device=v.device)]

    def gather(self, owned):
        """Global vector from the ranks' owned parts (a list in rank order)."""
        if isinstance(owned[0], np.ndarray):
            return np.concatenate(owned)
        return torch.cat(list(owned))

    def exchange_plan(self, r):
        """({peer: local positions of the owned values r sends to peer}, {peer: local ghost positions r fills from
        peer}), both in ascending global id, so sender and receiver agree on the order."""
        r0, r1 = self.rows[r]
        ghosts = self.ext[r][r1 - r0:]
        sends, recvs = {}, {}
        for p in range(self.world):
            if p == r:
                continue
            mine = np.where(self.owner[ghosts] == p)[0]
            if mine.size:
                recvs[p] = (r1 - r0) + mine
            theirs = self.ext[p][self.n_owned(p):]
            need = theirs[self.owner[theirs] == r]
            if need.size:
                sends[p] = need - r0
        return sends, recvs


class ProcessGroupComm:
    """This process is one rank: ghost updates by isend / irecv and sums by all_reduce over the default process
    group (NCCL between GPUs, gloo on CPUs)."""

    def __init__(self, part, rank, device):
        self.ranks = [rank]
        sends, recvs = part.exchange_plan(rank)
        self.send_idx = {p: torch.as_tensor(v, device=device) for p, v in sends.items()}
        self.recv_idx = {p: torch.as_tensor(v, device=device) for p, v in recvs.items()}

    def exchange(self, xs):
        import torch.distributed as dist
        x = xs[0]
        reqs, bufs = [], {}
        for p, idx in self.recv_idx.items():
            bufs[p] = torch.empty(idx.numel(), dtype=x.dtype, device=x.device)
            reqs.append(dist.irecv(bufs[p], src=p))
        for p, idx in self.send_idx.items():
            reqs.append(dist.isend(x[idx].contiguous(), dst=p))
        for q in reqs:
            q.wait()
        for p, idx in self.recv_idx.items():
            x[idx] = bufs[p]

    def allreduce(self, parts):
        import torch.distributed as dist
        t = parts[0].clone()
        if dist.is_initialized() and dist.get_world_size() > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t


class EmulatedComm:
    """Every rank in this process: the exchange copies owners' values into the readers' ghost slots and the
    reductions sum the ranks' partial sums in rank order."""

    def __init__(self, part, device):
        self.ranks = list(range(part.world))
        self.moves = []   # (dst rank, dst positions, src rank, src positions)
        for r in self.ranks:
            for p, dst in part.exchange_plan(r)[1].items():
                src = part.exchange_plan(p)[0][r]
                self.moves.append((r, torch.as_tensor(dst, device=device), p, torch.as_tensor(src, device=device)))

    def exchange(self, xs):
        for r, dst, p, src in self.moves:
            xs[r][dst] = xs[p][src]

    def allreduce(self, parts):
        t = parts[0].clone()
        for q in parts[1:]:
            t += q
        return t


def _sums(comm, pairs_per_rank):
    """Global sums of dot products: pairs_per_rank[i] = [(a, b), ...] for the i-th rank of this process."""
    parts = [torch.stack([torch.dot(a, b) for a, b in pairs]).to(torch.float64) for pairs in pairs_per_rank]
    return [float(v) for v in comm.allreduce(parts).cpu()]


def distributed_cg(backends, comm, bs, xs, dinvs, tol=1e-10, maxiter=1000):
    """Jacobi-CG on the split system, single-reduction form.  Lists hold one entry per rank this process runs
    (``comm.ranks``): ``bs``/``dinvs`` the owned right-hand side and 1/diag, ``xs`` the extended x0 (updated in
    place; ghosts current on return).  Per iteration one exchange of z and one allreduce of (w, z), (r, z), (r, r).
    Stops when r.r <= tol^2 b.b (jax.scipy's rule, jax_linear_solver.py:262-283) or after ``maxiter`` iterations.
    Returns the iteration count."""
    L = range(len(backends))
    ms = [be.n_owned for be in backends]
    comm.exchange(xs)
    rs = [bs[i] - backends[i].spmv(xs[i]) for i in L]
    zs = [torch.zeros_like(xs[i]) for i in L]
    for i in L:
        zs[i][:ms[i]] = dinvs[i] * rs[i]
    comm.exchange(zs)
    ws = [backends[i].spmv(zs[i]) for i in L]
    delta, gamma, rr, bb = _sums(comm, [[(ws[i], zs[i][:ms[i]]), (rs[i], zs[i][:ms[i]]), (rs[i], rs[i]),
                                         (bs[i], bs[i])] for i in L])
    atol2 = tol * tol * bb
    ps = [torch.zeros_like(bs[i]) for i in L]
    ss = [torch.zeros_like(bs[i]) for i in L]
    alpha, gamma_old, k = 0.0, 1.0, 0
    while rr > atol2 and k < maxiter:
        if k == 0:
            beta, alpha = 0.0, gamma / delta
        else:
            beta = gamma / gamma_old
            alpha = gamma / (delta - beta * gamma / alpha)
        for i in L:
            m = ms[i]
            ps[i] = zs[i][:m] + beta * ps[i]
            ss[i] = ws[i] + beta * ss[i]
            xs[i][:m] += alpha * ps[i]
            rs[i] = rs[i] - alpha * ss[i]
            zs[i][:m] = dinvs[i] * rs[i]
        comm.exchange(zs)
        ws = [backends[i].spmv(zs[i]) for i in L]
        gamma_old = gamma
        delta, gamma, rr = _sums(comm, [[(ws[i], zs[i][:ms[i]]), (rs[i], zs[i][:ms[i]]), (rs[i], rs[i])]
                                        for i in L])
        k += 1
    comm.exchange(xs)
    return k


def distributed_picard_step(backends, comm, hs, dt, picard_tol=1e-6, picard_maxiter=100, relative=True,
                            krylov_tol=1e-10, krylov_maxiter=1000):
    """One implicit step (richards_solver_v2.py:107-168) of the split domain: theta_n from h_n, then Picard
    iterations of (soil on the extended nodes, owner-computes assembly, distributed Jacobi-CG from x0 = h_m,
    globally reduced Picard norm).  ``hs``: the ranks' extended heads (ghosts current).  Returns (new heads,
    Picard iterations, Picard error, total Krylov iterations)."""
    L = range(len(backends))
    ms = [be.n_owned for be in backends]
    theta_n = [backends[i].theta(hs[i]) for i in L]
    h_m = [h.clone() for h in hs]
    err, it, kits = float("inf"), 0, 0
    while err >= picard_tol and it < picard_maxiter:
        sys = [backends[i].assemble(h_m[i], theta_n[i], dt) for i in L]
        xs = [h.clone() for h in h_m]
        kits += distributed_cg(backends, comm, [s[0] for s in sys], xs, [s[1] for s in sys], krylov_tol,
                               krylov_maxiter)
        ds = [xs[i][:ms[i]] - h_m[i][:ms[i]] for i in L]
        dd, xx = _sums(comm, [[(ds[i], ds[i]), (xs[i][:ms[i]], xs[i][:ms[i]])] for i in L])
        err = float(np.sqrt(dd) / np.sqrt(xx)) if relative else float(np.sqrt(dd))
        h_m = xs
        it += 1
    return h_m, it, err, kits


class DeviceBackend:
    """libwspm's kernels on one rank's extended mesh on its GPU: van Genuchten soil law, Richards row assembly
    (owned rows complete) with Dirichlet rows fused, Jacobi 1/diag and the SpMV.  ``bc_val_ext``: the Dirichlet
    value per extended node (NaN where free); ``Ks_elem``: per-element saturated conductivity of the rank's
    elements (phi's Ks then 1)."""

    def __init__(self, points_ext, elements_ext, n_owned, phi, bc_val_ext, Ks_elem=None, device="cuda",
                 layout="auto"):
        from .device import DeviceMesh
        from .engine import default_rule
        self.dm = DeviceMesh(points_ext, elements_ext, device=device, layout=layout)
        self.n_owned, self.phi = int(n_owned), tuple(float(v) for v in phi)
        self.bc = torch.as_tensor(np.asarray(bc_val_ext, dtype=np.float64), device=self.dm.device)
        self.Ks = None if Ks_elem is None else torch.as_tensor(np.asarray(Ks_elem, dtype=np.float64),
                                                               device=self.dm.device)
        self.Q, self.W = default_rule(self.dm.dim)
        self.vals = None

    def theta(self, h_ext):
        from .device import soil
        return soil("vg", h_ext, self.phi)[2]

    def assemble(self, h_ext, theta_n, dt):
        from .device import assemble_richards, soil
        C, K, th = soil("vg", h_ext, self.phi)
        vals, rhs, dinv, _ = assemble_richards(self.dm, th, theta_n, h_ext, K, C, self.Q, self.W, dt,
                                               bc_val=self.bc, Ks_elem=self.Ks)
        self.vals = vals
        m = self.n_owned
        return rhs[:m].clone(), dinv[:m].clone()

    def spmv(self, x_ext):
        from .device import spmv
        return spmv(self.dm, self.vals, x_ext)[:self.n_owned]


def split_problem(part, points, elements, phi, bc_val, Ks_elem=None, ranks=None, device="cuda", layout="auto"):
    """A DeviceBackend for each rank in ``ranks`` (default: all) of a global problem (bc_val: NaN where free)."""
    ranks = range(part.world) if ranks is None else ranks
    out = []
    for r in ranks:
        pts, el = part.local_mesh(r, points, elements)
        ks = None if Ks_elem is None else np.asarray(Ks_elem)[part.elems[r]]
        out.append(DeviceBackend(pts, el, part.n_owned(r), phi, np.asarray(bc_val)[part.ext[r]], ks,
                                 device=device, layout=layout))
    return out
