"""One Richards domain split into row strips (CPU): the partition's invariants, the exchange plans, and the split
Picard step -- all ranks in one process and as two gloo ranks -- against the oracle's single-domain step.

The ranks' local work here is a NumPy/SciPy back end over the oracle's soil law and assembly on each rank's
extended mesh (owned rows only); the device back end is checked against the same oracle in test_gpu_halo.py.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import assembly as oasm, krylov as okry, picard as opic, soil as osoil  # noqa: E402
from wspm_b200 import mesh  # noqa: E402
from wspm_b200.halo import (EmulatedComm, ProcessGroupComm, StripPartition,  # noqa: E402
                            distributed_picard_step)


class HostBackend:
    """Oracle soil law and assembly on one rank's extended mesh; rows of the owned nodes."""

    def __init__(self, points_ext, elements_ext, n_owned, phi, bc_val_ext):
        self.pts, self.el, self.n_owned = points_ext, elements_ext, n_owned
        self.phi, self.bc = phi, bc_val_ext
        self.A = None

    def theta(self, h_ext):
        return torch.as_tensor(osoil.van_genuchten_model(h_ext.numpy(), self.phi)[2])

    def assemble(self, h_ext, theta_n, dt):
        h = h_ext.numpy()
        C, K, th = osoil.van_genuchten_model(h, self.phi)
        A, b = oasm.assemble_richards(self.el, len(self.pts), self.pts, th, theta_n.numpy(), h, K, C, dt)
        nodes = np.where(~np.isnan(self.bc))[0]
        A, b = oasm.apply_dirichlet_rows(A, b, nodes, self.bc[nodes])
        m = self.n_owned
        self.A = A.tocsr()[:m]
        return torch.as_tensor(b[:m]), torch.as_tensor(okry.jacobi_inverse_diagonal(self.A[:, :m]))

    def spmv(self, x_ext):
        return torch.as_tensor(self.A @ x_ext.numpy())


def _problem(n=20):
    pts, tri = mesh.structured_triangles(n, 1.0)
    top = np.where(pts[:, 1] == 1.0)[0]
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, h_top=-0.1, h0=-1.0, maxiter=1000)
    bc = np.full(len(pts), np.nan)
    bc[prob.bc_nodes] = prob.bc_vals
    return pts, tri, prob, h0, bc


def _csr(tri, n):
    import scipy.sparse as sp
    r = np.repeat(tri, tri.shape[1], axis=1).ravel()
    c = np.tile(tri, (1, tri.shape[1])).ravel()
    A = sp.csr_matrix((np.ones(r.size), (r, c)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A.indptr, A.indices


def _backends(part, pts, tri, phi, bc, ranks):
    out = []
    for r in ranks:
        p, e = part.local_mesh(r, pts, tri)
        out.append(HostBackend(p, e, part.n_owned(r), phi, bc[part.ext[r]]))
    return out


@pytest.mark.parametrize("world", [1, 2, 3, 7])
def test_partition_invariants_and_exchange_plans(world):
    pts, tri = mesh.structured_triangles(12, 1.0)
    n = len(pts)
    indptr, indices = _csr(tri, n)
    part = StripPartition(indptr, indices, tri, world)
    owned = np.concatenate([np.arange(*part.rows[r]) for r in range(world)])
    assert np.array_equal(owned, np.arange(n))
    nnz = np.array([indptr[r1] - indptr[r0] for r0, r1 in part.rows])
    assert nnz.max() - nnz.min() <= 2 * np.diff(indptr).max()
    for r in range(world):
        r0, r1 = part.rows[r]
        ext = part.ext[r]
        assert np.array_equal(ext[:r1 - r0], np.arange(r0, r1))
        assert set(indices[indptr[r0]:indptr[r1]]) == set(ext)        # exactly the columns of the owned rows
        p, e = part.local_mesh(r, pts, tri)
        assert np.array_equal(ext[e], tri[part.elems[r]])
        # every element with an owned vertex is kept, and in ascending order
        keep = np.any((tri >= r0) & (tri < r1), axis=1)
        assert np.array_equal(part.elems[r], np.where(keep)[0])
        sends, recvs = part.exchange_plan(r)
        for p_, dst in recvs.items():
            src = part.exchange_plan(p_)[0][r]
            assert np.array_equal(part.ext[p_][src], ext[dst])         # same global ids, same order
            assert np.all(part.owner[ext[dst]] == p_)
        for p_, src in sends.items():
            assert np.all(src < r1 - r0)


def test_partition_rejects_more_ranks_than_rows():
    pts, tri = mesh.structured_triangles(2, 1.0)
    indptr, indices = _csr(tri, len(pts))
    with pytest.raises(ValueError):
        StripPartition(indptr, indices, tri, len(pts) + 1)


def test_emulated_exchange_fills_every_ghost():
    pts, tri = mesh.structured_triangles(10, 1.0)
    indptr, indices = _csr(tri, len(pts))
    part = StripPartition(indptr, indices, tri, 3)
    comm = EmulatedComm(part, "cpu")
    g = torch.arange(len(pts), dtype=torch.float64) * 1.5
    xs = [g[torch.as_tensor(part.ext[r])].clone() for r in range(3)]
    for r in range(3):
        xs[r][part.n_owned(r):] = -7.0
    comm.exchange(xs)
    for r in range(3):
        assert torch.equal(xs[r], g[torch.as_tensor(part.ext[r])])


@pytest.mark.parametrize("world", [1, 2, 3])
def test_split_picard_step_matches_single_domain_oracle(world):
    pts, tri, prob, h0, bc = _problem()
    dt = 1e-3
    theta_n = prob.model(h0)[2]
    h_ref, err_ref, it_ref = prob.timestep(h0, theta_n, dt)
    indptr, indices = _csr(tri, len(pts))
    part = StripPartition(indptr, indices, tri, world)
    bes = _backends(part, pts, tri, prob.phi, bc, range(world))
    comm = EmulatedComm(part, "cpu")
    hs = [torch.as_tensor(h0[part.ext[r]]) for r in range(world)]
    hs, it, err, kits = distributed_picard_step(bes, comm, hs, dt, krylov_maxiter=1000)
    h = part.gather([hs[r][:part.n_owned(r)].numpy() for r in range(world)])
    assert it == it_ref
    assert kits > 0
    np.testing.assert_allclose(h, h_ref, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(err, err_ref, rtol=1e-4)
    # ghosts hold the owners' values after the step
    for r in range(world):
        np.testing.assert_array_equal(hs[r].numpy(), h[part.ext[r]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pts, tri, prob, h0, bc = _problem()
        indptr, indices = _csr(tri, len(pts))
        part = StripPartition(indptr, indices, tri, world)
        be = _backends(part, pts, tri, prob.phi, bc, [rank])
        comm = ProcessGroupComm(part, rank, "cpu")
        hs, it, err, kits = distributed_picard_step(be, comm, [torch.as_tensor(h0[part.ext[rank]])], 1e-3,
                                                    krylov_maxiter=1000)
        mine = hs[0][:part.n_owned(rank)].contiguous()
        sizes = [part.n_owned(r) for r in range(world)]
        pad = max(sizes)
        buf = [torch.empty(pad, dtype=torch.float64) for _ in sizes]
        dist.all_gather(buf, torch.nn.functional.pad(mine, (0, pad - mine.numel())))
        parts = [b[:s] for b, s in zip(buf, sizes)]
        if rank == 0:
            np.savez(out_path, h=torch.cat(parts).numpy(), it=it, err=err, kits=kits)
    finally:
        dist.destroy_process_group()


def test_split_picard_step_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "split.npz")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    got = np.load(out)
    pts, tri, prob, h0, bc = _problem()
    h_ref, err_ref, it_ref = prob.timestep(h0, prob.model(h0)[2], 1e-3)
    assert int(got["it"]) == it_ref
    np.testing.assert_allclose(got["h"], h_ref, rtol=1e-9, atol=1e-11)
