"""The row-strip split of one Richards domain with libwspm's kernels as each rank's local back end (one GPU, all
ranks in one process, host-driven exchange): owned rows assemble exactly as the single-domain assembly does, and
the split Picard step reproduces the oracle's single-domain step."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import picard as opic  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu


def _problem(n=24):
    pts, tri = mesh.structured_triangles(n, 1.0)
    top = np.where(pts[:, 1] == 1.0)[0]
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, h_top=-0.1, h0=-1.0, maxiter=1000)
    bc = np.full(len(pts), np.nan)
    bc[prob.bc_nodes] = prob.bc_vals
    return pts, tri, prob, h0, bc


def _part(pts, tri, world):
    from wspm_b200.halo import StripPartition
    from wspm_b200.pattern import Pattern
    P = Pattern(tri, len(pts))
    return StripPartition(P.csr_indptr, P.csr_indices, tri, world)


@pytest.mark.parametrize("world", [2, 3])
def test_owned_rows_assemble_as_the_single_domain(world):
    from wspm_b200.device import DeviceMesh, assemble_richards, soil
    from wspm_b200.engine import default_rule
    from wspm_b200.halo import split_problem
    pts, tri, prob, h0, bc = _problem()
    rng = np.random.default_rng(1)
    h = h0 + rng.uniform(-0.5, 0.5, h0.size)
    th_n = prob.model(h)[2] - 1e-3
    dm = DeviceMesh(pts, tri)
    cu = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")
    C, K, th = soil("vg", cu(h), prob.phi)
    Q, W = default_rule(2)
    vals, rhs, dinv, _ = assemble_richards(dm, th, cu(th_n), cu(h), K, C, Q, W, 1e-3, bc_val=cu(bc))
    vals_h, rhs_h, dinv_h = vals.cpu().numpy(), rhs.cpu().numpy(), dinv.cpu().numpy()
    P = dm.pattern
    part = _part(pts, tri, world)
    for r, be in enumerate(split_problem(part, pts, tri, prob.phi, bc)):
        r0, r1 = part.rows[r]
        ext = part.ext[r]
        b_loc, d_loc = be.assemble(cu(h[ext]), cu(th_n[ext]), 1e-3)
        np.testing.assert_array_equal(b_loc.cpu().numpy(), rhs_h[r0:r1])
        np.testing.assert_array_equal(d_loc.cpu().numpy(), dinv_h[r0:r1])
        Pl = be.dm.pattern
        lv = be.vals.cpu().numpy()
        for i in range(r1 - r0):
            cols = Pl.csr_indices[Pl.csr_indptr[i]:Pl.csr_indptr[i + 1]].astype(np.int64)
            rows = np.full(cols.size, i, dtype=np.int64)
            got = lv[Pl.entry_pos(rows, Pl.slot(rows, cols))]
            g_rows = rows + r0
            g_cols = ext[cols]
            want = vals_h[P.entry_pos(g_rows, P.slot(g_rows, g_cols))]
            np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("world", [1, 2, 4])
def test_split_picard_step_on_the_device_matches_oracle(world):
    from wspm_b200.halo import EmulatedComm, distributed_picard_step, split_problem
    pts, tri, prob, h0, bc = _problem()
    dt = 1e-3
    h_ref, err_ref, it_ref = prob.timestep(h0, prob.model(h0)[2], dt)
    part = _part(pts, tri, world)
    bes = split_problem(part, pts, tri, prob.phi, bc)
    comm = EmulatedComm(part, "cuda")
    hs = [torch.as_tensor(h0[part.ext[r]], device="cuda") for r in range(world)]
    hs, it, err, kits = distributed_picard_step(bes, comm, hs, dt, krylov_maxiter=1000)
    h = part.gather([hs[r][:part.n_owned(r)] for r in range(world)]).cpu().numpy()
    assert it == it_ref
    np.testing.assert_allclose(h, h_ref, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(err, err_ref, rtol=1e-4)
