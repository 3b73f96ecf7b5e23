"""The reference's ilu / ssor / block_jacobi preconditioners on the device against the oracle.

The oracle restates what the reference's code computes (jax_linear_solver.py:38-252) and is pinned to the
published ilu rows; here the device sweeps must apply the same operator (1e-12 relative) and the
host-driven Krylov loops must take the same iterations to the same solution.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import analytic, assembly as oasm, krylov as okry, soil as osoil  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
VG = (3.35, 0.368, 0.102, 2.0, 0.5, 0.0922)


def cu(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")


def _system(layout, n=20, seed=0):
    from wspm_b200.device import DeviceMesh, apply_dirichlet
    pts, tri = mesh.structured_triangles(n, 1.0)
    rng = np.random.default_rng(seed)
    h = -rng.uniform(0.05, 2.0, len(pts))
    C, K, th = osoil.van_genuchten_model(h, VG)
    A, b = oasm.assemble_richards(tri, len(pts), pts, th, th - 0.001, h, K, C, 1e-3)
    top = np.where(pts[:, 1] == 1.0)[0]
    A, b = oasm.apply_dirichlet_rows(A, b, top, -0.1 * np.ones(top.size))
    dm = DeviceMesh(pts, tri, layout=layout)
    A = A.tocoo()
    P = dm.pattern
    host = np.zeros(P.nnz_padded)
    rows = A.row.astype(np.int64)
    host[P.entry_pos(rows, P.slot(rows, A.col.astype(np.int64)))] = A.data   # every entry of A is a pattern slot
    return dm, A.tocsr(), b, h, cu(host)


@pytest.mark.parametrize("layout", ["dia", "sell"])
@pytest.mark.parametrize("kind", ["ilu", "ssor", "block_jacobi"])
def test_preconditioner_matches_oracle(kind, layout):
    from wspm_b200.precond import ReferencePreconditioner
    dm, A, b, h, vals = _system(layout)
    v = np.random.default_rng(3).standard_normal(A.shape[0])
    want = okry.reference_preconditioner(A, kind, omega=1.0, block_size=2)(v)
    got = ReferencePreconditioner(dm, vals, kind)(cu(v)).cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("solver", ["cg", "bicgstab", "gmres"])
@pytest.mark.parametrize("kind", ["ilu", "ssor", "block_jacobi"])
def test_preconditioned_solves_match_oracle(solver, kind):
    from wspm_b200 import precond
    dm, A, b, h, vals = _system("auto")
    x_ref, k_ref = okry.solve_system(A, b, h, solver, kind, tol=1e-10, maxiter=200, restart=30)
    x, k = precond.solve(dm, vals, cu(b), cu(h), solver, kind, tol=1e-10, maxiter=200, restart=30)
    assert k == k_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-8, atol=1e-10)


def test_richards_solver_with_ilu_reproduces_published_row():
    """Test1, mesh 25, cg + ilu through the drop-in RichardsSolver (published Picard profile)."""
    import json
    from config.settings import SimulationConfig, SolverParameters, TimeSteppingParameters
    from src.solvers.richards_solver_v2 import RichardsSolver
    row = next(r for r in json.load(open(os.path.join(GOLD, "re2d_metrics.json")))
               if r["test_case"] == "Test1" and r["mesh"] == 25 and r["solver"] == "cg" and r["precond"] == "ilu")
    cfg = SimulationConfig(time=TimeSteppingParameters(dt_init=1e-3, Tmax=0.25),
                           solver=SolverParameters(solver_type="cg", precond_type="ilu"), test_case="Test1")
    cfg.mesh.mesh_size = "25"
    cfg.mesh.mesh_dir = None
    res = RichardsSolver(cfg, picard_profile="published").solve()
    pts = res["points"]
    m = analytic.final_errors(pts, res["pressure_head"][-1], res["theta"][-1], res["times"][-1], 1)
    assert int(np.sum(res["iterations"])) == row["iterations"]
    np.testing.assert_allclose(list(m.values()), row["metrics"], rtol=5e-4)


@pytest.mark.parametrize("layout", ["dia", "sell"])
def test_true_ilu0_factors_and_apply_match_oracle(layout):
    """wspm_ilu0_factor (true ILU(0), level-scheduled on the device) gives the oracle's factors, and the sweeps apply
    (LU)^-1 as the oracle does."""
    from wspm_b200 import _lib
    from wspm_b200.precond import ReferencePreconditioner
    dm, A, b, h, vals = _system(layout)
    LU = okry.true_ilu0(A).tocoo()
    P = dm.pattern
    want = np.zeros(P.nnz_padded)
    rows = LU.row.astype(np.int64)
    want[P.entry_pos(rows, P.slot(rows, LU.col.astype(np.int64)))] = LU.data
    pre = ReferencePreconditioner(dm, vals, "ilu0")
    got = pre.vals.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
    v = np.random.default_rng(5).standard_normal(A.shape[0])
    wv = okry.true_ilu0_apply(okry.true_ilu0(A), v)
    gv = pre(cu(v)).cpu().numpy()
    np.testing.assert_allclose(gv, wv, rtol=1e-12, atol=1e-12 * np.abs(wv).max())
    assert _lib.PRECOND_KIND["ilu0"] == 5


@pytest.mark.parametrize("solver", ["bicgstab", "gmres"])
def test_true_ilu0_preconditioned_solves(solver):
    """BiCGSTAB / GMRES with the true ILU(0) converge to the direct solution in fewer iterations than with Jacobi."""
    import scipy.sparse.linalg as spla
    from wspm_b200 import precond
    dm, A, b, h, vals = _system("auto", n=32)
    exact = spla.spsolve(A.tocsc(), b)
    x, k = precond.solve(dm, vals, cu(b), cu(h), solver, "ilu0", tol=1e-10, maxiter=400, restart=30)
    _, kj = precond.solve(dm, vals, cu(b), cu(h), solver, "jacobi", tol=1e-10, maxiter=400, restart=30)
    np.testing.assert_allclose(x.cpu().numpy(), exact, rtol=1e-7, atol=1e-8)
    if solver == "bicgstab":
        assert 0 < k < kj
    else:
        # GMRES counts restart cycles (one each here); compare the residual after one short cycle instead
        assert 0 < k <= kj
        res = []
        for kind in ("ilu0", "jacobi"):
            y, _ = precond.solve(dm, vals, cu(b), cu(h), solver, kind, tol=1e-14, maxiter=1, restart=6)
            res.append(np.linalg.norm(b - A @ y.cpu().numpy()))
        assert res[0] < res[1]
