"""The oracle against the reference's own golden artefacts (CPU).

Pins oracle/ to resultsRE2D CSV rows (Picard totals + six analytical-error
metrics, 5 significant digits) and to the Test3D npz fields (1e-12).
"""
import json
import os

import numpy as np
import pytest

from oracle import analytic, picard
from wspm_b200 import mesh

GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROWS = json.load(open(os.path.join(GOLD, "re2d_metrics.json")))

# Unpreconditioned BiCGSTAB at mesh 50 hits its 100-iteration cap in one Picard
# iteration of the reference run: Krylov-internal behaviour, not pinned.
UNPINNED = {("Test1", 50, "bicgstab", "none")}


def golden_rows(meshes, solvers=("cg", "bicgstab", "gmres", "direct"), preconds=("none", "jacobi", "ilu")):
    seen, out = set(), []
    for r in ROWS:
        key = (r["test_case"], r["mesh"], r["solver"], r["precond"])
        if r["mesh"] in meshes and r["solver"] in solvers and r["precond"] in preconds and key not in seen:
            seen.add(key)
            out.append(r)
    return out


def run_golden_profile(case, n, solver, precond):
    pts, tri = mesh.structured_triangles(n, 15.24)
    prob, h0 = picard.test_case_2d(pts, tri, case, solver=solver, precond=precond,
                                   picard_tol=1e-4, picard_max=30, picard_relative=False)
    res = picard.run_time_loop(prob, h0, 1e-3, 0.25, theta_at_end=False)
    m = analytic.final_errors(pts, res["pressure_head"][-1], res["theta"][-1], res["times"][-1], int(case[-1]))
    return res, list(m.values())


@pytest.mark.parametrize("row", golden_rows({25}), ids=lambda r: f"{r['test_case']}-{r['mesh']}-{r['solver']}-{r['precond']}")
def test_oracle_reproduces_csv_mesh25(row):
    res, metrics = run_golden_profile(row["test_case"], row["mesh"], row["solver"], row["precond"])
    assert res["iterations"].sum() == row["iterations"]
    np.testing.assert_allclose(metrics, row["metrics"], rtol=5e-4)


@pytest.mark.parametrize("row", golden_rows({50}, solvers=("cg", "gmres"), preconds=("jacobi",)),
                         ids=lambda r: f"{r['test_case']}-{r['mesh']}-{r['solver']}-{r['precond']}")
def test_oracle_reproduces_csv_mesh50(row):
    res, metrics = run_golden_profile(row["test_case"], row["mesh"], row["solver"], row["precond"])
    assert res["iterations"].sum() == row["iterations"]
    np.testing.assert_allclose(metrics, row["metrics"], rtol=5e-4)


def test_unpinned_row_is_documented():
    rows = {(r["test_case"], r["mesh"], r["solver"], r["precond"]) for r in ROWS}
    assert UNPINNED <= rows


@pytest.mark.parametrize("solver", ["bicgstab", "gmres"])
def test_oracle_reproduces_test3d_npz(solver):
    g = np.load(os.path.join(GOLD, f"test3d_{solver}.npz"))
    pts, tets = mesh.kuhn_tetrahedra(20, 15.24)
    prob, h0 = picard.test_case_3d(pts, tets, solver=solver, precond="none")
    res = picard.run_time_loop(prob, h0, 1e-4, 0.1, theta_at_end=False)
    np.testing.assert_array_equal(res["iterations"], g["iterations"])
    np.testing.assert_allclose(res["dt_values"], g["dt_values"], rtol=0, atol=0)
    np.testing.assert_allclose(res["times"], g["times"], rtol=1e-15)
    for k, s in enumerate(g["steps"]):
        np.testing.assert_allclose(res["pressure_head"][s], g["pressure_head"][k], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(res["theta"][s], g["theta"][k], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(res["errors"], g["errors"], rtol=1e-6)


def test_oracle_pipelined_cg_converges_like_cg():
    """The oracle's restatement of the device's pipelined inner CG: same solution as CG to the tolerance, the
    iteration count within a few of CG's (the pipelined recurrences drift by rounding only)."""
    from scipy.sparse import diags
    from oracle import krylov
    n = 400
    rng = np.random.default_rng(3)
    main = 2.0 + rng.uniform(0.0, 1.0, n)
    A = diags([-np.ones(n - 1), main, -np.ones(n - 1)], [-1, 0, 1], format="csr")
    b = rng.standard_normal(n)
    d = krylov.jacobi_inverse_diagonal(A)
    x1, k1 = krylov.cg(A, b, np.zeros(n), tol=1e-10, maxiter=1000, dinv=d)
    x2, k2 = krylov.pipelined_cg(A, b, np.zeros(n), tol=1e-10, maxiter=1000, dinv=d)
    assert abs(k1 - k2) <= 2
    assert np.linalg.norm(b - A @ x2) <= 2e-10 * np.linalg.norm(b)
    np.testing.assert_allclose(x2, x1, rtol=1e-8, atol=1e-8)
    # a cap stops the run with exactly maxiter updates
    _, k3 = krylov.pipelined_cg(A, b, np.zeros(n), tol=0.0, maxiter=7, dinv=d)
    assert k3 == 7


def test_oracle_true_ilu0_reproduces_a_on_its_pattern():
    """The defining property of ILU(0): (L U)_ij = A_ij on every position of A's pattern (here a 2D P1 Richards
    matrix with Dirichlet rows), and the factorization is exact for a tridiagonal matrix."""
    import scipy.sparse as sp
    from oracle import assembly as oasm, krylov as okry, soil as osoil
    from wspm_b200 import mesh
    pts, tri = mesh.structured_triangles(12, 1.0)
    h = -np.linspace(0.1, 2.0, len(pts))
    C, K, th = osoil.van_genuchten_model(h, (3.35, 0.368, 0.102, 2.0, 0.5, 0.0922))
    A, b = oasm.assemble_richards(tri, len(pts), pts, th, th - 1e-3, h, K, C, 1e-3)
    top = np.where(pts[:, 1] == 1.0)[0]
    A, b = oasm.apply_dirichlet_rows(A, b, top, -0.1 * np.ones(top.size))
    LU = okry.true_ilu0(A)
    L = sp.tril(LU, -1) + sp.eye(A.shape[0])
    U = sp.triu(LU)
    prod = (L @ U).tocsr()
    Ac = A.tocoo()
    np.testing.assert_allclose(np.asarray(prod[Ac.row, Ac.col]).ravel(), Ac.data, rtol=1e-12,
                               atol=1e-12 * np.abs(Ac.data).max())
    n = 25
    T = sp.diags([-np.ones(n - 1), 3 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    x = np.random.default_rng(1).standard_normal(n)
    np.testing.assert_allclose(T @ okry.true_ilu0_apply(okry.true_ilu0(T), x), x, atol=1e-12)
