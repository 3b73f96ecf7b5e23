"""Parity of the CUDA path (libwspm.so through the C ABI) with the oracle.

Tolerances: element/assembly values and SpMV are compared to 1e-13 relative
(to the largest entry); Krylov solutions, which differ from the oracle's only
by summation order, to a few times the solver tolerance; whole Picard runs
against the reference's own goldens (CSV metrics 5e-4 relative, Picard
iteration totals exactly; Test3D npz fields 1e-8 relative).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import analytic, assembly as oasm, krylov as okry, picard as opic, soil as osoil  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def dev():
    from wspm_b200 import device
    return device


def cu(a, dtype=torch.float64):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy()


VG = (3.35, 0.368, 0.102, 2.0, 0.5, 0.0922)
EXP = (0.164, 0.45, 0.15, 0.1)


@pytest.mark.parametrize("model,phi", [("vg", VG), ("exp", EXP), ("vg", (3.6, 0.43, 0.078, 1.56, 1 - 1 / 1.56, 0.2496))])
def test_soil_models(model, phi):
    rng = np.random.default_rng(1)
    h = np.concatenate([-10 ** rng.uniform(-4, 1.5, 5000), [0.0, 1e-300, -0.0, 0.5, -1e-300]])
    C, K, th = dev().soil(model, cu(h), phi)
    ref = (osoil.van_genuchten_model if model == "vg" else osoil.exponential_model)(h, phi)
    # theta and C are well conditioned; K = Ks Se^.5 (1-(1-Se^(1/m))^m)^2 cancels at both ends, amplifying
    # the last-ulp differences between two correct pow() implementations
    # (wet end, Se^(1/m) -> 1) and as Se -> 0 (1 - (1 - u)^m ~ m u loses the digits of u)
    amp = np.ones_like(h)
    if model == "vg":
        m = phi[4]
        se = np.clip((ref[2] - phi[2]) / (phi[1] - phi[2]), 0, 1)
        u = se ** (1.0 / m)
        t = 1.0 - (1.0 - u) ** m
        amp = 1.0 + 1.0 / np.maximum(1.0 - u, 1e-300) + 1.0 / np.maximum(t, 1e-300)
    for name, got, want in zip("CKt", (C, K, th), ref):
        rtol = 4e-14 * (amp if name == "K" else 1.0)
        got = host(got)
        bad = np.abs(got - want) > rtol * np.abs(want)
        assert not bad.any(), (name, h[bad][:4], got[bad][:4], want[bad][:4])


def _assembly_case(kind):
    rng = np.random.default_rng(2)
    if kind == "tri-exp":
        pts, el = mesh.structured_triangles(25, 15.24)
        model, phi, Ks = "exp", EXP, None
        h = -15.24 + rng.uniform(0, 10, len(pts))
    elif kind == "tri-vg-ks":
        pts, el = mesh.structured_triangles(40, 1.0)
        model, phi = "vg", VG[:5] + (1.0,)
        Ks = 0.0922 * np.exp(rng.standard_normal(len(el)))
        h = -rng.uniform(0.05, 2.0, len(pts))
    elif kind == "tri-ragged":
        pts, el = mesh.structured_triangles(17, 1.0)
        perm = rng.permutation(len(pts))
        inv = np.argsort(perm)
        pts, el = pts[perm], inv[el][rng.permutation(len(el))]
        model, phi, Ks = "vg", VG, None
        h = -rng.uniform(0.05, 2.0, len(pts))
    else:
        pts, el = mesh.kuhn_tetrahedra(6, 15.24)
        model, phi, Ks = "exp", EXP, None
        h = -15.24 + rng.uniform(0, 10, len(pts))
    return pts, el, model, phi, Ks, h


@pytest.mark.parametrize("kind,layout", [("tri-exp", "dia"), ("tri-exp", "sell"), ("tri-vg-ks", "auto"),
                                         ("tri-ragged", "auto"), ("tet-exp", "dia"), ("tet-exp", "sell")])
def test_assembly_matches_oracle(kind, layout):
    from wspm_b200.engine import default_rule
    pts, el, model, phi, Ks, h = _assembly_case(kind)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout=layout)
    fn = osoil.van_genuchten_model if model == "vg" else osoil.exponential_model
    C, K, th_m = fn(h, phi)
    th_n = fn(h - 0.01, phi)[2]
    dt = 3e-3
    A_ref, b_ref = oasm.assemble_richards(el, len(pts), pts, th_m, th_n, h, K, C, dt, Ks_elem=Ks)
    Q, W = default_rule(pts.shape[1])
    vals, rhs, dinv, vals32 = D.assemble_richards(dm, cu(th_m), cu(th_n), cu(h), cu(K), cu(C), Q, W, dt,
                                                  Ks_elem=None if Ks is None else cu(Ks), want_f32=True)
    A = dm.pattern.to_scipy(host(vals))
    scale = np.abs(A_ref.data).max()
    assert np.abs((A - A_ref).toarray()).max() <= 1e-13 * scale
    np.testing.assert_allclose(host(rhs), b_ref, rtol=0, atol=1e-13 * np.abs(b_ref).max())
    np.testing.assert_allclose(host(dinv), okry.jacobi_inverse_diagonal(A_ref), rtol=1e-13)
    np.testing.assert_allclose(host(vals32), host(vals).astype(np.float32), rtol=0, atol=0)
    # padding slots stay exactly zero
    mask = np.ones(dm.nnz_padded, bool)
    mask[dm.pattern.sell_index] = False
    assert np.all(host(vals)[mask] == 0.0)


@pytest.mark.parametrize("layout", ["dia", "sell"])
def test_assembly_with_dirichlet_rows_and_apply_dirichlet(layout):
    from wspm_b200.engine import default_rule
    pts, el = mesh.structured_triangles(25, 15.24)
    top, bottom = opic.boundary_nodes_2d(pts, "Test1")
    h = -15.24 * np.ones(len(pts))
    C, K, th = osoil.exponential_model(h, EXP)
    hup = opic.upper_bc("Test1", pts[top, 0], EXP[0], np.exp(EXP[0] * h[top]))
    nodes, values = opic.dirichlet_arrays(len(pts), [(top, hup), (bottom, -15.0)])
    A_ref, b_ref = oasm.assemble_richards(el, len(pts), pts, th, th, h, K, C, 1e-3)
    A_ref, b_ref = oasm.apply_dirichlet_rows(A_ref, b_ref, nodes, values)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout=layout)
    bc = D.merge_dirichlet(len(pts), [(top, hup), (bottom, -15.0)])
    Q, W = default_rule(2)
    vals, rhs, dinv, _ = D.assemble_richards(dm, cu(th), cu(th), cu(h), cu(K), cu(C), Q, W, 1e-3, bc_val=cu(bc))
    A = dm.pattern.to_scipy(host(vals))
    assert np.abs((A - A_ref).toarray()).max() <= 1e-13 * np.abs(A_ref.data).max()
    np.testing.assert_allclose(host(rhs), b_ref, rtol=1e-13, atol=1e-13)
    # the stand-alone Dirichlet op on an un-constrained assembly gives the same system
    vals2, rhs2, _, _ = D.assemble_richards(dm, cu(th), cu(th), cu(h), cu(K), cu(C), Q, W, 1e-3)
    D.apply_dirichlet(dm, nodes, values, vals2, rhs2)
    np.testing.assert_array_equal(host(vals2), host(vals))
    np.testing.assert_array_equal(host(rhs2), host(rhs))
    np.testing.assert_allclose(host(D.jacobi_dinv(dm, vals)), host(dinv), rtol=0)


@pytest.mark.parametrize("kind", ["tet", "tri"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("layout", ["dia", "sell"])
def test_spmv(dtype, layout, kind):
    """SpMV against SciPy: DIA (the 16-byte-per-thread kernel: 15 diagonals for tetrahedra, 7 for triangles; the
    triangle mesh has a row count that is not a multiple of the 16-byte group) and SELL."""
    rng = np.random.default_rng(3)
    pts, el = mesh.kuhn_tetrahedra(7) if kind == "tet" else mesh.structured_triangles(30, 1.0)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout=layout)
    data = rng.standard_normal(dm.pattern.nnz)
    x = rng.standard_normal(len(pts))
    vals = cu(dm.pattern.sell_from_csr_values(data), dtype)
    y = host(D.spmv(dm, vals, cu(x, dtype)))
    A = dm.pattern.to_scipy(dm.pattern.sell_from_csr_values(data))
    tol = 1e-13 if dtype == torch.float64 else 2e-5
    np.testing.assert_allclose(y, A @ x, rtol=0, atol=tol * np.abs(A).sum(axis=1).max() * np.abs(x).max())
    if dtype == torch.float64:
        # the matrix object of the shims: CSR fields, @, todense
        M = D.CSRMatrix(dm, vals)
        np.testing.assert_array_equal(M.indptr, A.indptr)
        np.testing.assert_array_equal(M.indices, A.indices)
        np.testing.assert_array_equal(host(M.data), A.data)
        np.testing.assert_allclose(host(M @ cu(x)), y, rtol=0, atol=0)
        np.testing.assert_array_equal(host(M.todense()), A.toarray())


def _linear_system(n=30, dirichlet=True):
    from wspm_b200.engine import default_rule
    pts, el = mesh.structured_triangles(n, 15.24)
    rng = np.random.default_rng(4)
    h = -15.24 + rng.uniform(0, 12, len(pts))
    C, K, th = osoil.exponential_model(h, EXP)
    A, b = oasm.assemble_richards(el, len(pts), pts, th, th - 1e-3, h, K, C, 5e-3)
    if dirichlet:
        top, bottom = opic.boundary_nodes_2d(pts, "Test1")
        nodes, values = opic.dirichlet_arrays(len(pts), [(top, -1.0), (bottom, -15.0)])
        A, b = oasm.apply_dirichlet_rows(A, b, nodes, values)
    return pts, el, A, b, h


@pytest.mark.parametrize("solver,precond,layout", [("cg", "jacobi", "dia"), ("cg", "jacobi", "sell"),
                                                   ("cg", "none", "dia"), ("bicgstab", "none", "sell"),
                                                   ("bicgstab", "jacobi", "dia"), ("gmres", "jacobi", "dia"),
                                                   ("gmres", "none", "sell")])
def test_krylov_solve_matches_oracle(solver, precond, layout):
    pts, el, A, b, h = _linear_system()
    D = dev()
    dm = D.DeviceMesh(pts, el, layout=layout)
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    dinv = D.jacobi_dinv(dm, vals) if precond == "jacobi" else None
    x_ref, k_ref = okry.solve_system(A, b, h, solver, precond, tol=1e-10, maxiter=400, restart=30)
    x, res = D.krylov_solve(dm, vals, cu(b), cu(h), solver=solver, dinv=dinv, tol=1e-10, maxiter=400, restart=30)
    status, iters = host(res)[:2]
    assert status == 0
    assert abs(int(iters) - k_ref) <= max(2, k_ref // 20)
    exact = np.linalg.solve(A.toarray(), b)
    err = np.linalg.norm(host(x) - exact) / np.linalg.norm(exact)
    err_ref = np.linalg.norm(x_ref - exact) / np.linalg.norm(exact)
    assert err <= max(10 * err_ref, 1e-9)
    np.testing.assert_allclose(host(x), x_ref, rtol=1e-7, atol=1e-7)


@pytest.mark.parametrize("solver,layout,n", [("cg", "dia", 30), ("cg", "dia", 256), ("cg", "sell", 30),
                                             ("bicgstab", "dia", 30), ("bicgstab", "dia", 256),
                                             ("bicgstab", "sell", 30), ("gmres", "dia", 30), ("gmres", "dia", 256),
                                             ("gmres", "sell", 30)])
def test_krylov_solve_mixed_reaches_fp64_residual(solver, layout, n):
    """wspm_krylov_solve_mixed: FP32 corrections (CG: pipelined on the DIA layout, single-reduction on SELL;
    BiCGSTAB; GMRES(30)) inside FP64 refinement reach the FP64 residual 1e-8 ||b|| and the FP64 solution of the
    oracle; a second call replays the cached graph and gives bitwise the same x."""
    pts, el, A, b, h = _linear_system(n=n)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout=layout)
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    dinv = D.jacobi_dinv(dm, vals)
    sid = D._lib.SOLVERS[solver]
    ws = torch.empty(int(D.lib.wspm_krylov_mixed_workspace_doubles(dm.n_nodes, dm.nnz_padded, sid, 30)),
                     dtype=torch.float64, device="cuda")
    bb, xx = cu(b), torch.empty(dm.n_nodes, dtype=torch.float64, device="cuda")
    res = torch.zeros(4, dtype=torch.int32, device="cuda")
    kw = dict(dinv=dinv, tol=1e-8, workspace=ws, x_out=xx, result=res, solver=solver, restart=30,
              inner_maxiter=20000 if solver != "gmres" else 2000)
    x, res = D.krylov_solve_mixed(dm, vals, bb, cu(h), **kw)
    status, inner, corrections = host(res)[:3]
    assert status == 0 and corrections >= 1 and inner > 0
    xh = host(x)
    assert np.linalg.norm(b - A @ xh) <= 1.0001e-8 * np.linalg.norm(b)
    exact = np.linalg.solve(A.toarray(), b) if n <= 30 else okry.solve_system(A, b, h, solver, "jacobi", tol=1e-12,
                                                                             maxiter=20000, restart=30)[0]
    np.testing.assert_allclose(xh, exact, rtol=1e-6, atol=1e-6)
    first = x.clone()
    x2, _ = D.krylov_solve_mixed(dm, vals, bb, cu(h), **kw)
    assert torch.equal(first, x2)


@pytest.mark.parametrize("iters", [3, 25])
def test_warm_started_cg_iterates_match_oracle_on_many_blocks(iters):
    """The resident FP64 CG from a non-zero x0 on a DIA system spread over every block (256^2 mesh): its start-up
    computes r = b - A x0 with the row-group SpMV of the iterations, so a wrong start shows in the iterates.  The
    system is the symmetric one (no Dirichlet rows): on a non-symmetric matrix the single-reduction form and the
    textbook iteration differ beyond rounding."""
    pts, el, A, b, h = _linear_system(n=256, dirichlet=False)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout="dia")
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    dinv = D.jacobi_dinv(dm, vals)
    x, res = D.krylov_solve(dm, vals, cu(b), cu(h), solver="cg", dinv=dinv, tol=1e-14, maxiter=iters)
    status, k = host(res)[:2]
    x_ref, k_ref = okry.cg(A, b, h, tol=1e-14, maxiter=iters, dinv=okry.jacobi_inverse_diagonal(A))
    assert status == 1 and k == iters == k_ref
    np.testing.assert_allclose(host(x), x_ref, rtol=1e-9, atol=1e-9)


def test_krylov_maxiter_status_is_reported():
    pts, el, A, b, h = _linear_system(dirichlet=False)
    D = dev()
    dm = D.DeviceMesh(pts, el)
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    x, res = D.krylov_solve(dm, vals, cu(b), cu(h), solver="cg", tol=1e-14, maxiter=3)
    status, iters = host(res)[:2]
    x_ref, k_ref = okry.cg(A, b, h, tol=1e-14, maxiter=3)
    assert status == 1 and iters == 3 == k_ref
    np.testing.assert_allclose(host(x), x_ref, rtol=1e-11)


def test_zero_rhs_gmres_returns_x0():
    pts, el, A, b, h = _linear_system(n=8)
    D = dev()
    dm = D.DeviceMesh(pts, el)
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    x, res = D.krylov_solve(dm, vals, cu(np.zeros_like(b)), cu(h), solver="gmres", tol=1e-10)
    np.testing.assert_array_equal(host(x), h)
    assert host(res)[1] == 0


def _cg_iterations(dm, vals, b, x0, dinv, iters, mode):
    """`iters` iterations of a persistent CG kernel (tolerance 0) through wspm_cg_iterations."""
    import ctypes
    from wspm_b200 import _lib
    work = torch.empty(int(_lib.lib.wspm_krylov_workspace_doubles(dm.n_nodes, 0, 0)), dtype=torch.float64,
                       device="cuda")
    done = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = x0.clone()
    _lib.check("cg_iterations", _lib.lib.wspm_cg_iterations(
        ctypes.byref(dm.c_pat), mode, _lib.dptr(vals), _lib.dptr(b), _lib.dptr(x), _lib.dptr(dinv), iters,
        _lib.dptr(work), work.numel(), _lib.dptr(done), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return x, int(done.item())


@pytest.mark.parametrize("n", [30, 256])
@pytest.mark.parametrize("warp_specialized", [True, False])
def test_pipelined_cg_iterates_match_cg(n, warp_specialized):
    """The pipelined CG kernel (the mixed path's inner solver) against the oracle's restatement of the same
    algorithm: after k iterations from a nonzero x0, x agrees to FP64 rounding (1e-9 norm-wise) and, in FP32, to
    FP32 rounding (1e-4).  Against textbook CG it agrees only up to the recurrence drift of the pipelined form
    (1.3e-5 relative after 25 iterations at n = 256, the same in the oracle restatement and for the
    single-reduction kernel), so that comparison is loose.  n = 256 has 148 blocks of 448 rows."""
    pts, el, A, b, h = _linear_system(n=n)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout="dia")
    assert dm.pattern.n_diags > 0
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    dinv = D.jacobi_dinv(dm, vals)
    dj = okry.jacobi_inverse_diagonal(A)
    k = 25
    pipe = 2 | (0 if warp_specialized else 4)
    x_pref, kp = okry.pipelined_cg(A, b, h, tol=0.0, maxiter=k, dinv=dj)
    x_ref, k_ref = okry.cg(A, b, h, tol=0.0, maxiter=k, dinv=dj)
    assert kp == k_ref == k
    nrm = np.linalg.norm(x_ref)
    x_cg, k1 = _cg_iterations(dm, vals, cu(b), cu(h), dinv, k, 0)
    x_p, k2 = _cg_iterations(dm, vals, cu(b), cu(h), dinv, k, pipe)
    assert (k1, k2) == (k, k)
    assert np.linalg.norm(host(x_p) - x_pref) <= 1e-9 * nrm
    # the single-reduction kernel's recurrences drift from textbook CG alike (1.3e-5 at n = 256)
    assert np.linalg.norm(host(x_cg) - x_ref) <= 1e-4 * nrm
    assert np.linalg.norm(host(x_p) - x_ref) <= 1e-4 * nrm
    # FP32: fewer iterations, before the iterates reach FP32 rounding (where the scalar recurrences of either
    # form may produce a non-finite step and stop the run)
    k32 = 10
    x_pref, _ = okry.pipelined_cg(A, b, h, tol=0.0, maxiter=k32, dinv=dj)
    x_ref, _ = okry.cg(A, b, h, tol=0.0, maxiter=k32, dinv=dj)
    v32, b32, h32, d32 = vals.float(), cu(b, torch.float32), cu(h, torch.float32), dinv.float()
    x_cg32, k3 = _cg_iterations(dm, v32, b32, h32, d32, k32, 1)
    x_p32, k4 = _cg_iterations(dm, v32, b32, h32, d32, k32, 1 | pipe)
    assert (k3, k4) == (k32, k32)
    assert np.linalg.norm(host(x_p32).astype(np.float64) - x_pref) <= 1e-4 * nrm
    # the single-reduction FP32 kernel against textbook FP64 CG: FP32 rounding plus the recurrence drift
    assert np.linalg.norm(host(x_cg32).astype(np.float64) - x_ref) <= 1e-2 * nrm


def test_pipelined_cg_rejects_sell_patterns():
    from wspm_b200._lib import WSPM_UNSUPPORTED, WspmError
    pts, el, A, b, h = _linear_system(n=8)
    D = dev()
    dm = D.DeviceMesh(pts, el, layout="sell")
    vals = cu(dm.pattern.sell_from_csr_values(A.data))
    with pytest.raises(WspmError) as e:
        _cg_iterations(dm, vals, cu(b), cu(h), D.jacobi_dinv(dm, vals), 5, 2)
    assert e.value.code == WSPM_UNSUPPORTED


def _engine_test_case(case, n, solver, precond, layout="auto", **kw):
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(n, 15.24)
    top, bottom = opic.boundary_nodes_2d(pts, case)
    h0 = -15.24 * np.ones(len(pts))
    hup = opic.upper_bc(case, pts[top, 0], EXP[0], np.exp(EXP[0] * h0[top]))
    bc = merge_dirichlet(len(pts), [(top, hup), (bottom, -15.0)])
    eng = PicardEngine(DeviceMesh(pts, tri, layout=layout), "exp", EXP, bc_val=bc, solver=solver, precond=precond,
                       **kw)
    return pts, tri, eng, h0


@pytest.mark.parametrize("case", ["Test1", "Test2", "Test3"])
def test_picard_engine_reproduces_csv_golden_mesh25(case):
    import json
    rows = [r for r in json.load(open(os.path.join(GOLD, "re2d_metrics.json")))
            if r["test_case"] == case and r["mesh"] == 25 and r["solver"] == "cg" and r["precond"] == "jacobi"]
    pts, tri, eng, h0 = _engine_test_case(case, 25, "cg", "jacobi", layout="sell" if case == "Test3" else "auto",
                                          picard_tol=1e-4, picard_maxiter=30, picard_relative=False)
    res = eng.run(h0, 1e-3, 0.25, theta_at_end=False)
    m = analytic.final_errors(pts, res["pressure_head"][-1], res["theta"][-1], res["times"][-1], int(case[-1]))
    assert res["iterations"].sum() == rows[0]["iterations"]
    np.testing.assert_allclose(list(m.values()), rows[0]["metrics"], rtol=5e-4)


def test_picard_engine_matches_oracle_vg_unit_square():
    """The VG unit-square workload (50x50, h0 = -1, top -0.1, cg+jacobi, relative Picard 1e-6)."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(50, 1.0)
    top = np.where(pts[:, 1] == 1.0)[0]
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top)
    ref = opic.run_time_loop(prob, h0, 1e-4, 0.02)
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    eng = PicardEngine(DeviceMesh(pts, tri), "vg", opic.VG_UNIT_PHI, bc_val=bc, solver="cg", precond="jacobi")
    res = eng.run(h0, 1e-4, 0.02)
    np.testing.assert_array_equal(res["iterations"], ref["iterations"])
    np.testing.assert_allclose(res["pressure_head"], ref["pressure_head"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(res["theta"], ref["theta"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("solver", ["bicgstab", "gmres"])
def test_picard_engine_test3d_golden(solver):
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    g = np.load(os.path.join(GOLD, f"test3d_{solver}.npz"))
    pts, tets = mesh.kuhn_tetrahedra(20, 15.24)
    top, bottom = opic.boundary_nodes_3d(pts)
    h0 = -15.24 * np.ones(len(pts))
    hup = opic.upper_bc("Test3D", pts[top, 0], EXP[0], np.exp(EXP[0] * h0[top]), y=pts[top, 1])
    bc = merge_dirichlet(len(pts), [(top, hup), (bottom, -15.0)])
    eng = PicardEngine(DeviceMesh(pts, tets), "exp", EXP, bc_val=bc, solver=solver, precond="none",
                       picard_tol=1e-4, picard_maxiter=30, picard_relative=False)
    res = eng.run(h0, 1e-4, 0.1, theta_at_end=False)
    np.testing.assert_array_equal(res["iterations"], g["iterations"])
    np.testing.assert_allclose(res["dt_values"], g["dt_values"], rtol=0)
    for k, s in enumerate(g["steps"]):
        np.testing.assert_allclose(res["pressure_head"][s], g["pressure_head"][k], rtol=1e-8, atol=1e-8)


@pytest.mark.parametrize("layout", ["auto", "sell"])
def test_mixed_precision_refinement_reaches_fp64_residual(layout):
    """DIA (auto): the inner FP32 solves use the pipelined CG kernel; SELL: the single-reduction kernel.  Both
    reach the FP64 residual and the FP64 path's Picard iterations."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet, spmv
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(96, 1.0)
    rng = np.random.default_rng(5)
    Ks = 0.0922 * np.exp(rng.standard_normal(len(tri)))
    top = np.where(pts[:, 1] == 1.0)[0]
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    phi = opic.VG_UNIT_PHI[:5] + (1.0,)
    dm = DeviceMesh(pts, tri, layout=layout)
    assert (dm.pattern.n_diags > 0) == (layout == "auto")
    out = {}
    for mixed in (False, True):
        eng = PicardEngine(dm, "vg", phi, Ks_elem=Ks, bc_val=bc, solver="cg", precond="jacobi", krylov_tol=1e-8,
                           krylov_maxiter=5000, mixed=mixed)
        res = eng.run(-np.ones(len(pts)), 1e-4, 1e-3, fixed_dt=True, max_steps=3)
        assert np.all(res["status"] == 0)
        # true residual of the last linear system
        r = eng.rhs - spmv(dm, eng.vals, eng.x)
        assert float(torch.linalg.norm(r) / torch.linalg.norm(eng.rhs)) <= 1.01e-8
        out[mixed] = res
    np.testing.assert_array_equal(out[True]["iterations"], out[False]["iterations"])
    np.testing.assert_allclose(out[True]["pressure_head"], out[False]["pressure_head"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("solver,dim", [("bicgstab", 3), ("gmres", 2), ("bicgstab", 2)])
def test_mixed_precision_nonsymmetric_solvers_in_the_picard_step(solver, dim):
    """FP32 BiCGSTAB / GMRES(30) corrections inside the FP64 refinement of the Picard graph (and in its host-driven
    mode): the same Picard iterations as the plain FP64 solver, every linear system to the FP64 residual 1e-8, heads
    agreeing to that accuracy, and the FP64 oracle's step reproduced."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet, spmv
    from wspm_b200.engine import PicardEngine
    if dim == 3:
        pts, el = mesh.kuhn_tetrahedra(14, 1.0)
        top = np.where(np.abs(pts[:, 2] - 1.0) < 1e-12)[0]
        Ks = None
    else:
        pts, el = mesh.structured_triangles(64, 1.0)
        top = np.where(pts[:, 1] == 1.0)[0]
        Ks = 0.0922 * np.exp(np.random.default_rng(7).standard_normal(len(el)))
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    phi = opic.VG_UNIT_PHI if Ks is None else opic.VG_UNIT_PHI[:5] + (1.0,)
    dm = DeviceMesh(pts, el)
    kw = dict(Ks_elem=Ks, bc_val=bc, solver=solver, precond="jacobi", krylov_tol=1e-8, restart=30,
              krylov_maxiter=2000 if solver == "bicgstab" else 200, inner_maxiter=2000 if solver == "bicgstab" else 200)
    out = {}
    for mixed, host_loop in ((False, False), (True, False), (True, True)):
        eng = PicardEngine(dm, "vg", phi, mixed=mixed, **kw)
        eng.host_loop = host_loop
        res = eng.run(-np.ones(len(pts)), 1e-4, 1e-3, fixed_dt=True, max_steps=2)
        assert np.all(res["status"] == 0), res["status"]
        r = eng.rhs - spmv(dm, eng.vals, eng.x)
        assert float(torch.linalg.norm(r) / torch.linalg.norm(eng.rhs)) <= 1.01e-8
        out[(mixed, host_loop)] = res
    for key in ((True, False), (True, True)):
        np.testing.assert_array_equal(out[key]["iterations"], out[(False, False)]["iterations"])
        np.testing.assert_allclose(out[key]["pressure_head"], out[(False, False)]["pressure_head"], rtol=1e-6,
                                   atol=1e-7)
    np.testing.assert_array_equal(out[(True, True)]["pressure_head"], out[(True, False)]["pressure_head"])
    prob, h0 = opic.vg_dirichlet_case(pts, el, top, Ks_elem=Ks, solver=solver, precond="jacobi", tol=1e-8,
                                      maxiter=2000 if solver == "bicgstab" else 200, restart=30)
    ref = opic.run_time_loop(prob, h0, 1e-4, 1e-3, fixed_dt=True, max_steps=2)
    np.testing.assert_array_equal(out[(True, False)]["iterations"], ref["iterations"])
    np.testing.assert_allclose(out[(True, False)]["pressure_head"], ref["pressure_head"], rtol=1e-6, atol=1e-7)


def test_fused_refinement_start_matches_standalone_residual():
    """Without edge terms the mixed path starts its refinement loop inside the assembly launch; with a zero-flux
    Neumann edge (the same linear systems) it runs the stand-alone residual kernel.  Both reach the FP64 residual,
    the same Picard iterations and the same heads to the solver tolerance."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet, spmv
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(96, 1.0)
    rng = np.random.default_rng(6)
    Ks = 0.0922 * np.exp(rng.standard_normal(len(tri)))
    top = np.where(pts[:, 1] == 1.0)[0]
    bottom = np.where(pts[:, 1] == 0.0)[0]
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    phi = opic.VG_UNIT_PHI[:5] + (1.0,)
    dm = DeviceMesh(pts, tri)
    out = {}
    for edges in (None, bottom):
        eng = PicardEngine(dm, "vg", phi, Ks_elem=Ks, bc_val=bc, solver="cg", precond="jacobi", krylov_tol=1e-8,
                           krylov_maxiter=5000, mixed=True, neumann_nodes=edges, neumann_flux=0.0)
        res = eng.run(-np.ones(len(pts)), 1e-4, 1e-3, fixed_dt=True, max_steps=3)
        assert np.all(res["status"] == 0)
        r = eng.rhs - spmv(dm, eng.vals, eng.x)
        assert float(torch.linalg.norm(r) / torch.linalg.norm(eng.rhs)) <= 1.01e-8
        out[edges is None] = res
    np.testing.assert_array_equal(out[True]["iterations"], out[False]["iterations"])
    np.testing.assert_allclose(out[True]["pressure_head"], out[False]["pressure_head"], rtol=1e-7, atol=1e-8)


def test_picard_step_is_bitwise_repeatable():
    pts, tri, eng, h0 = _engine_test_case("Test2", 50, "cg", "jacobi")
    a = eng.run(h0, 1e-3, 0.02)
    b = eng.run(h0, 1e-3, 0.02)
    np.testing.assert_array_equal(a["pressure_head"], b["pressure_head"])
    np.testing.assert_array_equal(a["iterations"], b["iterations"])


@pytest.mark.parametrize("solver,precond,mixed", [("cg", "jacobi", False), ("cg", "jacobi", True),
                                                  ("bicgstab", "none", False), ("gmres", "jacobi", False)])
def test_host_loop_mode_matches_device_loop(solver, precond, mixed):
    """The host-driven step (for profiling tools) runs the same kernels: results are bitwise equal."""
    pts, tri, eng, h0 = _engine_test_case("Test1", 25, solver, precond, mixed=mixed)
    a = eng.run(h0, 1e-3, 0.02)
    eng.host_loop = True
    b = eng.run(h0, 1e-3, 0.02)
    np.testing.assert_array_equal(a["iterations"], b["iterations"])
    np.testing.assert_array_equal(a["krylov_iterations"], b["krylov_iterations"])
    np.testing.assert_array_equal(a["pressure_head"], b["pressure_head"])


@pytest.mark.parametrize("kind,n", [("tri", 64), ("tri", 50), ("tet", 8)])
def test_structural_zero_diagonals_are_exactly_zero(kind, n):
    """A Picard plan on a DIA pattern marks the diagonals whose element stiffness factors are all exactly zero; the
    step's CG and refinement kernels skip them.  Every diagonal it marks must hold exact zeros after assembly (at
    the last Picard iterate, both precisions).  On the split-square grid with exact binary coordinates (n = 64) the
    two diagonals of the edges opposite the right angles (offsets +-(n+2)) are such zeros."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    if kind == "tri":
        pts, el = mesh.structured_triangles(n, 1.0)
        top = np.where(pts[:, 1] == 1.0)[0]
    else:
        pts, el = mesh.kuhn_tetrahedra(n, 1.0)
        top = np.where(np.abs(pts[:, 2] - 1.0) < 1e-12)[0]
    dm = DeviceMesh(pts, el)
    offs = dm.pattern.diag_offsets
    assert dm.pattern.n_diags > 0
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    for mixed in (False, True):
        eng = PicardEngine(dm, "vg", opic.VG_UNIT_PHI, bc_val=bc, solver="cg", precond="jacobi", krylov_tol=1e-8,
                           krylov_maxiter=5000, mixed=mixed)
        live = eng.live_diagonals
        res = eng.run(-np.ones(len(pts)), 1e-4, 1e-3, fixed_dt=True, max_steps=2)
        assert np.all(res["status"] == 0)
        ld = 32 * dm.pattern.n_slices
        vals = host(eng.vals).reshape(len(offs), ld)
        for k, o in enumerate(offs):
            if not (live >> k) & 1:
                assert o != 0 and np.all(vals[k] == 0.0), (k, o)
        if mixed:
            v32 = host(eng.vals32).reshape(len(offs), ld)
            assert all(np.all(v32[k] == 0.0) for k in range(len(offs)) if not (live >> k) & 1)
        if kind == "tri" and n == 64:
            dead = {int(o) for k, o in enumerate(offs) if not (live >> k) & 1}
            assert dead == {n + 2, -(n + 2)}, dead


def _device_pattern_cases():
    from wspm_b200 import mesh as m
    pts, tri = m.structured_triangles(40, 1.0)
    rng = np.random.default_rng(11)
    perm = rng.permutation(len(pts))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(pts))
    p3, tets = m.kuhn_tetrahedra(6, 1.0)
    doms = m.vg_parameter_ensemble(12, 3, sides=(32, 48, 64))
    sizes = np.array([len(d[0]) for d in doms])
    off = np.concatenate([[0], np.cumsum(sizes)])
    union = np.concatenate([d[1] + off[i] for i, d in enumerate(doms)])
    z = np.load(os.path.join(GOLD, "solute_pinns25.npz"))
    return [("tri_auto", tri, len(pts), "auto"), ("tri_sell", tri, len(pts), "sell"),
            ("tri_permuted", inv[tri], len(pts), "auto"), ("tet_auto", tets, len(p3), "auto"),
            ("ensemble_union", union, int(off[-1]), "sell"), ("solute_unstructured", z["triangles"], len(z["points"]),
                                                               "auto")]


@pytest.mark.parametrize("case", range(6))
def test_device_pattern_builder_matches_host_builder(case):
    """wspm_pattern_device_count / _fill build, on the GPU, exactly the arrays of the host builder (CSR, storage
    layout, diagonal positions, incidence with packed row positions) -- structured DIA and SELL, a randomly
    renumbered mesh, tetrahedra, an ensemble's block-diagonal union and the reference's unstructured SoluteTest
    mesh."""
    from wspm_b200.pattern import Pattern
    name, el, n, layout = _device_pattern_cases()[case]
    host = Pattern(el, n, layout=layout, builder="native")
    dev = Pattern(el, n, layout=layout, builder="device")
    assert (dev.layout, dev.n_diags, dev.nnz, dev.nnz_padded, dev.max_width, dev.max_inc) == \
           (host.layout, host.n_diags, host.nnz, host.nnz_padded, host.max_width, host.max_inc), name
    for k in ("csr_indptr", "csr_indices", "sell_index", "slice_ptr", "slice_width", "cols", "diag_pos",
              "diag_offsets", "inc_ptr", "inc_width", "inc_elem", "inc_slots"):
        np.testing.assert_array_equal(getattr(dev, k), getattr(host, k), err_msg=f"{name}: {k}")


def test_device_pattern_builder_rejects_bad_meshes():
    from wspm_b200.pattern import Pattern
    pts, tri = mesh.structured_triangles(4, 1.0)
    bad = tri.copy()
    bad[0, 0] = len(pts)
    with pytest.raises(ValueError):
        Pattern(bad, len(pts), builder="device")
    with pytest.raises(ValueError):
        Pattern(tri, len(pts) + 3, builder="device")          # nodes that belong to no element


def test_engine_on_a_device_built_pattern_matches_host_built():
    """A Picard run on the device-built pattern (DeviceMesh reuses its device arrays) equals the run on the host
    pattern bit for bit."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(48, 1.0)
    top = np.where(pts[:, 1] == 1.0)[0]
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    out = []
    for builder in ("native", "device"):
        eng = PicardEngine(DeviceMesh(pts, tri, builder=builder), "vg", opic.VG_UNIT_PHI, bc_val=bc, solver="cg",
                           precond="jacobi", krylov_tol=1e-8, krylov_maxiter=5000, mixed=True)
        out.append(eng.run(-np.ones(len(pts)), 1e-4, 1e-3, fixed_dt=True, max_steps=2)["pressure_head"])
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("case", ["tri-binary", "tri-decimal", "tri-jitter", "tet-binary", "tet-decimal"])
@pytest.mark.parametrize("mixed", [False, True])
def test_element_shape_table_gives_bitwise_identical_steps(case, mixed):
    """The plan's element-shape path (distinct element Jacobians found once; each element-row's geometric factors
    read from a per-shape table) runs the same Picard steps bit for bit as the assembly that recomputes every
    element's geometry: a grid with exact binary coordinates has 2 triangle shapes (6 Kuhn tetrahedra); a jittered
    mesh has one shape per element, too many, and keeps the recomputing kernel; a triangle grid with coordinates
    i/300 has 800 shapes and a Kuhn grid with coordinates i/21 3,072 (more than the shared-memory table holds): both
    take the global table with 4-bit row positions."""
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    rng = np.random.default_rng(7)
    if case == "tri-binary":
        pts, el = mesh.structured_triangles(64, 1.0)
        want = 2
    elif case == "tri-decimal":   # coordinates i/300: 800 shapes, the global table with 4-bit row positions
        pts, el = mesh.structured_triangles(300, 1.0)
        want = 800
    elif case == "tri-jitter":
        pts, el = mesh.structured_triangles(40, 1.0)
        inner = np.all((pts > 0) & (pts < 1), axis=1)
        pts = pts.copy()
        pts[inner] += rng.uniform(-0.2, 0.2, (int(inner.sum()), 2)) / 40
        want = 0
    elif case == "tet-binary":
        pts, el = mesh.kuhn_tetrahedra(8, 1.0)
        want = 6
    else:   # coordinates i/21: 3,072 distinct Jacobians, the global table with 4-bit row positions
        pts, el = mesh.kuhn_tetrahedra(21, 1.0)
        want = 3072
    dim = pts.shape[1]
    top = np.where(pts[:, dim - 1] == pts[:, dim - 1].max())[0]
    Ks = 0.0922 * np.exp(rng.standard_normal(len(el)))
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    dm = DeviceMesh(pts, el)
    runs, shapes, engines = [], [], []
    for flag in (True, False):
        eng = PicardEngine(dm, "vg", (3.35, 0.368, 0.102, 2.0, 0.5, 1.0), Ks_elem=Ks, bc_val=bc,
                           solver="cg" if dim == 2 else "bicgstab", precond="jacobi", krylov_tol=1e-10,
                           krylov_maxiter=5000, mixed=mixed, inner_tol=1e-5, inner_maxiter=5000,
                           element_shapes=flag)
        shapes.append(eng.element_shape_count())
        runs.append(eng.run(-np.ones(len(pts)), 1e-3, 1.0, fixed_dt=True, max_steps=3))
        engines.append(eng)
    assert shapes == [want, 0]
    np.testing.assert_array_equal(runs[0]["pressure_head"], runs[1]["pressure_head"])
    assert list(runs[0]["iterations"]) == list(runs[1]["iterations"])
    assert list(runs[0]["krylov_iterations"]) == list(runs[1]["krylov_iterations"])
    # one assembly of each plan's current system (wspm_picard_assemble): the same arrays bit for bit
    for eng in engines:
        eng.assemble()
    torch.cuda.synchronize()
    for name in ("vals", "rhs", "dinv"):
        assert torch.equal(getattr(engines[0], name), getattr(engines[1], name)), name
