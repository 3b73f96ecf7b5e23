"""The allocation-free CG entry point (wspm_cg_solve_noalloc) against the regular one.

Callers that cannot allocate device memory (code running inside a JAX
program, whose allocator has reserved most of the GPU, or inside a stream
capture) use wspm_cg_solve_noalloc: its scratch is a static array inside the
library.  This file is collected last on purpose, so that a run stopping at
the first failure has already run every other test; it must also pass on its
own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _system(n=40):
    from oracle import assembly as oasm, picard as opic, soil as osoil
    from wspm_b200 import mesh
    pts, el = mesh.structured_triangles(n, 15.24)
    h = -15.24 + np.linspace(0.0, 12.0, len(pts))
    C, K, th = osoil.exponential_model(h, (0.164, 0.45, 0.15, 0.1))
    A, b = oasm.assemble_richards(el, len(pts), pts, th, th - 1e-3, h, K, C, 5e-3)
    top, bottom = opic.boundary_nodes_2d(pts, "Test1")
    nodes, values = opic.dirichlet_arrays(len(pts), [(top, -1.0), (bottom, -15.0)])
    A, b = oasm.apply_dirichlet_rows(A, b, nodes, values)
    return pts, el, A, b, h


def test_noalloc_rejects_oversized_systems_before_launching():
    from wspm_b200 import _lib
    pat = _lib.WspmPattern()
    pat.n_rows = _lib.NOALLOC_MAX_ROWS + 1
    rc = _lib.lib.wspm_cg_solve_noalloc(ctypes.byref(pat), None, None, None, None, 1e-8, 0.0, 10, None, None)
    assert rc == _lib.WSPM_BAD_ARG


def _noalloc(dm, vals, bt, x0, dinv, tol, maxiter, stream):
    from wspm_b200 import _lib
    x = x0.clone()
    result = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    rc = _lib.lib.wspm_cg_solve_noalloc(ctypes.byref(dm.c_pat), _lib.dptr(vals), _lib.dptr(bt), _lib.dptr(x),
                                        _lib.dptr(dinv), tol, 0.0, maxiter, _lib.dptr(result), stream)
    assert rc == _lib.WSPM_OK
    torch.cuda.synchronize()
    return x.cpu().numpy(), result.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["jacobi", "none"])
def test_noalloc_cg_matches_workspace_cg_twice(precond):
    """Two calls in a row on the shared static scratch, each equal bit for bit to wspm_krylov_solve's CG (the
    same resident kernel, the Krylov vectors in the library's array instead of the caller's workspace); without
    a preconditioner (dinv NULL) also checked against the oracle's textbook CG."""
    from oracle import krylov as okry
    from wspm_b200 import _lib
    from wspm_b200.device import DeviceMesh, jacobi_dinv, krylov_solve
    pts, el, A, b, h = _system()
    dm = DeviceMesh(pts, el)
    vals = torch.as_tensor(dm.pattern.sell_from_csr_values(A.data), device="cuda")
    bt = torch.as_tensor(b, device="cuda")
    h0 = torch.as_tensor(h, device="cuda")
    dinv = jacobi_dinv(dm, vals) if precond == "jacobi" else None
    maxiter = 2000
    x_ref, res_ref = krylov_solve(dm, vals, bt, h0, solver="cg", dinv=dinv, tol=1e-10, maxiter=maxiter)
    x_ref = x_ref.cpu().numpy().copy()
    ref = res_ref.cpu().numpy().copy()
    assert ref[0] == 0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        x, got = _noalloc(dm, vals, bt, h0, dinv, 1e-10, maxiter, stream)
        assert got[0] == _lib.WSPM_OK and got[1] == ref[1], (call, got, ref)
        np.testing.assert_array_equal(x, x_ref)
    if precond == "none":
        x_or, k_or = okry.solve_system(A, b, h, "cg", "none", tol=1e-10, maxiter=maxiter)
        assert abs(int(got[1]) - k_or) <= max(2, k_or // 20), (got[1], k_or)
        exact = np.linalg.solve(A.toarray(), b)
        err = np.linalg.norm(x - exact) / np.linalg.norm(exact)
        err_or = np.linalg.norm(x_or - exact) / np.linalg.norm(exact)
        assert err <= max(10 * err_or, 1e-9), (err, err_or)
        np.testing.assert_allclose(x, x_or, rtol=1e-7, atol=1e-7)


@pytest.mark.gpu
def test_noalloc_cg_reports_the_iteration_cap():
    """A cap below the iterations the solve needs ends with WSPM_MAXITER and exactly `maxiter` iterations."""
    from wspm_b200 import _lib
    from wspm_b200.device import DeviceMesh, jacobi_dinv
    pts, el, A, b, h = _system()
    dm = DeviceMesh(pts, el)
    vals = torch.as_tensor(dm.pattern.sell_from_csr_values(A.data), device="cuda")
    bt = torch.as_tensor(b, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _, got = _noalloc(dm, vals, bt, torch.as_tensor(h, device="cuda"), jacobi_dinv(dm, vals), 1e-10, 3, stream)
    assert got[0] == _lib.WSPM_MAXITER and got[1] == 3, got
