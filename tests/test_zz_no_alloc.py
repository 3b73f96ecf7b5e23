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


@pytest.mark.gpu
def test_noalloc_cg_matches_workspace_cg_twice():
    from wspm_b200 import _lib
    from wspm_b200.device import DeviceMesh, jacobi_dinv, krylov_solve
    pts, el, A, b, h = _system()
    dm = DeviceMesh(pts, el)
    vals = torch.as_tensor(dm.pattern.sell_from_csr_values(A.data), device="cuda")
    bt = torch.as_tensor(b, device="cuda")
    dinv = jacobi_dinv(dm, vals)
    x_ref, res_ref = krylov_solve(dm, vals, bt, torch.as_tensor(h, device="cuda"), solver="cg", dinv=dinv,
                                  tol=1e-10, maxiter=500)
    x_ref = x_ref.clone()
    ref = res_ref.cpu().numpy().copy()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    first = None
    for call in range(2):                      # two calls in a row share the static scratch
        x = torch.as_tensor(h, device="cuda").clone()
        result = torch.full((4,), -7, dtype=torch.int32, device="cuda")
        rc = _lib.lib.wspm_cg_solve_noalloc(ctypes.byref(dm.c_pat), _lib.dptr(vals), _lib.dptr(bt), _lib.dptr(x),
                                            _lib.dptr(dinv), 1e-10, 0.0, 500, _lib.dptr(result), stream)
        assert rc == _lib.WSPM_OK, call
        torch.cuda.synchronize()
        got = result.cpu().numpy()
        assert got[0] == ref[0] == 0 and got[1] == ref[1], (call, got, ref)
        # the workspace entry runs the single-reduction CG kernel, this one the two-reduction form: the same
        # iteration count, iterates equal to the accuracy of a 1e-10 relative-residual solve
        np.testing.assert_allclose(x.cpu().numpy(), x_ref.cpu().numpy(), rtol=1e-8, atol=1e-9)
        # the second call on the reused scratch repeats the first bit for bit
        if first is None:
            first = x.cpu().numpy().copy()
        else:
            np.testing.assert_array_equal(x.cpu().numpy(), first)
