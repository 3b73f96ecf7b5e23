"""Transport path (solute / nitrogen) on the GPU against the oracle restatement.

No numeric goldens exist in the reference for these paths, so parity is
against oracle/transport.py only (parity-unpinned).  Tolerance: 1e-12 relative
to the largest entry for assembled matrices and vectors.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import soil as osoil, transport as otr  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu
VG_SOLUTE = (3.6, 0.43, 0.078, 1.56, 1 - 1 / 1.56, 0.2496)


def cu(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def field(n=20, L=1.0, seed=0):
    rng = np.random.default_rng(seed)
    pts, tri = mesh.structured_triangles(n, L)
    h = -0.3 - 0.5 * pts[:, 1] + 0.05 * rng.standard_normal(len(pts))
    return pts, tri, h


def close(got, want, rel=1e-12):
    want = np.asarray(want)
    scale = max(np.abs(want).max(), 1e-300)
    assert np.abs(np.asarray(got) - want).max() <= rel * scale, np.abs(np.asarray(got) - want).max() / scale


@pytest.mark.parametrize("layout", ["dia", "sell"])
def test_flux_dispersion(layout):
    from wspm_b200.device import DeviceMesh, flux_dispersion
    pts, tri, h = field()
    dm = DeviceMesh(pts, tri, layout=layout)
    got = flux_dispersion(dm, cu(h), VG_SOLUTE, 0.5, 0.1, 0.0288)
    want = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.5, 0.1, 0.0288)
    for g, w in zip(got, want):
        close(host(g), w, 1e-12)


@pytest.mark.parametrize("lumped,mu,sorption,mu_up,layout", [(False, 0.0, 0.0, 0.0, "dia"),
                                                            (True, 0.12, 0.5, 0.0, "dia"),
                                                            (True, 0.048, 0.0, 0.12, "sell")])
def test_adr_assembly(lumped, mu, sorption, mu_up, layout):
    from wspm_b200.device import DeviceMesh, assemble_adr
    from wspm_b200.engine import default_rule
    pts, tri, h = field(seed=1)
    fx = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.5, 0.1, 0.0)
    qx, qz, aq, Dxx, Dxz, Dzz, th = fx
    rng = np.random.default_rng(2)
    c_n = rng.uniform(0, 1, len(pts))
    c_up = rng.uniform(0, 2, len(pts)) if mu_up else None
    dt = 1e-3
    K, M, F = otr.assemble_adr(tri, len(pts), pts, th, qx, qz, Dxx, Dxz, Dzz, mu=mu, sorption=sorption, mu_up=mu_up,
                               c_up=c_up)
    if lumped:
        M = otr.lump(M)
    A_ref = ((1.0 / dt) * M + K).tocsr()
    b_ref = (1.0 / dt) * (M @ c_n) + F
    dm = DeviceMesh(pts, tri, layout=layout)
    Q, W = default_rule(2)
    vals, rhs, dinv = assemble_adr(dm, *[cu(a) for a in (th, qx, qz, Dxx, Dxz, Dzz, c_n)], dt, Q, W, mu=mu,
                                   sorption=sorption, mu_up=mu_up, c_up=None if c_up is None else cu(c_up),
                                   lumped=lumped)
    A = dm.pattern.to_scipy(host(vals))
    assert np.abs((A - A_ref).toarray()).max() <= 1e-12 * np.abs(A_ref.data).max()
    close(host(rhs), b_ref)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_edge_terms(mode):
    from wspm_b200.device import BoundaryEdges, DeviceMesh, apply_edge_terms, assemble_adr
    from wspm_b200.engine import default_rule
    pts, tri, h = field(seed=3)
    qx, qz, aq, Dxx, Dxz, Dzz, th = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.5, 0.1, 0.0)
    _, Kn, _ = osoil.van_genuchten_model(h, VG_SOLUTE)
    c_n = np.linspace(0, 1, len(pts))
    K, M, F = otr.assemble_adr(tri, len(pts), pts, th, qx, qz, Dxx, Dxz, Dzz)
    A0 = ((1.0 / 1e-3) * M + K).tocsr()
    b0 = (1.0 / 1e-3) * (M @ c_n)
    top = np.where(pts[:, 1] == 1.0)[0]
    if mode == 0:
        A_ref, b_ref = A0, otr.neumann_rhs(b0, -0.05, top, pts)
    elif mode == 1:
        A_ref, b_ref = A0, otr.freedrainage_water_rhs(b0, Kn, top, pts)
    elif mode == 2:
        A_ref, b_ref = otr.cauchy(A0, b0, -0.05, 50.0, top, pts)
    else:
        A_ref, b_ref = otr.freedrainage_nitrogen(A0, b0, Kn, th, top, pts)
    dm = DeviceMesh(pts, tri)
    Q, W = default_rule(2)
    vals, rhs, _ = assemble_adr(dm, *[cu(a) for a in (th, qx, qz, Dxx, Dxz, Dzz, c_n)], 1e-3, Q, W)
    edges = BoundaryEdges(dm, top)
    apply_edge_terms(dm, edges, mode, rhs, vals=vals, flux=-0.05, c_in=50.0, K=cu(Kn), theta=cu(th))
    A = dm.pattern.to_scipy(host(vals))
    assert np.abs((A - A_ref).toarray()).max() <= 1e-12 * np.abs(A_ref.data).max()
    close(host(rhs), b_ref)


def test_coupled_richards_step_with_neumann_and_drainage():
    """solve_richards_step of the nitrogen driver: VG, Neumann on top, free drainage at the bottom."""
    from wspm_b200.device import DeviceMesh
    from wspm_b200.engine import PicardEngine
    pts, tri = mesh.structured_triangles(25, 1.0)
    top = np.where(np.abs(pts[:, 1] - 1.0) < 1e-10)[0]
    bottom = np.where(np.abs(pts[:, 1]) < 1e-10)[0]
    phi = VG_SOLUTE
    h0 = -1.0 * np.ones(len(pts))
    _, _, th0 = osoil.van_genuchten_model(h0, phi)
    h_ref, err_ref, it_ref = otr.richards_neumann_step(pts, tri, h0, th0, 1e-3, phi, top, -0.05, fd_nodes=bottom,
                                                       solver="gmres", precond="none", picard_tol=1e-6)
    eng = PicardEngine(DeviceMesh(pts, tri), "vg", phi, solver="gmres", precond="none", krylov_tol=1e-10,
                       krylov_maxiter=100, restart=30, picard_tol=1e-6, picard_maxiter=100, picard_relative=False,
                       neumann_nodes=top, neumann_flux=-0.05, drainage_nodes=bottom)
    eng.set_state(h0)
    res = eng.step(1e-3)
    assert res["status"] == 0 and res["iterations"] == it_ref
    np.testing.assert_allclose(host(eng.h_n), h_ref, rtol=1e-9, atol=1e-10)
