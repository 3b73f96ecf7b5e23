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


# ---------------------------------------------------------------- transport steps and drivers
def _config(test_case, mesh_size, mesh_dir, solver="gmres", precond="jacobi", dt=1e-3):
    from config.settings import SimulationConfig, SolverParameters, TimeSteppingParameters
    cfg = SimulationConfig(time=TimeSteppingParameters(dt_init=dt, Tmax=1.0),
                           solver=SolverParameters(solver_type=solver, precond_type=precond), test_case=test_case)
    cfg.mesh.mesh_size = mesh_size
    cfg.mesh.mesh_dir = mesh_dir
    return cfg


def _solute_mesh(tmp_path, n=20):
    """[-0.5, 0.5] x [0, 2] split squares written as the reference's SoluteTest CSV files (1-based elements)."""
    pts, tri = mesh.structured_triangles(n, 1.0)
    pts = np.column_stack([pts[:, 0] - 0.5, 2.0 * pts[:, 1]])
    d = tmp_path / "solute"
    d.mkdir(parents=True, exist_ok=True)
    np.savetxt(d / "p_Pinns_t.csv", pts, delimiter=",")
    np.savetxt(d / "t_Pinns_t.csv", tri + 1, delimiter=",", fmt="%d")
    return str(tmp_path)


def test_solute_step_matches_oracle():
    from wspm_b200.device import DeviceMesh
    from wspm_b200.engine import default_rule
    from wspm_b200.transport import edges_or_none, solute_step
    pts, tri, h = field(seed=4)
    top = np.where(pts[:, 1] == 1.0)[0]
    fx = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.5, 0.1, 0.0)
    qx, qz, aq, Dxx, Dxz, Dzz, th = fx
    c_n = np.linspace(0.1, 0.3, len(pts))
    want = otr.solute_step(pts, tri, c_n, th, th, qx, qz, Dxx, Dxz, Dzz, 1e-3, top, -0.1, 1.0,
                           solver="gmres", precond="jacobi")
    dm = DeviceMesh(pts, tri)
    got, _ = solute_step(dm, cu(c_n), *[cu(a) for a in (th, qx, qz, Dxx, Dxz, Dzz)], 1e-3, default_rule(2),
                         edges_or_none(dm, top), -0.1, 1.0, solver="gmres", precond="jacobi")
    np.testing.assert_allclose(host(got), want, rtol=1e-9, atol=1e-11)


def test_nitrogen_species_chain_matches_oracle():
    from wspm_b200.device import DeviceMesh
    from wspm_b200.engine import default_rule
    from wspm_b200.transport import edges_or_none, nitrogen_species_step
    pts, tri, h = field(seed=5)
    top = np.where(np.abs(pts[:, 1] - 1.0) < 1e-10)[0]
    bot = np.where(np.abs(pts[:, 1]) < 1e-10)[0]
    qx, qz, aq, Dxx, Dxz, Dzz, th = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.04, 0.0004, 0.288e-4)
    _, Kn, _ = osoil.van_genuchten_model(h, VG_SOLUTE)
    rng = np.random.default_rng(6)
    c1, c2, c3 = (rng.uniform(0, 5, len(pts)) for _ in range(3))
    dm = DeviceMesh(pts, tri)
    ce, fe = edges_or_none(dm, top), edges_or_none(dm, bot)
    kw = dict(solver="gmres", precond="jacobi")
    species = [(c1, 0.12, 1.6e-6 * 0.34e-6, 0.0, 50.0), (c2, 0.048, 0.0, 0.12, 0.0), (c3, 0.012, 0.0, 0.048, 20.0)]
    up_ref = up_gpu = None
    for c_n, mu, sorp, mu_up, c_in in species:
        want = otr.nitrogen_species_step(pts, tri, c_n, th, qx, qz, Dxx, Dxz, Dzz, Kn, 2e-3, mu, sorp, mu_up, up_ref,
                                         top, -0.05, c_in, bot, **kw)
        got, _ = nitrogen_species_step(dm, cu(c_n), *[cu(a) for a in (th, qx, qz, Dxx, Dxz, Dzz, Kn)], 2e-3,
                                       default_rule(2), mu=mu, sorption=sorp, mu_up=mu_up, c_up=up_gpu,
                                       cauchy_edges=ce, cauchy_flux=-0.05, c_in=c_in, fd_edges=fe, **kw)
        np.testing.assert_allclose(host(got), want, rtol=1e-9, atol=1e-9 * max(1.0, np.abs(want).max()))
        up_ref, up_gpu = want, cu(want)


def _oracle_transport_run(pts, tri, cfg, steps, nitrogen):
    """The drivers' time loop restated on the oracle's step functions."""
    from src.models.boundary import extract_boundary_nodes
    phi = cfg.van_genuchten.to_array()
    bn = extract_boundary_nodes(pts, cfg.test_case)
    kw = dict(solver=cfg.solver.solver_type, precond=cfg.solver.precond_type, tol=cfg.solver.tol,
              maxiter=cfg.solver.maxiter, restart=cfg.solver.restart)
    n = len(pts)
    h_n = (-1.0 if nitrogen else -1.3) * np.ones(n)
    if nitrogen:
        p = cfg.nitrogen
        cs = [np.full(n, p.c_init_NH4), np.full(n, p.c_init_NO2), np.full(n, p.c_init_NO3)]
    else:
        c_n = np.full(n, cfg.solute.c_init)
    dt = cfg.time.dt_init
    hist = []
    for _ in range(steps):
        _, _, th_n = osoil.van_genuchten_model(h_n, phi)
        if nitrogen:
            h, err, it = otr.richards_neumann_step(pts, tri, h_n, th_n, dt, phi, bn.neumann, -0.05,
                                                   fd_nodes=bn.freedrainage, picard_tol=1e-6, **kw)
            p = cfg.nitrogen
            qx, qz, aq, Dxx, Dxz, Dzz, th = otr.fluxes_and_dispersion(pts, tri, h, phi, p.DL, p.DT, p.Dm)
            _, Kn, _ = osoil.van_genuchten_model(h, phi)
            up = None
            new = []
            for c_n, mu, sorp, mu_up, c_in in ((cs[0], p.mu1, p.rho * p.Kd, 0.0, p.c_inlet_NH4),
                                               (cs[1], p.mu2, 0.0, p.mu1, p.c_inlet_NO2),
                                               (cs[2], p.mu3, 0.0, p.mu2, p.c_inlet_NO3)):
                c = otr.nitrogen_species_step(pts, tri, c_n, th, qx, qz, Dxx, Dxz, Dzz, Kn, dt, mu, sorp, mu_up, up,
                                              bn.cauchy, -0.05, c_in, bn.freedrainage, **kw)
                new.append(c)
                up = c
            cs = new
            hist.append((h, it, *cs))
            dt = min(1.2 * dt, 0.01) if it <= 5 else (dt if it <= 15 else max(0.5 * dt, 1e-6))
        else:
            h, err, it = otr.richards_neumann_step(pts, tri, h_n, th_n, dt, phi, bn.neumann, -0.1, picard_tol=1e-4,
                                                   **kw)
            s = cfg.solute
            qx, qz, aq, Dxx, Dxz, Dzz, th = otr.fluxes_and_dispersion(pts, tri, h, phi, s.DL, s.DT, s.Dm)
            c_n = otr.solute_step(pts, tri, c_n, th, th_n, qx, qz, Dxx, Dxz, Dzz, dt, bn.cauchy, -0.1, s.c_inlet,
                                  **kw)
            hist.append((h, it, c_n))
            t = cfg.time
            dt = max(t.lambda_amp * dt if it <= t.m_it else (dt if it <= t.M_it else t.lambda_red * dt), 1e-6)
        h_n = h
    return hist


def test_coupled_solver_matches_oracle_driver(tmp_path):
    from src.solvers.coupled_solver_v2 import CoupledSolver
    cfg = _config("SoluteTest", "t", _solute_mesh(tmp_path))
    solver = CoupledSolver(cfg)
    assert len(solver.boundary_nodes.cauchy) >= 2
    res = solver.solve(max_steps=3)
    want = _oracle_transport_run(solver.points, solver.triangles, cfg, 3, nitrogen=False)
    for s, (h, it, c) in enumerate(want):
        assert res["iterations"][s] == it
        np.testing.assert_allclose(res["pressure_head"][s], h, rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(res["solute"][s], c, rtol=1e-8, atol=1e-10)
    assert set(res) >= {"pressure_head", "theta", "solute", "times", "iterations", "errors", "dt_values",
                        "final_solute", "triangles"}


def test_nitrogen_solver_matches_oracle_driver():
    from src.solvers.nitrogen_solver import NitrogenSolver
    cfg = _config("NitrogenTest", "25", None, dt=2e-3)
    solver = NitrogenSolver(cfg)
    res = solver.solve(max_steps=3)
    want = _oracle_transport_run(solver.points, solver.triangles, cfg, 3, nitrogen=True)
    for s, (h, it, nh4, no2, no3) in enumerate(want):
        assert res["iterations"][s] == it
        np.testing.assert_allclose(res["pressure_head"][s], h, rtol=1e-9, atol=1e-10)
        for key, c in (("NH4_concentration", nh4), ("NO2_concentration", no2), ("NO3_concentration", no3)):
            np.testing.assert_allclose(res[key][s], c, rtol=1e-8, atol=1e-8 * max(1.0, np.abs(c).max()))


def test_mass_integral_and_peclet_courant_match_oracle():
    from src.models.transport_utilities import calculate_peclet_courant
    from src.utils.mass_balance import integrate_2d_domain
    pts, tri, h = field(seed=8)
    th = osoil.van_genuchten_model(h, VG_SOLUTE)[2]
    assert abs(integrate_2d_domain(th, pts, tri) - otr.integrate_2d_domain(th, pts, tri)) <= 1e-13 * abs(
        otr.integrate_2d_domain(th, pts, tri))
    qx, qz, aq, Dxx, Dxz, Dzz, th = otr.fluxes_and_dispersion(pts, tri, h, VG_SOLUTE, 0.5, 0.1, 0.0288)
    got = calculate_peclet_courant(pts, tri, qx, qz, th, Dxx, Dzz, 1e-3)
    want = otr.peclet_courant(pts, tri, qx, qz, th, Dxx, Dzz, 1e-3)
    np.testing.assert_allclose(got, want, rtol=1e-13)
