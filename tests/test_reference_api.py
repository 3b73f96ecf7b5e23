"""The reference-facing API (config/, src/) mirrors the reference's names and behaviour."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_settings_defaults_and_quirks():
    from config.settings import SimulationConfig, SolverParameters, VanGenuchtenParameters, create_config_from_dict
    cfg = SimulationConfig()
    assert cfg.solver.solver_type == "gmres" and cfg.solver.precond_type == "ilu"
    assert cfg.solver.tol == 1e-10 and cfg.solver.maxiter == 100 and cfg.solver.restart == 30
    assert cfg.time.m_it == 5 and cfg.time.M_it == 7 and cfg.time.lambda_amp == 2.0
    # m is frozen at 1 - 1/1.56 when only n changes (settings.py:17)
    assert VanGenuchtenParameters(n=2.0).m == pytest.approx(1 - 1 / 1.56)
    np.testing.assert_allclose(cfg.exponential.to_array(), [0.164, 0.45, 0.15, 0.1])
    d = cfg.to_dict()
    assert set(d) == {"exponential", "van_genuchten", "solute", "time", "solver", "mesh", "test_case",
                      "save_frequency"}
    cfg2 = create_config_from_dict(json.loads(json.dumps(d)))
    assert cfg2.solver == cfg.solver
    assert SolverParameters().precision == "fp64"


def test_cli_flags_match_reference():
    from src.cli import build_config, parse_args
    a = parse_args(["--test-case", "Test1", "--mesh-size", "50", "--solver", "cg", "--preconditioner", "jacobi",
                    "--dt", "1e-4", "--tmax", "0.25"])
    assert (a.solver, a.preconditioner, a.dt, a.tmax, a.save_frequency) == ("cg", "jacobi", 1e-4, 0.25, 5)
    d = parse_args([])
    assert (d.mesh_size, d.test_case, d.solver, d.preconditioner, d.dt, d.tmax, d.output_dir) == \
        ("25", "Test1", "gmres", "none", 1e-6, 1.0, "results")
    cfg = build_config(parse_args(["--test-case", "VGDirichlet", "--mesh-dir", "generate"]))
    assert cfg.mesh.mesh_dir is None and cfg.van_genuchten.m == 0.5 and cfg.van_genuchten.n == 2.0


def test_loader_generates_reference_meshes():
    import hashlib
    from src.mesh.loader import load_and_validate_mesh
    dig = json.load(open(os.path.join(GOLD, "mesh_digests.json")))
    p, t, info = load_and_validate_mesh("50", None, "Test1")
    assert hashlib.sha256(p.tobytes()).hexdigest() == dig["richards/p50"]["sha256"]
    assert info["num_points"] == 2601 and info["num_elements"] == 5000
    p, t, info = load_and_validate_mesh("25", None, "Test3D")
    assert hashlib.sha256(t.tobytes()).hexdigest() == dig["richards/t_3D"]["sha256"]
    with pytest.raises(FileNotFoundError):
        load_and_validate_mesh("50", "/nonexistent", "Test1")


def test_exact_solution_matches_oracle():
    from oracle import analytic
    from src.utils.exact_solutions import exact_solution
    x = np.linspace(0, 15.24, 37)
    y = np.linspace(0, 15.24, 37)
    a0, eps0 = 0.164, np.exp(0.164 * -15.24)
    d = a0 * (0.45 - 0.15) / 0.1
    for tn in (1, 2, 3):
        for t in (0.0, 0.05, 0.2):
            h1, s1 = exact_solution(x, y, t, tn, 15.24, a0, eps0, d)
            h2, s2 = analytic.exact_solution(x, y, t, tn, 15.24, a0, eps0, d)
            np.testing.assert_allclose(h1, h2, rtol=1e-12, atol=1e-12)


def test_boundary_sets_and_bottom_truncation():
    from src.models.boundary import BOTTOM_VALUE, extract_boundary_nodes
    from wspm_b200 import mesh
    p, t = mesh.structured_triangles(25, 15.24)
    bn = extract_boundary_nodes(p, "Test1")
    assert len(bn.top) == 26 and len(bn.bottom) == 26 + 2 * 25
    assert len(extract_boundary_nodes(p, "Test3").bottom) == 26
    assert BOTTOM_VALUE == -15.0


@pytest.mark.gpu
def test_richards_solver_published_profile_matches_csv():
    from config.settings import SimulationConfig, SolverParameters, TimeSteppingParameters
    from src.solvers.richards_solver_v2 import RichardsSolver
    from src.utils.error_calculation import calculate_final_errors
    rows = [r for r in json.load(open(os.path.join(GOLD, "re2d_metrics.json")))
            if r["test_case"] == "Test2" and r["mesh"] == 25 and r["solver"] == "bicgstab" and r["precond"] == "jacobi"]
    cfg = SimulationConfig(time=TimeSteppingParameters(dt_init=1e-3, Tmax=0.25),
                           solver=SolverParameters(solver_type="bicgstab", precond_type="jacobi"), test_case="Test2")
    cfg.mesh.mesh_size, cfg.mesh.mesh_dir = "25", None
    res = RichardsSolver(cfg, picard_profile="published").solve()
    m = calculate_final_errors(res, cfg)
    assert int(res["iterations"].sum()) == rows[0]["iterations"]
    np.testing.assert_allclose(list(m.values()), rows[0]["metrics"], rtol=5e-4)


@pytest.mark.gpu
def test_direct_solver_through_shims_matches_engine():
    from config.settings import SimulationConfig, SolverParameters, TimeSteppingParameters
    from src.solvers.richards_solver_v2 import RichardsSolver
    out = {}
    for st, pc in (("direct", "none"), ("cg", "jacobi")):
        cfg = SimulationConfig(time=TimeSteppingParameters(dt_init=1e-3, Tmax=0.01),
                               solver=SolverParameters(solver_type=st, precond_type=pc), test_case="Test1")
        cfg.mesh.mesh_size, cfg.mesh.mesh_dir = "25", None
        out[st] = RichardsSolver(cfg).solve()
    np.testing.assert_array_equal(out["direct"]["iterations"], out["cg"]["iterations"])
    np.testing.assert_allclose(out["direct"]["pressure_head"], out["cg"]["pressure_head"], rtol=1e-8, atol=1e-8)


@pytest.mark.gpu
def test_cli_writes_reference_outputs(tmp_path):
    from src.cli import main
    res = main(["--test-case", "Test1", "--mesh-size", "25", "--solver", "cg", "--preconditioner", "jacobi",
                "--dt", "1e-3", "--tmax", "0.05", "--output-dir", str(tmp_path), "--mesh-dir", "generate"])
    z = np.load(tmp_path / "numerical_results_Test1.npz", allow_pickle=True)
    for k in ("pressure_head", "theta", "times", "points", "iterations", "errors", "dt_values", "simulation_time",
              "elements", "l2_pressure", "linf_pressure", "l2_saturation", "linf_saturation",
              "l2_relative_pressure", "l2_relative_saturation"):
        assert k in z.files
    cfg = json.load(open(tmp_path / "simulation_config.json"))
    assert cfg["solver"]["solver_type"] == "cg" and cfg["test_case"] == "Test1"
    assert z["pressure_head"].shape == (len(res["times"]), 676)


@pytest.mark.gpu
def test_reference_shims_assemble_and_solve():
    import torch
    from oracle import assembly as oasm, soil as osoil
    from src.models.boundary import apply_dirichlet_bcs
    from src.models.exponential import exponential_model
    from src.numerics.assembly_re_v2 import assemble_global_matrices_sparse_re
    from src.numerics.gauss import gauss_triangle
    from src.solvers.solver_types import solve_system
    from config.settings import SolverParameters
    from wspm_b200 import mesh
    p, t = mesh.structured_triangles(20, 15.24)
    h = -15.24 + np.linspace(0, 10, len(p))
    phi = np.array([0.164, 0.45, 0.15, 0.1])
    C, K, th = exponential_model(h, phi)
    Q, W = gauss_triangle(3)
    A, b = assemble_global_matrices_sparse_re(t, len(p), p, th, th, h, K, C, Q, W, 1e-3)
    Cr, Kr, tr = osoil.exponential_model(h, phi)
    Ar, br = oasm.assemble_richards(t, len(p), p, tr, tr, h, Kr, Cr, 1e-3)
    assert np.abs((A.to_scipy() - Ar).toarray()).max() <= 1e-13 * np.abs(Ar.data).max()
    nodes = np.arange(21)
    A, b = apply_dirichlet_bcs(A, b, nodes, -1.0)
    Ar, br = oasm.apply_dirichlet_rows(Ar, br, nodes, -1.0)
    x, info = solve_system(A, b, torch.as_tensor(h, device="cuda"), SolverParameters("cg", "jacobi", tol=1e-12,
                                                                                      maxiter=1000))
    np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(Ar.toarray(), br), rtol=1e-9, atol=1e-9)
    assert int(info[0]) == 0
