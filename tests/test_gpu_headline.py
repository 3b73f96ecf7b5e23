"""The headline workload against the FP64 oracle: van Genuchten soil, per-element log-normal Ks
(sigma_lnK 1), h0 -1, top Dirichlet -0.1, dt 1e-4 fixed, relative Picard 1e-6, every linear solve to a
1e-8 relative residual (src/solvers/richards_solver_v2.py:107-168 per step).

* FP64 path (one CUDA graph per step, resident Jacobi-CG): the same Picard iterations as the oracle every
  step, and pressure head and theta within 1e-10 relative (the tolerance of the FP64 mode).
* Mixed path (FP32 pipelined CG inside FP64 refinement to the same 1e-8 residual): the same Picard
  iterations; its error against the oracle is recorded and bounded by 1e-8 relative.

256^2 (66,049 nodes) runs against the NumPy oracle, which is pinned to the reference's goldens;
1024^2 (1,050,625 nodes, the benchmark's size) against the C restatement of the same oracle
(oracle/richards2d.c, itself checked against the NumPy oracle in tests/test_oracle_c.py).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import picard as opic  # noqa: E402
from wspm_b200 import mesh  # noqa: E402

pytestmark = pytest.mark.gpu
FP64_RTOL = 1e-10
MIXED_RTOL = 1e-8
SEED = 2024


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _gpu_runs(pts, tri, Ks, top, steps):
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    dm = DeviceMesh(pts, tri)
    bc = merge_dirichlet(len(pts), [(top, -0.1)])
    phi = opic.VG_UNIT_PHI[:5] + (1.0,)
    out = {}
    for mixed in (False, True):
        eng = PicardEngine(dm, "vg", phi, Ks_elem=Ks, bc_val=bc, solver="cg", precond="jacobi", krylov_tol=1e-8,
                           krylov_maxiter=20000, mixed=mixed, inner_tol=1e-5, inner_maxiter=20000,
                           refine_maxiter=30, picard_tol=1e-6, picard_maxiter=100, picard_relative=True)
        res = eng.run(-np.ones(len(pts)), 1e-4, 1.0, fixed_dt=True, max_steps=steps)
        assert np.all(res["status"] == 0), res["status"]
        out["mixed" if mixed else "fp64"] = res
    return out


def test_headline_workload_256_matches_numpy_oracle():
    steps = 5
    pts, tri, Ks, top = mesh.lognormal_ks_square(256, SEED)
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, Ks_elem=Ks, tol=1e-8, maxiter=100000)
    ref = opic.run_time_loop(prob, h0, 1e-4, 1.0, fixed_dt=True, max_steps=steps)
    gpu = _gpu_runs(pts, tri, Ks, top, steps)
    for name, tol in (("fp64", FP64_RTOL), ("mixed", MIXED_RTOL)):
        res = gpu[name]
        np.testing.assert_array_equal(res["iterations"], ref["iterations"])
        for s in range(steps):
            eh = _rel(res["pressure_head"][s], ref["pressure_head"][s])
            et = _rel(res["theta"][s], ref["theta"][s])
            assert eh <= tol and et <= tol, (name, s, eh, et)
        print(f"256^2 {name}: max rel error vs oracle h "
              f"{max(_rel(res['pressure_head'][s], ref['pressure_head'][s]) for s in range(steps)):.2e}")


def test_headline_workload_1024_matches_c_oracle():
    from oracle import richards2d_c
    richards2d_c.build()
    steps = 3
    pts, tri, Ks, top = mesh.lognormal_ks_square(1024, SEED)
    nodes, vals = opic.dirichlet_arrays(len(pts), [(top, -0.1)])
    phi = opic.VG_UNIT_PHI[:5] + (1.0,)
    ref = richards2d_c.run_vg_fixed_dt(pts, tri, phi, nodes, vals, -np.ones(len(pts)), 1e-4, steps, Ks_elem=Ks,
                                       cg_tol=1e-8, keep_steps=True)
    gpu = _gpu_runs(pts, tri, Ks, top, steps)
    theta_ref = [opic.van_genuchten_model(h, opic.VG_UNIT_PHI[:5] + (1.0,))[2] for h in ref["h_steps"]]
    for name, tol in (("fp64", FP64_RTOL), ("mixed", MIXED_RTOL)):
        res = gpu[name]
        np.testing.assert_array_equal(res["iterations"], ref["picard_its"])
        for s in range(steps):
            eh = _rel(res["pressure_head"][s], ref["h_steps"][s])
            et = _rel(res["theta"][s], theta_ref[s])
            assert eh <= tol and et <= tol, (name, s, eh, et)
    np.testing.assert_array_equal(gpu["fp64"]["krylov_iterations"], ref["cg_its"])
