"""The oracle's coupled water + solute driver against the reference's own logged runs (CPU).

tests/golden/solute_traces.json holds the per-step progress lines of the reference's SoluteTest runs
(logs/40103214: direct solver, logs/40115876: gmres, both without preconditioner) on the 3,828-node mesh
data/mesh/solute/p_Pinns_25.csv (tests/golden/solute_pinns25.npz), and logs/40146207 (gmres) on the
16,384-node p_Pinns_16384.csv (its first steps here; the whole run in tests/test_gpu_solute_trace.py): time after the step (2 decimals),
the last Picard error (3 significant digits), the Picard iterations and the next dt.  The oracle's
restatement of CoupledSolver.solve (src/solvers/coupled_solver_v2.py:223-300) prints the same lines.
Soil: the logged run's configuration (resultsSolute/simulation_config.json: VG Ks 0.25, alpha 3.6,
n 1.56, theta_s .43, theta_r .078), dt0 1e-4, Tmax 1, Krylov tol 1e-10 / maxiter 100 / restart 30.
"""
import json
import os

import numpy as np
import pytest

from oracle import transport as otr

GOLD = os.path.join(os.path.dirname(__file__), "golden")
PHI = (3.6, 0.43, 0.078, 1.56, 1 - 1 / 1.56, 0.25)


def solute_case(size="25"):
    from src.models.boundary import extract_boundary_nodes
    z = np.load(os.path.join(GOLD, f"solute_pinns{size}.npz"))
    pts, tri = z["points"], z["triangles"].astype(np.int64)
    bn = extract_boundary_nodes(pts, "SoluteTest")
    return pts, tri, bn


def printed(time_after, err, its, dt_new):
    return [f"{time_after:.2f}", f"{err:.2e}", int(its), f"{dt_new:.2e}"]


@pytest.mark.parametrize("solver,job,steps,size", [("direct", "40103214", None, "25"), ("gmres", "40115876", 25, "25"),
                                                   ("gmres", "40146207", 8, "16384")])
def test_oracle_reproduces_logged_solute_run(solver, job, steps, size):
    trace = json.load(open(os.path.join(GOLD, "solute_traces.json")))[job]
    assert trace["solver"] == solver and trace["precond"] == "none"
    pts, tri, bn = solute_case(size)
    assert len(pts) == int(trace["summary"]["nodes"]) and len(tri) == int(trace["summary"]["elements"])
    out = otr.coupled_time_loop(pts, tri, PHI, bn.neumann, bn.cauchy, 1e-4, 1.0, solver=solver, precond="none",
                                tol=1e-10, maxiter=100, restart=30, max_steps=steps)
    want = trace["steps"] if steps is None else trace["steps"][:steps]
    got = [printed(out["time"][s], out["error"][s], out["iterations"][s], out["dt"][s]) for s in range(len(want))]
    assert got == want
    if steps is None:
        s = trace["summary"]
        assert len(out["time"]) == len(trace["steps"]) == 131
        assert sum(out["iterations"]) == int(s["total_iterations"])
        assert max(out["iterations"]) == int(s["max_iterations"])
        assert f"{out['error'][-1]:.2e}" == s["final_error"]
        assert f"{np.mean(out['error']):.2e}" == s["average_error"]
