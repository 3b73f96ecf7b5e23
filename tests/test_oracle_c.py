"""The C + OpenMP oracle (oracle/richards2d.c) against the NumPy oracle it restates (CPU).

The NumPy oracle is pinned to the reference's goldens (tests/test_oracle_goldens.py); the C
restatement runs the same fixed-dt van Genuchten time loop fast enough for the 1024^2 workload.
Both must take the same Picard iterations every step and agree to rounding (1e-13 relative).
"""
import numpy as np
import pytest

from oracle import picard as opic
from wspm_b200 import mesh


@pytest.fixture(scope="module")
def c_oracle():
    from oracle import richards2d_c
    richards2d_c.build()
    return richards2d_c


@pytest.mark.parametrize("n,per_element_ks,threads", [(48, True, 0), (48, True, 1), (40, False, 3)])
def test_c_oracle_matches_numpy_oracle(c_oracle, n, per_element_ks, threads):
    pts, tri, Ks, top = mesh.lognormal_ks_square(n, 7)
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, Ks_elem=Ks if per_element_ks else None, tol=1e-8,
                                      maxiter=100000)
    ref = opic.run_time_loop(prob, h0, 1e-4, 1.0, fixed_dt=True, max_steps=3)
    phi = prob.phi
    out = c_oracle.run_vg_fixed_dt(pts, tri, phi, prob.bc_nodes, prob.bc_vals, h0, 1e-4, 3,
                                   Ks_elem=Ks if per_element_ks else None, cg_tol=1e-8, threads=threads,
                                   keep_steps=True)
    np.testing.assert_array_equal(out["picard_its"], ref["iterations"])
    for s in range(3):
        h_ref = ref["pressure_head"][s]
        assert np.linalg.norm(out["h_steps"][s] - h_ref) / np.linalg.norm(h_ref) <= 1e-13
    np.testing.assert_array_equal(out["h"], out["h_steps"][-1])


def test_c_oracle_rejects_bad_connectivity(c_oracle):
    pts, tri = mesh.structured_triangles(4, 1.0)
    bad = tri.copy()
    bad[0, 0] = len(pts)
    with pytest.raises(RuntimeError):
        c_oracle.run_vg_fixed_dt(pts, bad, opic.VG_UNIT_PHI, [], [], -np.ones(len(pts)), 1e-4, 1)
