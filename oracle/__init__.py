"""CPU oracle for the JAX-WSPM implicit P1-FEM Picard path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ``jax-wspm_b200``
package, its CUDA library or its Python shims) imports this package.  Only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or as the timed CPU baseline.

The oracle is a NumPy/SciPy FP64 restatement of the reference (JAX-WSPM,
pure Python + JAX; JAX itself is not installed here, so the reference
cannot be imported).  Each function cites the reference ``file:line`` it
follows.  Krylov solvers restate the published algorithms with the stopping
semantics of ``jax.scipy.sparse.linalg`` (jax/jaxlib, unpinned in the
reference's requirements.txt:1-2): ``||r|| <= max(tol*||b||, atol)``,
``maxiter`` counted in iterations for CG/BiCGSTAB and in restart cycles for
GMRES.

Parity pinning (see ``tests/golden``):
  * ``resultsRE2D/benchmark_results_*_Test{1,2,3}_WA.csv`` -- Picard
    iteration totals and the six analytical-error metrics for the 2D
    Richards tests at mesh 25 and 50 (reproduced by ``oracle.picard``);
  * ``results3D/numerical_results_Test3D_*_mesh25.npz`` -- per-step Picard
    iteration counts and full pressure-head fields for Test3D.
Solute and nitrogen transport have no numeric goldens in the reference:
those parts of the oracle are parity-unpinned (literal restatements only).
"""
