"""Command line (drop-in for src/cli.py:51-236).

    python -m src.cli --test-case Test1 --mesh-size 50 --solver cg --preconditioner jacobi \
                      --dt 1e-4 --tmax 0.25 --output-dir results

Same flags, choices and defaults as the reference; writes the same
``simulation_config.json`` and ``numerical_results_<case>.npz`` (keys of
cli.py:155-194).  Plots, the banner and the psutil summary are not produced
(visual/cosmetic; matplotlib is not a dependency).  Additions, under new
names only: ``--precision {fp64,mixed}``, ``--picard-profile {v2,published}``,
``--mesh-dir`` (``generate`` builds the structured meshes in memory) and the
``VGDirichlet`` test case.
"""
import argparse
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

from config.settings import (ExponentialParameters, SimulationConfig, SoluteParameters,  # noqa: E402
                             SolverParameters, TimeSteppingParameters, VanGenuchtenParameters)

MESH_CHOICES = ['25', '50', '100', '200', '400', '1024', '2048', '4096', '8192', '16384', '65536', '267039',
                '1014454']


def parse_args(argv=None):
    p = argparse.ArgumentParser(description="Richards Equation and Solute Transport Solver",
                                formatter_class=argparse.ArgumentDefaultsHelpFormatter)
    p.add_argument("--mesh-size", choices=MESH_CHOICES, default="25", help="Mesh resolution")
    p.add_argument("--test-case", choices=["Test1", "Test2", "Test3", "Test3D", "SoluteTest", "NitrogenTest",
                                           "VGDirichlet"], default="Test1", help="Test case to simulate")
    p.add_argument("--solver", choices=["gmres", "cg", "bicgstab", "direct"], default="gmres",
                   help="Linear solver type")
    p.add_argument("--preconditioner", choices=["none", "jacobi", "ilu", "block_jacobi", "ssor"], default="none",
                   help="Preconditioner type")
    p.add_argument("--dt", type=float, default=1e-6, help="Initial time step size")
    p.add_argument("--tmax", type=float, default=1.0, help="Maximum simulation time")
    p.add_argument("--output-dir", type=str, default="results", help="Directory for output files")
    p.add_argument("--save-frequency", type=int, default=5, help="Frequency of saving results")
    # additions
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                   help="fp64, or FP32 Krylov inside FP64 iterative refinement")
    p.add_argument("--picard-profile", choices=["v2", "published"], default="v2",
                   help="Picard stopping rule: current source (v2) or the published-CSV driver")
    p.add_argument("--mesh-dir", type=str, default="data/mesh",
                   help="mesh directory, or 'generate' for the in-memory structured meshes")
    return p.parse_args(argv)


def build_config(args):
    cfg = SimulationConfig(exponential=ExponentialParameters(), van_genuchten=VanGenuchtenParameters(),
                           solute=SoluteParameters(),
                           time=TimeSteppingParameters(dt_init=args.dt, Tmax=args.tmax),
                           solver=SolverParameters(solver_type=args.solver, precond_type=args.preconditioner,
                                                   precision=args.precision),
                           test_case=args.test_case, save_frequency=args.save_frequency)
    cfg.mesh.mesh_size = args.mesh_size
    cfg.mesh.mesh_dir = None if args.mesh_dir == "generate" else args.mesh_dir
    cfg.picard_profile = args.picard_profile
    if args.test_case == "VGDirichlet":
        # the unit-square VG workload: theta_r .102, theta_s .368, alpha 3.35, n 2, m .5 (set explicitly:
        # the reference's default m is frozen at 1 - 1/1.56), Ks .0922
        cfg.van_genuchten = VanGenuchtenParameters(Ks=0.0922, thetas=0.368, thetar=0.102, alpha=3.35, n=2.0, m=0.5)
    return cfg


def make_solver(cfg):
    if cfg.test_case == "Test3D":
        from src.solvers.richards_solver_3D_v2 import RichardsSolver3D
        return RichardsSolver3D(cfg)
    if cfg.test_case == "SoluteTest":
        from src.solvers.coupled_solver_v2 import CoupledSolver
        return CoupledSolver(cfg)
    if cfg.test_case == "NitrogenTest":
        from src.solvers.nitrogen_solver import NitrogenSolver
        return NitrogenSolver(cfg)
    from src.solvers.richards_solver_v2 import RichardsSolver
    return RichardsSolver(cfg)


def main(argv=None):
    args = parse_args(argv)
    out = Path(args.output_dir)
    out.mkdir(parents=True, exist_ok=True)
    cfg = build_config(args)
    with open(out / "simulation_config.json", "w") as f:
        json.dump(cfg.to_dict(), f, indent=4)
    print(f"Test case: {args.test_case}")
    print(f"Solver: {args.solver} with {args.preconditioner} preconditioner ({args.precision})")
    solver = make_solver(cfg)
    results = solver.solve()
    if args.test_case in ("Test1", "Test2", "Test3"):
        from src.utils.error_calculation import calculate_final_errors
        results.update(calculate_final_errors(results, cfg))
    save = {"pressure_head": results["pressure_head"], "theta": results.get("theta"), "times": results["times"],
            "points": results["points"], "iterations": results["iterations"], "errors": results["errors"],
            "dt_values": results["dt_values"], "simulation_time": results["simulation_time"],
            "memory_usage": 0.0}
    if args.test_case == "Test3D":
        save["elements"] = results["tetrahedra"]
    elif args.test_case == "SoluteTest":
        save["solute"] = results.get("solute")
        save["elements"] = results["triangles"]
    elif args.test_case == "NitrogenTest":
        for k in ("NH4_concentration", "NO2_concentration", "NO3_concentration"):
            save[k] = results[k]
        save["elements"] = results["triangles"]
        save["solute"] = None
    else:
        save["solute"] = None
        save["elements"] = results["triangles"]
    if args.test_case in ("Test1", "Test2", "Test3"):
        for k in ("l2_pressure", "linf_pressure", "l2_saturation", "linf_saturation", "l2_relative_pressure",
                  "l2_relative_saturation"):
            save[k] = float(results.get(k, 0))
    np.savez(out / f"numerical_results_{args.test_case}.npz", **save)
    its = np.asarray(results["iterations"])
    print(f"steps {len(its)}, Picard iterations {int(its.sum())}, simulation time {results['simulation_time']:.3f} s")
    if "l2_pressure" in results:
        print("errors: " + ", ".join(f"{k}={results[k]:.4e}" for k in ("l2_pressure", "linf_pressure",
                                                                      "l2_saturation", "linf_saturation")))
    return results


if __name__ == "__main__":
    main()
