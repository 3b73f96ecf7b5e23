"""Regenerate the committed golden fixtures from the reference tree.

Run where a checkout of the reference project is available (read-only is
fine), giving its root directory as the argument or in the environment
variable WSPM_REFERENCE_ROOT:

    python tests/golden/make_goldens.py /path/to/JAX-WSPM

It writes, next to this script:
  * ``re2d_metrics.json``  -- every row of resultsRE2D/benchmark_results_*_WA.csv
    (test case, mesh, solver, preconditioner, Picard iteration total and the six
    analytical-error metrics to 5 significant digits);
  * ``test3d_<solver>.npz`` -- results3D/numerical_results_Test3D_*_mesh25.npz:
    per-step iterations, dt, times, Picard errors and the pressure-head field of
    steps 0, 4 and 9 (the full 10 x 9261 field is not needed);
  * ``solute_pinns25.npz`` -- the SoluteTest mesh data/mesh/solute/p_Pinns_25.csv /
    t_Pinns_25.csv as loaded (float64 points, 0-based int64 triangles);
  * ``solute_traces.json`` -- the per-step progress lines of the reference's
    SoluteTest runs in logs/ (time after the step, last Picard error, Picard
    iterations and the next dt, as printed: 2 decimals / 3 significant digits)
    and the totals of their .out summaries, for the 3,828-node mesh (bicgstab,
    gmres, direct; no preconditioner) and the 16,384-node mesh (gmres);
  * ``solute_pinns16384.npz`` -- the 16,384-node SoluteTest mesh
    (p_Pinns_16384.csv / t_Pinns_16384.csv; triangles stored as int32);
  * ``mesh_digests.json`` -- shape and SHA-256 of the reference meshes
    (data/mesh/richards/p*.csv, t*.csv, p_3D.csv, t_3D.csv; nitrogen p_*.csv,
    t_*.csv) as loaded by src/mesh/loader.py:69-71 (float64 points, 0-based
    int64 connectivity), so the structured generators can be checked without
    the reference tree.
Nothing at test time reads the reference tree.
"""
import csv
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def digest(a):
    a = np.ascontiguousarray(a)
    return {"shape": list(a.shape), "dtype": str(a.dtype), "sha256": hashlib.sha256(a.tobytes()).hexdigest()}


def load_csv(path, dtype):
    return np.loadtxt(path, delimiter=",", dtype=dtype, ndmin=2)


def main(ref):
    rows = []
    d = os.path.join(ref, "resultsRE2D")
    for name in sorted(os.listdir(d)):
        if not name.endswith(".csv"):
            continue
        hw = "gpu" if "_gpu_" in name else "cpu"
        with open(os.path.join(d, name)) as f:
            for r in csv.DictReader(f):
                rows.append({"file": name, "hw": hw, "test_case": r["test_case"], "mesh": int(r["mesh_size"]),
                             "solver": r["solver"], "precond": r["preconditioner"],
                             "iterations": int(r["iterations"]),
                             "metrics": [float(r[k]) for k in ("l2_pressure", "linf_pressure", "l2_saturation",
                                                               "linf_saturation", "l2_relative_pressure",
                                                               "l2_relative_saturation")],
                             "simulation_time": float(r["simulation_time"])})
    with open(os.path.join(HERE, "re2d_metrics.json"), "w") as f:
        json.dump(rows, f, indent=0)

    for solver in ("bicgstab", "gmres"):
        z = np.load(os.path.join(ref, "results3D", f"numerical_results_Test3D_{solver}_{solver}_none_mesh25.npz"),
                    allow_pickle=True)
        np.savez_compressed(os.path.join(HERE, f"test3d_{solver}.npz"),
                            iterations=z["iterations"], dt_values=z["dt_values"], times=z["times"],
                            errors=z["errors"], steps=np.array([0, 4, 9]),
                            pressure_head=z["pressure_head"][[0, 4, 9]], theta=z["theta"][[0, 4, 9]])

    meshes = {}
    mdir = os.path.join(ref, "data", "mesh")
    for n in (25, 50, 100, 200):
        meshes[f"richards/p{n}"] = digest(load_csv(os.path.join(mdir, "richards", f"p{n}.csv"), np.float64))
        meshes[f"richards/t{n}"] = digest(load_csv(os.path.join(mdir, "richards", f"t{n}.csv"), np.int64) - 1)
    meshes["richards/p_3D"] = digest(load_csv(os.path.join(mdir, "richards", "p_3D.csv"), np.float64))
    meshes["richards/t_3D"] = digest(load_csv(os.path.join(mdir, "richards", "t_3D.csv"), np.int64) - 1)
    for n in (25, 50, 100):
        meshes[f"nitrogen/p_{n}"] = digest(load_csv(os.path.join(mdir, "nitrogen", f"p_{n}.csv"), np.float64))
        meshes[f"nitrogen/t_{n}"] = digest(load_csv(os.path.join(mdir, "nitrogen", f"t_{n}.csv"), np.int64) - 1)
    with open(os.path.join(HERE, "mesh_digests.json"), "w") as f:
        json.dump(meshes, f, indent=1)

    sp = load_csv(os.path.join(mdir, "solute", "p_Pinns_25.csv"), np.float64)
    st = load_csv(os.path.join(mdir, "solute", "t_Pinns_25.csv"), np.int64) - 1
    np.savez_compressed(os.path.join(HERE, "solute_pinns25.npz"), points=sp, triangles=st)
    sp = load_csv(os.path.join(mdir, "solute", "p_Pinns_16384.csv"), np.float64)
    st = load_csv(os.path.join(mdir, "solute", "t_Pinns_16384.csv"), np.int64) - 1
    np.savez_compressed(os.path.join(HERE, "solute_pinns16384.npz"), points=sp, triangles=st.astype(np.int32))
    traces = {}
    for job in ("40115866", "40115876", "40103214", "40146207"):
        traces[job] = solute_trace(os.path.join(ref, "logs", job))
    with open(os.path.join(HERE, "solute_traces.json"), "w") as f:
        json.dump(traces, f, indent=0)
    print(f"wrote {len(rows)} CSV rows, 2 Test3D fixtures, {len(meshes)} mesh digests, SoluteTest mesh and "
          f"{len(traces)} traces")


def solute_trace(prefix):
    """Per-step lines of a SoluteTest log (tqdm prints each state twice: consecutive repeats dropped) and the
    run's summary totals."""
    import re
    err = open(prefix + ".err", errors="replace").read()
    steps = []
    for m in re.finditer(r"Time: ([0-9.]+), Error: ([0-9.e+-]+), Iterations: (\d+), dt: ([0-9.e+-]+)", err):
        rec = [m.group(1), m.group(2), int(m.group(3)), m.group(4)]
        if not steps or steps[-1] != rec:
            steps.append(rec)
    out = open(prefix + ".out", errors="replace").read()
    head = re.search(r"Solver: (\w+) with (\w+) preconditioner", out)
    mesh = re.search(r"Loading files: (\S+), (\S+) with size", out)
    tot = {k: re.search(pat, out).group(1) for k, pat in
           (("total_iterations", r"Total Iterations: (\d+)"), ("average_error", r"Average Error: ([0-9.e+-]+)"),
            ("nodes", r"Number of Nodes: (\d+)"), ("elements", r"Number of Elements: (\d+)"))}
    for k, pat in (("max_iterations", r"Max[^:]*Iterations[^:]*: (\d+)"), ("final_error", r"Final Error: ([0-9.e+-]+)")):
        m = re.search(pat, out)
        if m:
            tot[k] = m.group(1)
    return {"solver": head.group(1), "precond": head.group(2), "mesh": [mesh.group(1), mesh.group(2)],
            "steps": steps, "summary": tot}


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WSPM_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_goldens.py REFERENCE_ROOT (or set WSPM_REFERENCE_ROOT)")
    main(root)
