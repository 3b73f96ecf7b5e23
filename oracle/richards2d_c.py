"""ctypes front end of the C + OpenMP oracle (oracle/richards2d.c).

Test infrastructure, like the rest of ``oracle/``: the fixed-dt 2D Richards
time loop with van Genuchten soil and Jacobi-CG, restated in C so that the
1024^2 workload runs on all host cores in seconds per step.  It follows the
NumPy oracle (oracle/picard.py, which is pinned to the reference's goldens)
and is checked against it in tests/test_oracle_c.py.  Only tests/, smoke()
and bench.py's CPU-baseline and reference legs load it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "richards2d.c")
LIB = os.path.join(HERE, "liboracle_richards2d.so")
# the system gcc carries the OpenMP runtime (libgomp); WSPM_ORACLE_CC overrides
CC = os.environ.get("WSPM_ORACLE_CC", "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc")


def build(force=False):
    """Compile the C oracle (portable -O3, no -march: it runs on whatever host cores the box has)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    tmp = LIB + ".tmp"
    subprocess.run([CC, "-O3", "-fopenmp", "-fPIC", "-shared", "-std=c11", SRC, "-o", tmp, "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is not built (oracle.richards2d_c.build())")
        lib = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        lib.oracle_richards2d_vg_run.restype = ctypes.c_int
        lib.oracle_richards2d_vg_run.argtypes = [ctypes.c_int64, ctypes.c_int64, P, P, P, P, P, P, ctypes.c_int64,
                                                 ctypes.c_double, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.c_double, ctypes.c_int64, ctypes.c_int32,
                                                 P, P, P, P, ctypes.POINTER(ctypes.c_double)]
        lib.oracle_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def max_threads():
    return int(_load().oracle_max_threads())


def default_threads():
    """Host cores this process may use: the affinity mask, capped by a cgroup CPU quota when one is set
    (OpenMP's default would start one spinning thread per visible core even under a smaller quota)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    quota = None
    try:
        q, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]      # cgroup v2: "max 100000" or "Q P"
        if q != "max":
            quota = int(q) / int(period)
    except (OSError, ValueError):
        try:
            q = int(open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read())    # cgroup v1
            period = int(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
            if q > 0:
                quota = q / period
        except (OSError, ValueError):
            pass
    if quota is not None:
        n = max(1, min(n, int(quota)))
    return n


def run_vg_fixed_dt(points, triangles, phi, bc_nodes, bc_vals, h0, dt, n_steps, Ks_elem=None, picard_tol=1e-6,
                    picard_max=100, picard_relative=True, cg_tol=1e-8, cg_maxiter=100000, threads=0,
                    keep_steps=False):
    """Fixed-dt time loop; returns dict(h (last step), h_steps (or None), picard_its, cg_its, seconds, threads).

    ``phi`` = (alpha, theta_s, theta_r, n, m, Ks); with ``Ks_elem`` the element conductivity is
    Ks_elem[e] * K(h) with phi[5] = 1 (oracle/assembly.py:assemble_richards)."""
    lib = _load()
    pts = np.ascontiguousarray(points, dtype=np.float64)
    tri = np.ascontiguousarray(triangles, dtype=np.int64)
    n, e = pts.shape[0], tri.shape[0]
    ks = None if Ks_elem is None else np.ascontiguousarray(Ks_elem, dtype=np.float64)
    ph = np.ascontiguousarray(phi, dtype=np.float64)
    bn = np.ascontiguousarray(bc_nodes, dtype=np.int64)
    bv = np.ascontiguousarray(bc_vals, dtype=np.float64)
    h = np.array(h0, dtype=np.float64, copy=True)
    hs = np.zeros((n_steps, n)) if keep_steps else None
    pits = np.zeros(n_steps, dtype=np.int32)
    kits = np.zeros(n_steps, dtype=np.int64)
    sec = ctypes.c_double(0.0)
    threads = int(threads) if threads and threads > 0 else default_threads()
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    rc = lib.oracle_richards2d_vg_run(n, e, ptr(pts), ptr(tri), ptr(ks), ptr(ph), ptr(bn), ptr(bv), bn.size,
                                      float(dt), int(n_steps), float(picard_tol), int(picard_max),
                                      int(picard_relative), float(cg_tol), int(cg_maxiter), int(threads), ptr(h),
                                      ptr(hs), ptr(pits), ptr(kits), ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError(f"oracle_richards2d_vg_run failed ({rc})")
    return {"h": h, "h_steps": hs, "picard_its": pits, "cg_its": kits, "seconds": sec.value, "threads": threads}
