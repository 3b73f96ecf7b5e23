#!/usr/bin/env python
"""Benchmark: DOF x Picard-iterations / s of the implicit 2D Richards step on B200.

Workload (the 1024^2 configuration): unit square, 1024 x 1024 cells split into
2 P1 triangles (2,097,152 elements, 1,050,625 nodes), van Genuchten-Mualem soil
(theta_r .102, theta_s .368, alpha 3.35, n 2, m .5) with per-element
log-normal Ks (ln Ks ~ N(ln .0922, 1), seed-generated), h0 = -1, Dirichlet
h = -0.1 on the top edge, no-flux elsewhere; 20 implicit steps at dt = 1e-4;
Picard tolerance 1e-6 (relative); every linear solve to a 1e-8 relative
residual.  Two paths on the same GPU: plain FP64 Jacobi-CG and FP32 Jacobi-CG
inside FP64 iterative refinement on the true residual (the headline `value`).

A "step" is one implicit time step (a full device-resident Picard loop).  The
timed region runs K steps from the initial state after W untimed warm-up
steps; L2 is flushed (a 256 MiB write) between timed steps, outside the
events.  `--impl reference` times the CPU oracle (the NumPy/SciPy
restatement of the reference's algorithm; JAX is not installed) on a bounded
sample: one Picard iteration of the same workload per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "jax-wspm_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "DOF*Picard-iters/s at 1e-8 residual (1024^2 2D Richards, mixed FP32/FP64 refinement; FP64 alongside)"
UNIT = "DOF*Picard-iter/s"
VG_PHI_UNIT_KS = (3.35, 0.368, 0.102, 2.0, 0.5, 1.0)
KS_MEAN = 0.0922


def workload(n, seed):
    from wspm_b200 import mesh
    pts, tri = mesh.structured_triangles(n, 1.0)
    rng = np.random.default_rng(seed)
    Ks = np.exp(np.log(KS_MEAN) + 1.0 * rng.standard_normal(len(tri)))
    top = np.where(pts[:, 1] == 1.0)[0]
    return pts, tri, Ks, top


def algorithmic_bytes_cg(N, nnz, w):
    """One Jacobi-CG iteration: B_spmv + 11 N w, B_spmv = nnz (w+4) + (N+1) 4 + 2 N w."""
    return nnz * (w + 4) + (N + 1) * 4 + 2 * N * w + 11 * N * w


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for s in self.samples for j in range(4) if s[5 + j].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def allreduce_sum(v, world):
    import torch
    if world == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def allreduce_max(v, world):
    import torch
    if world == 1:
        return v
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_path(eng, h0, dt, steps, warmup, world, flush):
    """Warm up, then time `steps` steps from h0 with per-step CUDA events; returns totals."""
    import torch
    eng.set_state(h0)
    eng.dt_dev.fill_(dt)
    for _ in range(warmup):
        eng.launch_step(dt)
    torch.cuda.synchronize()
    eng.set_state(h0)
    res_buf = torch.zeros((steps, 8), dtype=torch.int32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier(world)
    for k in range(steps):
        flush()
        ev[k][0].record()
        eng.launch_step(dt)
        ev[k][1].record()
        res_buf[k].copy_(eng.result)
    barrier(world)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    r = res_buf.cpu().numpy()
    its, kits, refs, bodies = int(r[:, 1].sum()), int(r[:, 2].sum()), int(r[:, 3].sum()), r[:, 6]
    launches = sum(eng.kernel_launches(int(r[k, 1]), int(r[k, 3]), int(bodies[k])) for k in range(steps))
    return {"ms": ms, "picard_its": its, "krylov_its": kits, "refinements": refs, "status": r[:, 0].tolist(),
            "launches": launches}


def time_e2e(eng, h0, dt, steps, world, flush):
    """Same metric through the public step API with host (pinned) buffers: H2D + step + D2H per step."""
    import torch
    N = eng.dm.n_nodes
    h_host = torch.from_numpy(np.asarray(h0, dtype=np.float64)).pin_memory()
    out_host = torch.empty(N, dtype=torch.float64).pin_memory()
    res_host = torch.empty((steps, 8), dtype=torch.int32).pin_memory()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    eng.set_state(h0)
    barrier(world)
    for k in range(steps):
        flush()
        ev[k][0].record()
        src = h_host if k == 0 else out_host
        eng.h_n.copy_(src, non_blocking=True)
        eng.launch_step(dt)
        out_host.copy_(eng.h_n, non_blocking=True)
        res_host[k].copy_(eng.result, non_blocking=True)
        ev[k][1].record()
    barrier(world)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    its = int(res_host[:, 1].sum())
    return {"ms": ms, "picard_its": its, "h2d": N * 8, "d2h": N * 8 + 32}


def roofline_probe(dm, eng, fp32, reps=200, pipelined=False):
    """Average duration of one Jacobi-CG iteration of the persistent CG kernel on the assembled system
    (pipelined: the kernel of the mixed path's FP32 inner solve).

    The solve starts from x = 0 (so the residual cannot reach zero within `reps` iterations) and the kernel
    reports how many iterations it ran; a short run raises instead of being timed."""
    import ctypes
    import torch
    from wspm_b200 import _lib
    from wspm_b200._lib import check, lib
    N = dm.n_nodes
    if fp32:
        vals, dinv, b = eng.vals32, eng.dinv.float(), eng.rhs.float()
    else:
        vals, dinv, b = eng.vals, eng.dinv, eng.rhs.clone()
    x = torch.zeros_like(b)
    mode = (1 if fp32 else 0) | (2 if pipelined else 0)
    done = torch.zeros(1, dtype=torch.int32, device="cuda")
    work = torch.empty(int(lib.wspm_krylov_workspace_doubles(N, 0, 0)), dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(iters):
        x.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check("cg_iterations", lib.wspm_cg_iterations(ctypes.byref(dm.c_pat), mode, _lib.dptr(vals),
                                                       _lib.dptr(b), _lib.dptr(x), _lib.dptr(dinv), iters,
                                                       _lib.dptr(work), work.numel(), _lib.dptr(done), st))
        e1.record()
        torch.cuda.synchronize()
        if int(done.item()) != iters:
            raise RuntimeError(f"CG probe ran {int(done.item())} of {iters} iterations")
        return e0.elapsed_time(e1)
    run(20)
    t0 = min(run(0) for _ in range(3))
    tr = min(run(reps) for _ in range(3))
    return (tr - t0) / reps * 1e-3     # seconds per CG iteration


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(key):
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get(key)
    return None


def cpu_baseline(n, seed, picard_its=1):
    """Oracle (NumPy/SciPy, single thread) on one Picard iteration of the same workload."""
    from oracle import picard as opic
    pts, tri, Ks, top = workload(n, seed)
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, Ks_elem=Ks, tol=1e-8, maxiter=100000)
    _, _, theta_n = prob.model(h0)
    t0 = time.perf_counter()
    h = h0.copy()
    for _ in range(picard_its):
        A, b = prob.linear_system(h, theta_n, 1e-4)
        from oracle.krylov import solve_system
        h, _ = solve_system(A, b, h, "cg", "jacobi", tol=1e-8, maxiter=100000)
    dt = time.perf_counter() - t0
    return {"value": len(pts) * picard_its / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{picard_its} Picard iteration(s) of the {n}^2 workload (assembly + Jacobi-CG to 1e-8), "
                      f"NumPy/SciPy oracle, 1 thread, {dt:.1f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import picard as opic
    from oracle.krylov import solve_system
    pts, tri, Ks, top = workload(args.n, args.seed)
    prob, h0 = opic.vg_dirichlet_case(pts, tri, top, Ks_elem=Ks, tol=1e-8, maxiter=100000)
    _, _, theta_n = prob.model(h0)

    def one():
        A, b = prob.linear_system(h0, theta_n, 1e-4)
        solve_system(A, b, h0, "cg", "jacobi", tol=1e-8, maxiter=100000)

    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    dt = time.perf_counter() - t0
    v = len(pts) * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"2D Richards {args.n}^2 VG, per-element log-normal Ks, dt 1e-4, "
                                   "1 Picard iteration per step (bounded CPU sample)",
                       "nodes": len(pts), "elements": len(tri), "seed": args.seed},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": "one Picard iteration (assembly + Jacobi-CG to 1e-8) of the same workload "
                                       "per step; NumPy/SciPy oracle (JAX, the reference's runtime, is not "
                                       "installed), single thread"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cg_probe(args):
    """Small profiling target: one soil + assembly launch, then N iterations of the persistent CG kernel."""
    import ctypes
    import torch
    from wspm_b200 import _lib
    from wspm_b200.device import DeviceMesh, assemble_richards, merge_dirichlet, soil
    from wspm_b200.engine import default_rule
    torch.cuda.set_device(0)
    pts, tri, Ks, top = workload(args.n, args.seed)
    N = len(pts)
    dm = DeviceMesh(pts, tri)
    h = torch.full((N,), -1.0, dtype=torch.float64, device="cuda")
    C, K, th = soil("vg", h, VG_PHI_UNIT_KS)
    bc = torch.as_tensor(merge_dirichlet(N, [(top, -0.1)]), device="cuda")
    Q, W = default_rule(2)
    vals, rhs, dinv, vals32 = assemble_richards(dm, th, th, h, K, C, Q, W, 1e-4, bc_val=bc,
                                                Ks_elem=torch.as_tensor(Ks, device="cuda"), want_f32=True)
    fp32 = args.cg_probe in ("fp32", "fp32p")
    mode = (1 if fp32 else 0) | (2 if args.cg_probe == "fp32p" else 0)
    v, b, x, d = (vals32, rhs.float(), h.float(), dinv.float()) if fp32 else (vals, rhs, h.clone(), dinv)
    work = torch.empty(int(_lib.lib.wspm_krylov_workspace_doubles(N, 0, 0)), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check("cg_iterations", _lib.lib.wspm_cg_iterations(
        ctypes.byref(dm.c_pat), mode, _lib.dptr(v), _lib.dptr(b), _lib.dptr(x), _lib.dptr(d), args.probe_iters,
        _lib.dptr(work), work.numel(), None, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    print(f"cg probe {args.cg_probe}: {args.probe_iters} iterations, |x| = {float(torch.linalg.norm(x.double())):.6e}")


def ensemble_domains(n_domains, seed, sides=tuple(range(32, 257, 16))):
    """Config-3 ensemble: side lengths uniform in {32, 48, ..., 256}; VG alpha, n, Ks log-uniform in
    [1, 10], [1.3, 3], [0.01, 1]; theta_r .05, theta_s .40; h0 -1, top Dirichlet -0.1 (as the unit-square case)."""
    from wspm_b200 import mesh
    rng = np.random.default_rng(seed)
    lu = lambda lo, hi: float(np.exp(rng.uniform(np.log(lo), np.log(hi))))  # noqa: E731
    cache, doms = {}, []
    for _ in range(n_domains):
        s = int(rng.choice(sides))
        if s not in cache:
            pts, tri = mesh.structured_triangles(s, 1.0)
            bc = np.full(len(pts), np.nan)
            bc[np.abs(pts[:, 1] - 1.0) < 1e-12] = -0.1
            cache[s] = (pts, tri, bc)
        pts, tri, bc = cache[s]
        n = lu(1.3, 3.0)
        doms.append((pts, tri, (lu(1.0, 10.0), 0.40, 0.05, n, 1.0 - 1.0 / n, lu(0.01, 1.0)), bc, None))
    return doms


def run_ensemble(args):
    """Batched ensemble (one launch per step for all domains) vs one single-domain engine per domain."""
    import torch
    from wspm_b200.device import DeviceMesh
    from wspm_b200.engine import PicardEngine
    from wspm_b200.ensemble import Ensemble
    from wspm_b200.ensemble import gather_domain_results, partition_domains
    world, rank, _ = dist_setup(args)
    all_doms = ensemble_domains(args.domains, args.seed)
    # shard the independent domains over the ranks, balancing nnz (7 per node for these meshes); no collective
    # on the data path, one gather of the per-domain iteration counts at the end
    mine = partition_domains([7 * len(d[0]) for d in all_doms], world)[rank]
    doms = [all_doms[int(i)] for i in mine]
    sizes = np.array([len(d[0]) for d in doms])
    dt0, tmax = 1e-4, 1.0
    kw = dict(krylov_tol=1e-10, krylov_maxiter=2000, picard_tol=1e-6, picard_maxiter=100)
    ens = Ensemble(doms, dt0=dt0, tmax=tmax, **kw)
    ens.set_state(-1.0)
    tuned = ens.autotune()
    for _ in range(args.warmup):
        ens.step()
    its_dev = torch.zeros(len(doms), dtype=torch.int64, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    e0.record()
    for _ in range(args.steps):
        act = ens.t < tmax                      # device-side mask: no host round trip in the timed loop
        ens.launch()
        its_dev += torch.where(act, ens.its, 0)
    e1.record()
    barrier(world)
    t_batch = allreduce_max(e0.elapsed_time(e1) * 1e-3, world)
    its_b = its_dev.cpu().numpy()
    dofits = int(allreduce_sum(float((sizes * its_b).sum()), world))
    its_all = gather_domain_results(mine, its_b, len(all_doms), world)
    # sequential: one engine per domain, each advanced by the same steps
    engines, meshes = [], {}
    for pts, tri, phi, bc, _ in doms:
        if len(pts) not in meshes:
            meshes[len(pts)] = DeviceMesh(pts, tri)
        eng = PicardEngine(meshes[len(pts)], "vg", phi, bc_val=bc, solver="cg", precond="jacobi",
                           krylov_maxiter=2000, krylov_tol=1e-10, picard_tol=1e-6, picard_maxiter=100,
                           picard_relative=True)
        eng.set_state(-1.0 * np.ones(len(pts)))
        engines.append(eng)
    from wspm_b200.engine import adapt_time_step
    dts = [dt0] * len(doms)
    for _ in range(args.warmup):
        for j, eng in enumerate(engines):
            dts[j] = float(adapt_time_step(dts[j], eng.step(dts[j])["iterations"]))
    its_s = np.zeros(len(doms), dtype=np.int64)
    barrier(world)
    e0.record()
    for _ in range(args.steps):
        for j, eng in enumerate(engines):
            eng.launch_step(dts[j])
            r = eng.read_result()           # the dt rule needs the step's iterations on the host
            its_s[j] += r["iterations"]
            dts[j] = float(adapt_time_step(dts[j], r["iterations"]))
    e1.record()
    barrier(world)
    t_seq = allreduce_max(e0.elapsed_time(e1) * 1e-3, world)
    dofits_seq = allreduce_sum(float((sizes * its_s).sum()), world)
    sizes_all = np.array([len(d[0]) for d in all_doms])
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": "ensemble DOF*Picard-iter/s (batched domains, one launch per step)",
            "value": dofits / t_batch, "unit": "DOF*Picard-iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
            "data": f"synthetic (seed {args.seed})",
            "config": {"workload": f"{len(doms)} independent 2D Richards domains, sides uniform in "
                                   "{32,...,256}, VG alpha/n/Ks log-uniform, theta_r .05, theta_s .40, "
                                   "h0 -1, top Dirichlet -0.1, dt0 1e-4 adaptive per domain",
                       "nodes_total": int(sizes_all.sum()), "domains": len(all_doms),
                       "parallelism": f"domains sharded over {world} rank(s), nnz-balanced" if world > 1
                       else "single GPU"},
            "scaling": "strong",
            "batched": {"seconds": t_batch, "picard_its": int(its_all.sum()), "block_threads": tuned,
                        "cluster_size": ens.cluster_size,
                        "autotune_ms": getattr(ens, "timing", {})},
            "sequential": {"seconds": t_seq, "value": dofits_seq / t_seq},
            "speedup_vs_sequential": (dofits / t_batch) / (dofits_seq / t_seq)}
    print(json.dumps(line))


def run_adjoint(args):
    """Adjoint vs forward time on the per-element-parameter problem, and a finite-difference check."""
    print(json.dumps(adjoint_measure(args.adjoint_n, args.adjoint_steps, args.seed, args.fd_params)))


def adjoint_measure(n, steps, seed, fd_params):
    import torch
    from wspm_b200 import mesh
    from wspm_b200.adjoint import ElementParamRichards
    from wspm_b200.device import DeviceMesh
    torch.cuda.set_device(0)
    pts, tri = mesh.structured_triangles(n, 1.0)
    bc = np.full(len(pts), np.nan)
    bc[np.abs(pts[:, 1] - 1.0) < 1e-12] = -0.1
    dm = DeviceMesh(pts, tri)
    rng = np.random.default_rng(seed)
    base = np.log([0.0922, 3.35, 2.0])
    params = base[None, :] + 0.3 * rng.standard_normal((len(tri), 3))
    target_params = base[None, :] + 0.3 * rng.standard_normal((len(tri), 3))
    sensors = rng.choice(np.where(np.isnan(bc))[0], 64, replace=False)
    h0 = torch.full((len(pts),), -1.0, dtype=torch.float64, device="cuda")
    tol = dict(picard_tol=1e-12, krylov_tol=1e-13, adjoint_tol=1e-12)
    prob = ElementParamRichards(dm, 0.102, 0.368, bc, 1e-3, steps, checkpoint_every=10, **tol)
    p = torch.as_tensor(params, dtype=torch.float64, device="cuda").view(-1)
    target = prob.simulate_theta(torch.as_tensor(target_params, dtype=torch.float64, device="cuda").view(-1), h0,
                                 sensors)
    prob.forward(p, h0, sensors, target)          # warm-up
    prob.backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = prob.forward(p, h0, sensors, target)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    picard_fwd = int(sum(prob.picard_its))
    t0 = time.perf_counter()
    grad = prob.backward()
    torch.cuda.synchronize()
    t_bwd = time.perf_counter() - t0
    g = grad.cpu().numpy().ravel()
    fd = {}
    if fd_params > 0:
        idx = rng.choice(g.size, fd_params, replace=False)
        eps, errs = 1e-6, []
        scale = np.abs(g).max()
        for j in idx:
            pp, pm = p.clone(), p.clone()
            pp[j] += eps
            pm[j] -= eps
            d = (float(prob.forward(pp, h0, sensors, target)) - float(prob.forward(pm, h0, sensors, target))) / (2 * eps)
            errs.append(abs(g[j] - d) / max(abs(d), 1e-3 * scale))
        fd = {"params": int(fd_params), "step": eps, "max_rel_err": float(max(errs)),
              "median_rel_err": float(np.median(errs))}
    line = {"metric": "adjoint/forward time (discrete adjoint, per-element ln Ks, ln alpha, ln n)",
            "value": t_bwd / t_fwd, "unit": "ratio", "n_gpus": 1, "higher_is_better": False, "dtype": "f64",
            "data": f"synthetic (seed {seed})",
            "config": {"workload": f"{n}^2 P1 triangles, VG means (Ks .0922, alpha 3.35, n 2), ln-parameter "
                                   f"perturbations sigma 0.3 per element, h0 -1, top Dirichlet -0.1, {steps} steps "
                                   "at dt 1e-3, 64 theta sensors every step, target from a second draw, "
                                   "checkpoints every 10 steps", "nodes": len(pts), "elements": len(tri),
                       "parameters": 3 * len(tri), "picard_tol": 1e-12},
            "forward_s": t_fwd, "backward_s": t_bwd, "loss": float(loss), "picard_its_forward": picard_fwd,
            "fd_check": fd}
    return line


def run_config2(args):
    """3D Richards (Kuhn tetrahedra, BiCGSTAB + Jacobi) and a three-species transport chain on a 2D grid."""
    import torch
    from wspm_b200 import mesh
    from wspm_b200.device import (DeviceMesh, apply_dirichlet, assemble_adr, flux_dispersion, jacobi_dinv,
                                  krylov_solve, merge_dirichlet)
    from wspm_b200.engine import PicardEngine, default_rule
    torch.cuda.set_device(0)
    # ---- 3D Richards: unit cube, n^3 hexahedra split in 6 tets, VG c0 soil, h0 -1, top face Dirichlet -0.1
    n = args.n3d
    pts, tets = mesh.kuhn_tetrahedra(n, 1.0)
    top = np.where(np.abs(pts[:, 2] - 1.0) < 1e-12)[0]
    dm3 = DeviceMesh(pts, tets)
    eng = PicardEngine(dm3, "vg", VG_PHI_UNIT_KS, bc_val=merge_dirichlet(len(pts), [(top, -0.1)]),
                       solver="bicgstab", precond="jacobi", krylov_tol=1e-8, krylov_maxiter=1000)
    eng.host_loop = args.host_loop          # host-driven loops: the same kernels, visible to profilers
    h0 = -np.ones(len(pts))
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    t3 = time_path(eng, h0, 1e-4, args.steps3d, args.warmup, 1, lambda: flush_buf.fill_(1.0))
    # ---- transport chain on an m x m grid: species 1 -> 2 -> 3, first-order rates k1, k2, sorption on species 2,
    # dispersivities 0.5 / 0.1, Dirichlet 1.0 for species 1 on the top edge, GMRES(30) + Jacobi
    m = args.n_transport
    p2, tri = mesh.structured_triangles(m, 1.0)
    dm2 = DeviceMesh(p2, tri)
    top2 = np.where(np.abs(p2[:, 1] - 1.0) < 1e-12)[0]
    hh = torch.as_tensor(-0.5 - 0.5 * p2[:, 1], dtype=torch.float64, device="cuda")
    Q, W = default_rule(2)
    c = [torch.zeros(len(p2), dtype=torch.float64, device="cuda") for _ in range(3)]
    k1, k2, sorption = 0.36, 0.2, 1.5 * 3.5

    def transport_step():
        qx, qz, aq, Dxx, Dxz, Dzz, th = flux_dispersion(dm2, hh, VG_PHI_UNIT_KS, 0.5, 0.1, 0.0)
        up = None
        for s_, (mu, sorp, mu_up) in enumerate(((k1, 0.0, 0.0), (k2, sorption, k1), (0.0, 0.0, k2))):
            vals, rhs, dinv = assemble_adr(dm2, th, qx, qz, Dxx, Dxz, Dzz, c[s_], 1e-3, Q, W, mu=mu, sorption=sorp,
                                           mu_up=mu_up, c_up=up, lumped=True)
            if s_ == 0:
                apply_dirichlet(dm2, top2, np.ones(top2.size), vals, rhs)
            c[s_], _ = krylov_solve(dm2, vals, rhs, c[s_], "gmres", dinv=jacobi_dinv(dm2, vals), tol=1e-10,
                                    maxiter=100, restart=30)
            up = c[s_]
    for _ in range(args.warmup):
        transport_step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps3d):
        transport_step()
    e1.record()
    torch.cuda.synchronize()
    t_tr = e0.elapsed_time(e1) / args.steps3d
    line = {"metric": "3D Richards DOF*Picard-iter/s (FP64, BiCGSTAB + Jacobi) and transport-chain step time",
            "value": len(pts) * t3["picard_its"] / (t3["ms"] * 1e-3), "unit": "DOF*Picard-iter/s", "n_gpus": 1,
            "steps": args.steps3d, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": f"{n}^3 unit cube, Kuhn split (6 tets per hexahedron), VG "
                                                        "c0 soil, h0 -1, top face Dirichlet -0.1, dt 1e-4 fixed",
                                            "nodes": len(pts), "elements": len(tets), "nnz": int(dm3.pattern.nnz)},
            "richards3d": {"ms_per_step": t3["ms"] / args.steps3d, "picard_its": t3["picard_its"],
                           "krylov_its": t3["krylov_its"]},
            "transport": {"workload": f"{m}^2 triangles, 3 species first-order chain (0.36, 0.2 /day), sorption "
                                      "rho_b Kd = 5.25 on species 2, dispersivity 0.5 / 0.1, Dirichlet 1.0 inflow of "
                                      "species 1 on the top edge, lumped mass, GMRES(30) + Jacobi, dt 1e-3",
                          "nodes": len(p2), "ms_per_step": t_tr}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--inner-tol", type=float, default=1e-5,
                    help="floor of the relative tolerance of each FP32 solve in the refinement loop")
    ap.add_argument("--cg-probe", choices=["fp64", "fp32", "fp32p"], default=None,
                    help="profiling target: assemble the workload once and run --probe-iters CG iterations "
                         "through wspm_cg_iterations, then exit (no JSON line)")
    ap.add_argument("--probe-iters", type=int, default=4)
    ap.add_argument("--ensemble", action="store_true",
                    help="batched-ensemble workload (independent domains, one launch per step) against one "
                         "single-domain engine per domain; prints its own JSON line")
    ap.add_argument("--domains", type=int, default=256)
    ap.add_argument("--adjoint", action="store_true",
                    help="discrete-adjoint workload: forward and backward time, finite-difference check; prints "
                         "its own JSON line")
    ap.add_argument("--adjoint-n", type=int, default=256)
    ap.add_argument("--adjoint-steps", type=int, default=100)
    ap.add_argument("--fd-params", type=int, default=32)
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement of the main line")
    ap.add_argument("--config2", action="store_true",
                    help="3D Richards on Kuhn tetrahedra and a three-species transport chain; own JSON line")
    ap.add_argument("--n3d", type=int, default=96)
    ap.add_argument("--steps3d", type=int, default=5)
    ap.add_argument("--n-transport", type=int, default=512)
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the Picard/Krylov loops from the host (same kernels; for ncu, which cannot "
                         "profile kernels inside conditional graphs)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.cg_probe:
        return cg_probe(args)
    if args.ensemble:
        return run_ensemble(args)
    if args.adjoint:
        return run_adjoint(args)
    if args.config2:
        return run_config2(args)

    import torch
    from wspm_b200.device import DeviceMesh, merge_dirichlet
    from wspm_b200.engine import PicardEngine
    world, rank, local = dist_setup(args)
    pts, tri, Ks, top = workload(args.n, args.seed)
    N, E = len(pts), len(tri)
    dm = DeviceMesh(pts, tri, device=f"cuda:{local}")
    bc = merge_dirichlet(N, [(top, -0.1)])
    h0 = -np.ones(N)
    dt = 1e-4
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    flush = lambda: flush_buf.fill_(1.0)  # noqa: E731
    common = dict(Ks_elem=Ks, bc_val=bc, solver="cg", precond="jacobi", krylov_tol=1e-8, krylov_maxiter=20000,
                  picard_tol=1e-6, picard_maxiter=100, picard_relative=True)
    eng64 = PicardEngine(dm, "vg", VG_PHI_UNIT_KS, mixed=False, **common)
    engmx = PicardEngine(dm, "vg", VG_PHI_UNIT_KS, mixed=True, inner_tol=args.inner_tol, inner_maxiter=20000,
                         refine_maxiter=30, **common)
    eng64.host_loop = engmx.host_loop = args.host_loop
    with ClockSampler(local) as clk:
        r64 = time_path(eng64, h0, dt, args.steps, args.warmup, world, flush)
        h64 = eng64.h_n.clone()
        rmx = time_path(engmx, h0, dt, args.steps, args.warmup, world, flush)
        hmx = engmx.h_n.clone()
    e2e = time_e2e(engmx, h0, dt, args.steps, world, flush)
    # accuracy of the mixed path against FP64 and of both against the true residual
    from wspm_b200.device import spmv
    res_true = {}
    for name, eng in (("fp64", eng64), ("mixed", engmx)):
        r = eng.rhs - spmv(dm, eng.vals, eng.x)
        res_true[name] = float(torch.linalg.norm(r) / torch.linalg.norm(eng.rhs))
    rel_diff = float(torch.linalg.norm(hmx - h64) / torch.linalg.norm(h64))
    # roofline of the dominant kernels (one Jacobi-CG iteration = fused K1 + K2)
    t_it32 = roofline_probe(dm, engmx, fp32=True, pipelined=True)
    t_it64 = roofline_probe(dm, eng64, fp32=False)
    nnz = dm.pattern.nnz
    peak, peak_kind = load_peaks()
    b32 = algorithmic_bytes_cg(N, nnz, 4)
    b64 = algorithmic_bytes_cg(N, nnz, 8)
    ms64 = allreduce_max(r64["ms"], world)
    msmx = allreduce_max(rmx["ms"], world)
    mse2e = allreduce_max(e2e["ms"], world)
    if rank != 0:
        barrier(world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    v64 = world * N * r64["picard_its"] / (ms64 * 1e-3)
    vmx = world * N * rmx["picard_its"] / (msmx * 1e-3)
    ve2e = world * N * e2e["picard_its"] / (mse2e * 1e-3)
    ach32 = b32 / t_it32 / 1e9
    ach64 = b64 / t_it64 / 1e9
    line = {
        "metric": METRIC, "value": vmx, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": msmx / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 Krylov + f64 refinement/assembly", "data": "synthetic (seeded log-normal Ks)",
        "config": {"workload": f"2D Richards {args.n}^2 P1 triangles, VG soil, per-element log-normal Ks "
                               f"(sigma_lnK 1, seed {args.seed}), h0 -1, top Dirichlet -0.1, dt 1e-4 fixed, "
                               f"{args.steps} steps from the initial state",
                   "nodes": N, "elements": E, "nnz": nnz, "picard_tol": 1e-6, "krylov_residual": 1e-8,
                   "l2_policy": "L2 flushed (256 MiB write) between timed steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "loop_control": "host" if args.host_loop else "device (CUDA graph conditional nodes)"},
        "fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "picard_its": r64["picard_its"],
                 "krylov_its": r64["krylov_its"], "true_rel_residual": res_true["fp64"]},
        "mixed": {"value": vmx, "picard_its": rmx["picard_its"], "inner_krylov_its": rmx["krylov_its"],
                  "refinements": rmx["refinements"], "true_rel_residual": res_true["mixed"],
                  "rel_diff_vs_fp64": rel_diff, "speedup_vs_fp64": vmx / v64},
        "status": {"fp64": r64["status"], "mixed": rmx["status"]},
        "e2e": {"value": ve2e, "unit": UNIT, "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "gpu_launches": rmx["launches"] + r64["launches"],
        "roofline": {"bound": "hbm", "kernel": "one FP32 Jacobi-CG iteration of the resident pipelined CG kernel (mixed path inner solve)",
                     "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak, "peak_kind": peak_kind,
                     "traffic": load_traffic("cg_iteration_f32"), "algorithmic_bytes": b32,
                     "seconds_per_iteration": t_it32,
                     "fp64": {"achieved": ach64, "frac": ach64 / peak, "algorithmic_bytes": b64,
                              "seconds_per_iteration": t_it64, "traffic": load_traffic("cg_iteration_f64")}},
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args.n, args.seed)
    if world == 1 and not args.no_adjoint:
        # second part of the metric: adjoint / forward time of the per-element-parameter run
        a = adjoint_measure(args.adjoint_n, args.adjoint_steps, args.seed, 0)
        line["adjoint"] = {"adjoint_over_forward": a["value"], "forward_s": a["forward_s"],
                           "backward_s": a["backward_s"], "workload": a["config"]["workload"],
                           "parameters": a["config"]["parameters"]}
    print(json.dumps(line))
    barrier(world)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
