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
events.  After the timed runs both GPU paths run the same K steps once more
(untimed) and every step's pressure head and theta are compared with the FP64
oracle's (the C + OpenMP restatement, oracle/richards2d.c, on all host cores;
its time for the whole workload is the CPU baseline).  `--impl reference`
times that oracle (JAX, the reference's runtime, is not installed) on the
same workload: W warm-up steps, then K time steps from the initial state.
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
    return mesh.lognormal_ks_square(n, seed, 1.0, KS_MEAN)


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
    res_f64 = torch.zeros((steps, 4), dtype=torch.float64, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier(world)
    for k in range(steps):
        flush()
        ev[k][0].record()
        eng.launch_step(dt)
        ev[k][1].record()
        res_buf[k].copy_(eng.result)
        res_f64[k].copy_(eng.result_f64)
    barrier(world)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    r = res_buf.cpu().numpy()
    its, kits, refs, bodies = int(r[:, 1].sum()), int(r[:, 2].sum()), int(r[:, 3].sum()), r[:, 6]
    launches = sum(eng.kernel_launches(int(r[k, 1]), int(r[k, 3]), int(bodies[k])) for k in range(steps))
    # seconds the resident CG kernels ran inside the timed steps (their own %globaltimer: a kernel node
    # inside a graph cannot be bracketed by CUDA events)
    krylov_s = float(res_f64[:, 1].sum().item())
    return {"ms": ms, "picard_its": its, "krylov_its": kits, "refinements": refs, "status": r[:, 0].tolist(),
            "launches": launches, "krylov_kernel_s": krylov_s}


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


def l2_read_bandwidth(nbytes, reps=(40, 200)):
    """Streaming-read bandwidth (GB/s) of a buffer of `nbytes` bytes (wspm_read_probe, 16-byte loads that bypass
    L1, each block its own contiguous share): the difference of two launches with different pass counts, timed
    with CUDA events, so the launch and the first (cold) pass cancel.  Best of three."""
    import ctypes
    import torch
    from wspm_b200 import _lib
    from wspm_b200._lib import check, lib
    n16 = max(1, int(nbytes) // 16)
    buf = torch.ones(4 * n16, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(r):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check("read_probe", lib.wspm_read_probe(_lib.dptr(buf), n16, r, 2, _lib.dptr(out), st))
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3
    run(reps[0])
    best = 0.0
    for _ in range(3):
        t0, t1 = run(reps[0]), run(reps[1])
        best = max(best, (reps[1] - reps[0]) * n16 * 16 / (t1 - t0) / 1e9)
    return best


def assembly_seconds(eng, reps=20):
    """Average duration (CUDA events) of one assembly of the plan's current system with the kernel its step runs
    (wspm_picard_assemble: rows, Dirichlet rows, Jacobi 1/diag; the element-shape path when the plan found few
    element shapes)."""
    import torch
    eng.assemble()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        eng.assemble()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / reps


def spmv_seconds(dm, vals, x, copies=4, reps=40):
    """Average duration of the stand-alone FP64 SpMV (wspm_spmv_f64) on the step's matrix: `reps` back-to-back
    launches cycling over `copies` copies of the matrix and both vectors (4 x 75.6 MB at 1024^2, more than twice
    the 126 MB L2, so every launch reads its operands from DRAM), one CUDA-event pair around all of them."""
    import torch
    from wspm_b200.device import spmv
    ops = [(vals.clone(), x.clone(), torch.empty_like(x)) for _ in range(copies)]
    for v, xx, y in ops:
        y.copy_(spmv(dm, v, xx))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for r in range(reps):
        v, xx, _ = ops[r % copies]
        spmv(dm, v, xx)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / reps


def assembly_public_seconds(eng, dm, reps=20):
    """The same through the plan-free entry point (wspm_assemble_richards), which recomputes every element's
    geometry (Ks gathered by element id, FP32 copy written)."""
    import torch
    from wspm_b200.device import assemble_richards, soil
    from wspm_b200.engine import default_rule
    C, K, th = soil("vg", eng.h_n, VG_PHI_UNIT_KS)
    Q, W = default_rule(2)
    args = (dm, th, th, eng.h_n, K, C, Q, W, 1e-4)
    kw = dict(bc_val=eng.bc_val, Ks_elem=eng.Ks_elem, want_f32=True)
    assemble_richards(*args, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        assemble_richards(*args, **kw)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / reps


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


def host_cores():
    """Host cores this process may use (affinity mask capped by a cgroup CPU quota)."""
    from oracle import richards2d_c
    return richards2d_c.default_threads()


def oracle_run(n, seed, steps, keep_steps=False, threads=None):
    """The FP64 oracle (C + OpenMP restatement, oracle/richards2d.c) on the same workload: `steps` fixed-dt
    steps from h0; returns the oracle's result dict (h per step when keep_steps, Picard/CG iterations, seconds
    of the time loop, threads)."""
    from oracle import picard as opic, richards2d_c
    richards2d_c.build()
    pts, tri, Ks, top = workload(n, seed)
    nodes, vals = opic.dirichlet_arrays(len(pts), [(top, -0.1)])
    out = richards2d_c.run_vg_fixed_dt(pts, tri, VG_PHI_UNIT_KS, nodes, vals, -np.ones(len(pts)), 1e-4, steps,
                                       Ks_elem=Ks, picard_tol=1e-6, picard_max=100, picard_relative=True,
                                       cg_tol=1e-8, cg_maxiter=100000, threads=threads or host_cores(),
                                       keep_steps=keep_steps)
    out["nodes"] = len(pts)
    return out


def cpu_baseline_from(ref, n, steps):
    v = ref["nodes"] * int(ref["picard_its"].sum()) / ref["seconds"]
    return {"value": v, "unit": UNIT, "cores": int(ref["threads"]), "kind": "port",
            "sample": f"the whole workload: {steps} steps of the {n}^2 case ({int(ref['picard_its'].sum())} Picard "
                      f"iterations, {int(ref['cg_its'].sum())} Jacobi-CG iterations to 1e-8), FP64 oracle "
                      f"restated in C + OpenMP (oracle/richards2d.c), {int(ref['threads'])} threads, "
                      f"{ref['seconds']:.1f} s (JAX, the reference's runtime, is not installed)"}


def parity_vs_oracle(ref, runs):
    """Max over steps of the relative L2 error of pressure head and theta against the oracle, per GPU path."""
    from oracle import soil as osoil
    th_ref = [osoil.van_genuchten_model(h, VG_PHI_UNIT_KS)[2] for h in ref["h_steps"]]
    out = {}
    for name, res in runs.items():
        eh = max(float(np.linalg.norm(res["pressure_head"][s] - ref["h_steps"][s]) / np.linalg.norm(ref["h_steps"][s]))
                 for s in range(len(th_ref)))
        et = max(float(np.linalg.norm(res["theta"][s] - th_ref[s]) / np.linalg.norm(th_ref[s]))
                 for s in range(len(th_ref)))
        out[name] = {"h_rel_err": eh, "theta_rel_err": et,
                     "picard_its_equal": bool(np.array_equal(res["iterations"], ref["picard_its"]))}
    return out


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = host_cores()
    oracle_run(args.n, args.seed, max(1, args.warmup), threads=cores)       # warm-up (not timed)
    ref = oracle_run(args.n, args.seed, args.steps, threads=cores)
    its = int(ref["picard_its"].sum())
    v = ref["nodes"] * its / ref["seconds"]
    cb = cpu_baseline_from(ref, args.n, args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref["seconds"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded log-normal Ks)",
            "config": workload_config(args),
            "picard_its": its, "krylov_its": int(ref["cg_its"].sum()),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def workload_config(args, world=1, host_loop=False):
    return {"workload": f"2D Richards {args.n}^2 P1 triangles, VG soil, per-element log-normal Ks "
                        f"(sigma_lnK 1, seed {args.seed}), h0 -1, top Dirichlet -0.1, dt 1e-4 fixed, "
                        f"{args.steps} steps from the initial state",
            "nodes": (args.n + 1) ** 2, "elements": 2 * args.n * args.n, "picard_tol": 1e-6,
            "krylov_residual": 1e-8, "l2_policy": "L2 flushed (256 MiB write) between timed steps",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "loop_control": "host" if host_loop else "device (CUDA graph conditional nodes)"}


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


def ensemble_domains(n_domains, seed):
    """Config-3 ensemble (wspm_b200.mesh.vg_parameter_ensemble): sides uniform in {32, 48, ..., 256}; VG alpha, n,
    Ks log-uniform in [1, 10], [1.3, 3], [0.01, 1]; theta_r .05, theta_s .40; h0 -1, top Dirichlet -0.1."""
    from wspm_b200 import mesh
    return mesh.vg_parameter_ensemble(n_domains, seed)


def run_ensemble(args):
    """Batched ensemble (one launch per step for all domains) vs one single-domain engine per domain."""
    world, rank, _ = dist_setup(args)
    line = ensemble_measure(args.domains, args.steps, args.warmup, args.seed, world, rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def ensemble_measure(n_domains, steps, warmup, seed, world=1, rank=0):
    import torch
    from wspm_b200.device import DeviceMesh
    from wspm_b200.engine import PicardEngine
    from wspm_b200.ensemble import Ensemble
    from wspm_b200.ensemble import gather_domain_results, partition_domains

    class _A:
        pass
    args = _A()
    args.domains, args.steps, args.warmup, args.seed = n_domains, steps, warmup, seed
    all_doms = ensemble_domains(args.domains, args.seed)
    # shard the independent domains over the ranks, balancing nnz (7 per node for these meshes); no collective
    # on the data path, one gather of the per-domain iteration counts at the end
    mine = partition_domains([7 * len(d[0]) for d in all_doms], world)[rank]
    doms = [all_doms[int(i)] for i in mine]
    sizes = np.array([len(d[0]) for d in doms])
    # start-up: the pattern of the block-diagonal union mesh, host builder vs device builder
    from wspm_b200.pattern import Pattern
    off = np.concatenate([[0], np.cumsum(sizes)])
    union = np.concatenate([d[1] + off[i] for i, d in enumerate(doms)])
    t0 = time.perf_counter()
    Pattern(union, int(off[-1]), layout="sell", builder="native")
    t_host = time.perf_counter() - t0
    Pattern(union, int(off[-1]), layout="sell", builder="device")      # warm (module load, first allocations)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Pattern(union, int(off[-1]), layout="sell", builder="device")
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    dt0, tmax = 1e-4, 1.0
    kw = dict(krylov_tol=1e-10, krylov_maxiter=2000, picard_tol=1e-6, picard_maxiter=100)
    ens = Ensemble(doms, dt0=dt0, tmax=tmax, **kw)
    ens.set_state(-1.0)
    tuned = ens.autotune()
    for _ in range(args.warmup):
        ens.step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    e0.record()
    # the time loop on the device: one CUDA graph, a WHILE node over the step launches
    its_dev, _ = ens.run_device(args.steps)
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
                        "loop": "on the device (one CUDA graph with a WHILE node over the steps)",
                        "cluster_size": ens.cluster_size,
                        "autotune_ms": getattr(ens, "timing", {})},
            "sequential": {"seconds": t_seq, "value": dofits_seq / t_seq},
            "speedup_vs_sequential": (dofits / t_batch) / (dofits_seq / t_seq),
            "startup_pattern": {"nodes": int(off[-1]), "elements": int(len(union)), "host_builder_s": t_host,
                                "device_builder_s": t_dev, "note": "device time includes copying the arrays back "
                                                                   "to host NumPy (the Pattern object keeps both)"}}
    return line


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


def config2_measure(n3d, steps, warmup, n_transport, host_loop=False):
    """3D Richards (Kuhn tetrahedra, BiCGSTAB + Jacobi) and the three-species transport chain (GMRES(30) + Jacobi),
    each in plain FP64 and in mixed precision (FP32 corrections of the same solver inside FP64 refinement)."""
    import torch
    from wspm_b200 import mesh
    from wspm_b200.device import (DeviceMesh, apply_dirichlet, assemble_adr, flux_dispersion, jacobi_dinv,
                                  krylov_solve, krylov_solve_mixed, merge_dirichlet, spmv)
    from wspm_b200.engine import PicardEngine, default_rule
    torch.cuda.set_device(0)
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    flush = lambda: flush_buf.fill_(1.0)  # noqa: E731
    # ---- 3D Richards: unit cube, n^3 hexahedra split in 6 tets, VG c0 soil, h0 -1, top face Dirichlet -0.1
    n = n3d
    pts, tets = mesh.kuhn_tetrahedra(n, 1.0)
    top = np.where(np.abs(pts[:, 2] - 1.0) < 1e-12)[0]
    dm3 = DeviceMesh(pts, tets)
    h0 = -np.ones(len(pts))
    r3, fields = {}, {}
    for name, mixed in (("fp64", False), ("mixed", True)):
        eng = PicardEngine(dm3, "vg", VG_PHI_UNIT_KS, bc_val=merge_dirichlet(len(pts), [(top, -0.1)]),
                           solver="bicgstab", precond="jacobi", krylov_tol=1e-8, krylov_maxiter=1000, mixed=mixed,
                           inner_tol=1e-5, inner_maxiter=1000, refine_maxiter=30)
        eng.host_loop = host_loop          # host-driven loops: the same kernels, visible to profilers
        t = time_path(eng, h0, 1e-4, steps, warmup, 1, flush)
        res = eng.rhs - spmv(dm3, eng.vals, eng.x)
        r3[name] = {"ms_per_step": t["ms"] / steps, "picard_its": t["picard_its"], "krylov_its": t["krylov_its"],
                    "value": len(pts) * t["picard_its"] / (t["ms"] * 1e-3),
                    "true_rel_residual": float(torch.linalg.norm(res) / torch.linalg.norm(eng.rhs))}
        if mixed:
            r3[name]["refinements"] = t["refinements"]
        else:
            # the 3D assembly as the FP64 step runs it, against the HBM roof (the 2D convention for tetrahedra:
            # conn E*16 + coords N*24 + two nodal fields + values + rhs + 1/diag)
            t_a = assembly_seconds(eng)
            E3, N3, nnz3 = len(tets), len(pts), dm3.pattern.nnz
            b_a = E3 * 16 + N3 * 24 + 2 * N3 * 8 + nnz3 * 8 + N3 * 8 + N3 * 8
            peak, _ = load_peaks()
            r3["assembly"] = {"kernel": "richards_rows_kernel<3> as the FP64 step runs it", "seconds": t_a,
                              "algorithmic_bytes": b_a, "achieved": b_a / t_a / 1e9, "peak": peak,
                              "frac": b_a / t_a / 1e9 / peak, "element_shapes": eng.element_shape_count()}
            if r3["assembly"]["element_shapes"] == 0:
                r3["assembly"]["note"] = ("the grid's coordinates (i/n) are not binary fractions for this n: its "
                                          "element Jacobians differ bitwise and the assembly recomputes each "
                                          "element's geometry")
        fields[name] = eng.h_n.clone()
        del eng
    r3["mixed"]["rel_diff_vs_fp64"] = float(torch.linalg.norm(fields["mixed"] - fields["fp64"]) /
                                            torch.linalg.norm(fields["fp64"]))
    r3["mixed"]["speedup_vs_fp64"] = r3["mixed"]["value"] / r3["fp64"]["value"]
    # ---- transport chain on an m x m grid: species 1 -> 2 -> 3, first-order rates k1, k2, sorption on species 2,
    # dispersivities 0.5 / 0.1, Dirichlet 1.0 for species 1 on the top edge, GMRES(30) + Jacobi
    m = n_transport
    p2, tri = mesh.structured_triangles(m, 1.0)
    dm2 = DeviceMesh(p2, tri)
    top2 = np.where(np.abs(p2[:, 1] - 1.0) < 1e-12)[0]
    hh = torch.as_tensor(-0.5 - 0.5 * p2[:, 1], dtype=torch.float64, device="cuda")
    Q, W = default_rule(2)
    k1, k2, sorption = 0.36, 0.2, 1.5 * 3.5
    rt, conc = {}, {}
    for name in ("fp64", "mixed"):
        c = [torch.zeros(len(p2), dtype=torch.float64, device="cuda") for _ in range(3)]
        stats = {"krylov": 0, "refinements": 0}

        def transport_step():
            qx, qz, aq, Dxx, Dxz, Dzz, th = flux_dispersion(dm2, hh, VG_PHI_UNIT_KS, 0.5, 0.1, 0.0)
            up = None
            for s_, (mu, sorp, mu_up) in enumerate(((k1, 0.0, 0.0), (k2, sorption, k1), (0.0, 0.0, k2))):
                vals, rhs, dinv = assemble_adr(dm2, th, qx, qz, Dxx, Dxz, Dzz, c[s_], 1e-3, Q, W, mu=mu,
                                               sorption=sorp, mu_up=mu_up, c_up=up, lumped=True)
                if s_ == 0:
                    apply_dirichlet(dm2, top2, np.ones(top2.size), vals, rhs)
                dinv = jacobi_dinv(dm2, vals)
                if name == "fp64":
                    c[s_], _ = krylov_solve(dm2, vals, rhs, c[s_], "gmres", dinv=dinv, tol=1e-10, maxiter=100,
                                            restart=30)
                else:
                    c[s_], _ = krylov_solve_mixed(dm2, vals, rhs, c[s_], dinv=dinv, tol=1e-10, inner_tol=1e-5,
                                                  inner_maxiter=100, refine_maxiter=30, solver="gmres", restart=30)
                up = c[s_]
        for _ in range(warmup):
            transport_step()
        for s_ in range(3):
            c[s_].zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            transport_step()
        e1.record()
        torch.cuda.synchronize()
        rt[name] = {"ms_per_step": e0.elapsed_time(e1) / steps}
        conc[name] = torch.cat(c)
    rt["mixed"]["rel_diff_vs_fp64"] = float(torch.linalg.norm(conc["mixed"] - conc["fp64"]) /
                                            torch.linalg.norm(conc["fp64"]))
    rt["mixed"]["speedup_vs_fp64"] = rt["fp64"]["ms_per_step"] / rt["mixed"]["ms_per_step"]
    return {"richards3d": dict(workload=f"{n}^3 unit cube, Kuhn split (6 tets per hexahedron), VG c0 soil, h0 -1, "
                                        f"top face Dirichlet -0.1, dt 1e-4 fixed, BiCGSTAB + Jacobi to 1e-8, "
                                        f"{steps} steps", nodes=len(pts), elements=len(tets),
                               nnz=int(dm3.pattern.nnz), **r3),
            "transport": dict(workload=f"{m}^2 triangles, 3 species first-order chain (0.36, 0.2 /day), sorption "
                                       "rho_b Kd = 5.25 on species 2, dispersivity 0.5 / 0.1, Dirichlet 1.0 inflow "
                                       "of species 1 on the top edge, lumped mass, GMRES(30) + Jacobi to 1e-10 "
                                       f"(mixed: true FP64 residual), dt 1e-3, {steps} steps", nodes=len(p2), **rt)}


def run_config2(args):
    """3D Richards on Kuhn tetrahedra and a three-species transport chain, FP64 and mixed; own JSON line."""
    r = config2_measure(args.n3d, args.steps3d, args.warmup, args.n_transport, args.host_loop)
    line = {"metric": "3D Richards DOF*Picard-iter/s (BiCGSTAB + Jacobi; FP64 and mixed) and transport-chain "
                      "step time (GMRES(30); FP64 and mixed)",
            "value": r["richards3d"]["mixed"]["value"], "unit": "DOF*Picard-iter/s", "n_gpus": 1,
            "steps": args.steps3d, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64 / f32+f64",
            "data": "synthetic", "config": {"workload": r["richards3d"]["workload"]}, **r}
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
    ap.add_argument("--fd-params-main", type=int, default=8,
                    help="parameters checked by central differences in the main line's adjoint measurement")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the config-2 (3D, transport) and ensemble measurements of the main line")
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
    nnz = dm.pattern.nnz
    nd, ld = dm.pattern.n_diags, 32 * dm.pattern.n_slices
    peak_hbm, peak_kind = load_peaks()
    # ---- rooflines.  The resident CG kernels keep their vectors in shared memory and read the matrix from L2
    # every iteration: their roof is the L2 read bandwidth, measured here with a streaming-read probe over a
    # buffer the size of the matrix.  Per-iteration times are the kernels' own live durations in the timed steps.
    t_it32 = rmx["krylov_kernel_s"] / max(1, rmx["krylov_its"])
    t_it64 = r64["krylov_kernel_s"] / max(1, r64["krylov_its"])
    # L2 bytes one iteration must move: pipelined FP32 = the matrix (nd diagonals of ld rows) + 1/diag read +
    # m = M w written and read by the SpMV; FP64 = the matrix + z written and read, x read and written, 1/diag
    # (only the diagonals the plan reads: structural-zero diagonals are skipped)
    live = engmx.live_diagonals
    nd_read = bin(live).count("1") if live is not None else nd
    l2_32 = nd_read * ld * 4 + 3 * N * 4
    l2_64 = nd_read * ld * 8 + 5 * N * 8
    l2_peak32 = l2_read_bandwidth(nd * ld * 4)
    l2_peak64 = l2_read_bandwidth(nd * ld * 8)
    b32 = algorithmic_bytes_cg(N, nnz, 4)
    b64 = algorithmic_bytes_cg(N, nnz, 8)
    # the assembly is the HBM-streaming kernel of the step (algorithmic bytes per launch: connectivity,
    # coordinates, two nodal fields, per-element Ks, values, rhs and 1/diag)
    t_asm = assembly_seconds(eng64)
    t_asm_public = assembly_public_seconds(engmx, dm)
    t_spmv = spmv_seconds(dm, eng64.vals, eng64.x)
    b_spmv = nd * ld * 8 + 2 * N * 8      # every stored diagonal (the stand-alone SpMV reads all of them) + x + y
    b_asm = E * 12 + N * 16 + 2 * N * 8 + E * 8 + nnz * 8 + N * 8 + N * 8
    ms64 = allreduce_max(r64["ms"], world)
    msmx = allreduce_max(rmx["ms"], world)
    mse2e = allreduce_max(e2e["ms"], world)
    # parity: both paths again over the same steps (untimed), every step against the FP64 oracle
    parity, ref = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        runs = {name: eng.run(h0, dt, 1.0, fixed_dt=True, max_steps=args.steps)
                for name, eng in (("fp64", eng64), ("mixed", engmx))}
        ref = oracle_run(args.n, args.seed, args.steps, keep_steps=True)
        parity = parity_vs_oracle(ref, runs)
    if rank != 0:
        barrier(world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    v64 = world * N * r64["picard_its"] / (ms64 * 1e-3)
    vmx = world * N * rmx["picard_its"] / (msmx * 1e-3)
    ve2e = world * N * e2e["picard_its"] / (mse2e * 1e-3)
    ach32 = l2_32 / t_it32 / 1e9
    ach64 = l2_64 / t_it64 / 1e9
    ach_asm = b_asm / t_asm / 1e9
    line = {
        "metric": METRIC, "value": vmx, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": msmx / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 Krylov + f64 refinement/assembly", "data": "synthetic (seeded log-normal Ks)",
        "config": dict(workload_config(args, world, args.host_loop), nnz=nnz),
        "fp64": {"value": v64, "ms_per_step": ms64 / args.steps, "picard_its": r64["picard_its"],
                 "krylov_its": r64["krylov_its"], "true_rel_residual": res_true["fp64"],
                 "cg_kernel_share": r64["krylov_kernel_s"] / (ms64 * 1e-3)},
        "mixed": {"value": vmx, "picard_its": rmx["picard_its"], "inner_krylov_its": rmx["krylov_its"],
                  "refinements": rmx["refinements"], "true_rel_residual": res_true["mixed"],
                  "rel_diff_vs_fp64": rel_diff, "speedup_vs_fp64": vmx / v64,
                  "cg_kernel_share": rmx["krylov_kernel_s"] / (msmx * 1e-3)},
        "status": {"fp64": r64["status"], "mixed": rmx["status"]},
        "e2e": {"value": ve2e, "unit": UNIT, "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]},
        "gpu_launches": rmx["launches"] + r64["launches"],
        "roofline": {"bound": "l2",
                     "kernel": "pcg_resident_kernel: FP32 pipelined Jacobi-CG, the mixed path's inner solve "
                               "(vectors in shared memory, matrix read from L2 every iteration)",
                     "achieved": ach32, "peak": l2_peak32, "unit": "GB/s", "frac": ach32 / l2_peak32,
                     "peak_kind": "measured in this run: wspm_read_probe, 16-byte L1-bypassing reads over a "
                                  "buffer the size of the FP32 matrix, CUDA events",
                     "l2_bytes_per_iteration": l2_32, "seconds_per_iteration": t_it32,
                     "diagonals_read": f"{nd_read} of {nd} (the others are structural zeros, skipped)",
                     "timing": "the kernel's own %globaltimer entry-to-exit durations summed over the timed "
                               "steps / inner iterations",
                     "traffic": load_traffic("cg_iteration_f32"),
                     "hbm_convention": {"bytes_per_iteration": b32, "achieved": b32 / t_it32 / 1e9,
                                        "peak": peak_hbm, "frac": b32 / t_it32 / 1e9 / peak_hbm,
                                        "note": "B_spmv + 11 N w counted as HBM bytes; the kernel moves almost "
                                                "none of them from HBM (traffic)"},
                     "fp64": {"kernel": "cg_resident_kernel (FP64 single-reduction Jacobi-CG)", "bound": "l2",
                              "achieved": ach64, "peak": l2_peak64, "frac": ach64 / l2_peak64,
                              "l2_bytes_per_iteration": l2_64, "seconds_per_iteration": t_it64,
                              "traffic": load_traffic("cg_iteration_f64"),
                              "hbm_convention": {"bytes_per_iteration": b64, "frac": b64 / t_it64 / 1e9 / peak_hbm}},
                     "assembly": {"kernel": "richards_rows_kernel as the FP64 step runs it (rows, Dirichlet, "
                                            "1/diag; geometric factors from the plan's element-shape table)",
                                  "bound": "hbm", "achieved": ach_asm, "peak": peak_hbm, "frac": ach_asm / peak_hbm,
                                  "peak_kind": peak_kind, "algorithmic_bytes": b_asm, "seconds": t_asm,
                                  "element_shapes": eng64.element_shape_count(),
                                  "recomputing_geometry": {"entry": "wspm_assemble_richards (no plan; FP32 copy "
                                                                    "written)", "seconds": t_asm_public,
                                                           "frac": b_asm / t_asm_public / 1e9 / peak_hbm}},
                     "spmv": {"kernel": "spmv_kernel (wspm_spmv_f64, DIA, FP64) on the step's matrix",
                              "bound": "hbm", "bytes": b_spmv, "seconds": t_spmv,
                              "achieved": b_spmv / t_spmv / 1e9, "peak": peak_hbm,
                              "frac": b_spmv / t_spmv / 1e9 / peak_hbm,
                              "l2_policy": "40 back-to-back launches over 4 copies of matrix and vectors "
                                           "(4 x 75.6 MB > L2), one CUDA-event pair"}},
        "clocks": clk.summary(),
    }
    if parity is not None:
        line["fp64_err_vs_oracle"] = parity["fp64"]["h_rel_err"]
        line["mixed_err_vs_oracle"] = parity["mixed"]["h_rel_err"]
        line["parity"] = {"oracle": f"FP64 oracle, C + OpenMP restatement (oracle/richards2d.c), "
                                    f"{int(ref['threads'])} threads", "steps": args.steps,
                          "measure": "max over steps of ||x_gpu - x_oracle|| / ||x_oracle||", **parity}
        line["cpu_baseline"] = cpu_baseline_from(ref, args.n, args.steps)
    if world == 1 and not args.no_adjoint:
        # second part of the metric: adjoint / forward time of the per-element-parameter run, with a
        # central-difference check of the gradient on a sample of the parameters
        a = adjoint_measure(args.adjoint_n, args.adjoint_steps, args.seed, args.fd_params_main)
        line["adjoint"] = {"adjoint_over_forward": a["value"], "forward_s": a["forward_s"],
                           "backward_s": a["backward_s"], "workload": a["config"]["workload"],
                           "parameters": a["config"]["parameters"], "fd_check": a["fd_check"]}
    if world == 1 and not args.no_extras:
        # the other configurations, bounded: 3D Richards and the transport chain in both precisions, and the
        # batched ensemble against sequential single-domain solves
        line["config2"] = config2_measure(args.n3d, 3, 2, args.n_transport)
        e = ensemble_measure(args.domains, 3, 2, args.seed)
        line["ensemble"] = {"workload": e["config"]["workload"], "domains": e["config"]["domains"],
                            "nodes_total": e["config"]["nodes_total"], "steps": 3,
                            "batched": e["batched"], "sequential": e["sequential"],
                            "batched_value": e["value"], "speedup_vs_sequential": e["speedup_vs_sequential"],
                            "startup_pattern": e["startup_pattern"]}
    print(json.dumps(line))
    barrier(world)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
