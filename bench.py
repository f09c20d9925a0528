"""Benchmark: Total-FETI dual solve time to 1e-8 on one B200 (per rank), through FETI4I.

Workload (default): heat conduction on a unit cube, 8x8x8 subdomains x 10x10x10 HEXA8
elements, log-uniform per-element conductivity on [1,100] (seed 0), T=0 on z=0,
unit source; lumped preconditioner; Schur complements stored in FP32 inside FP64
residual replacement (reliable updates); dual PCG to precision 1e-8.

One step = one dual PCG solve on device-resident data (FETI4ISolveResident).
``e2e`` = one FETI4ISolve call with host buffers (H2D right-hand side, device K+ f,
b, e, PCG, device primal recovery, D2H solution).  ``roofline`` is the tile SYMV
(F apply) kernel: algorithmic bytes per launch / CUDA-event launch time on the
library stream.  ``parity`` states the error of every solution the line times
against the oracle's FP64 solve and the primal residual on the assembled system.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FETI solve time @1e-8 rel err, mixed/batched vs FP64 GPU; F-apply HBM GB/s"
SCHUR = {"fp64": 0, "fp32": 1, "bf16": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2_heat_512")
    ap.add_argument("--schur", default="fp32", choices=sorted(SCHUR))
    ap.add_argument("--precond", type=int, default=1)
    ap.add_argument("--precision", type=float, default=1e-8)
    ap.add_argument("--tile-kernel", type=int, default=-1,
                    help="-1 autotuned (default), 0 register prefetch, 1 TMA bulk pipeline")
    ap.add_argument("--delta", type=float, default=0.003, help="residual replacement threshold")
    ap.add_argument("--nrhs", type=int, default=32, help="load cases of the batched (multi-RHS) leg, 0 to skip")
    ap.add_argument("--method", type=int, default=0, choices=[0, 1],
                    help="FETI_METHOD: 0 Total FETI, 1 Hybrid Total FETI on the config's clusters")
    ap.add_argument("--loads", default="traction", choices=["scaled", "traction"],
                    help="batched leg load cases: scaled copies of the config load, or seeded N(0,1e6) "
                         "nodal tractions on the x=1 face")
    ap.add_argument("--symm-tensor", type=int, default=1, choices=[0, 1],
                    help="batched leg: FP32 SYMM on the tensor cores (tcgen05, 3xTF32) instead of CUDA cores")
    ap.add_argument("--leg", default="solve", choices=["solve", "adjoint", "prep"],
                    help="adjoint: one forward + backward of the density-to-displacement map (torch.autograd); "
                         "prep: instance creation only (preprocessing times)")
    ap.add_argument("--adjoint-grid", type=int, nargs=2, default=[4, 6], metavar=("DOMAINS", "ELEMENTS"),
                    help="adjoint leg: DOMAINS^3 subdomains of ELEMENTS^3 HEXA8")
    ap.add_argument("--device-prep", type=int, default=1, choices=[0, 1],
                    help="subdomain eliminations and Schur complements on the GPU (1) or on the host (0)")
    ap.add_argument("--explicit", type=int, default=1, choices=[0, 1],
                    help="0: F applied through the subdomain K+ factors with no Schur complements stored "
                         "(FP64, single right-hand side)")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "partitioned"],
                    help="N > 1: one independent load case per GPU (replicas), or one dual problem whose "
                         "subdomains are split into blocks over the GPUs (partitioned; NCCL allreduce per apply)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.samples.append(f)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        mhz = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local, dist


def dist_max(dist, v):
    """Max over ranks (device tensor on NCCL, host tensor on gloo)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_load_case(rhs, rank):
    """The load case of one rank: rank 0 solves the workload's own right-hand side; rank r > 0 a
    seeded perturbation of it (each DOF scaled by 1 + N(0, 0.25^2), seed r).  With N GPUs the job
    is N independent load cases, one per GPU, with no exchange between the ranks."""
    if rank == 0:
        return rhs
    rng = np.random.default_rng(1000 + rank)
    return rhs * (1.0 + 0.25 * rng.standard_normal(rhs.shape))


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


def oracle_problem(P, precond):
    """The oracle (numpy restatement of ESPRESO's Total FETI) on the same mesh, and its dual PCG
    packed for the OpenMP C++ iteration (oracle/cpu_pcg.cpp) on all host cores."""
    from oracle import cpu as OC
    from oracle import feti as OF
    from oracle import numbering as ON
    num = ON.Numbering(P.elem_nodes, P.elem_domain, P.n_nodes, P.dpn, P.dirichlet)
    OP = OF.FETIProblem(num, P.elem_nodes, P.elem_domain, P.Ke, P.fe, P.coords,
                        build_dirichlet=precond in (OF.PREC_DIRICHLET, OF.PREC_SUPER_DIRICHLET))
    return OP, OC.CpuPCG(OP, precond, threads=os.cpu_count() or 1)


def oracle_u(OP, C, P, precision, f=None):
    """Displacements of the oracle's FP64 solve (global load ``f``, default the mesh's own)."""
    if f is not None:
        OP.set_rhs(f)
    lam, alpha = C.solve(precision=precision, max_it=5000)
    return OP.merge(OP.primal(lam, alpha), P.n_nodes).ravel()


def run_reference(args):
    """The reference arm: the oracle restatement of ESPRESO's FP64 CPU dual solve, timed as whole
    solves (b, e -> lambda, alpha: every PCG iteration, projector and preconditioner) over all host
    cores.  The preprocessing (factorisations, S_i, G, GG^T) is built once, untimed."""
    rank, world, local, dist = dist_init(args)
    if rank != 0:
        return
    from espreso_b200 import problems
    ncores = os.cpu_count() or 1
    P = problems.build_config(args.config)
    t0 = time.perf_counter()
    OP, C = oracle_problem(P, args.precond)
    setup_s = time.perf_counter() - t0
    b, e = OP.vec_b(), OP.vec_e()
    for _ in range(args.warmup):
        C.solve(b, e, precision=args.precision, max_it=5000)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        C.solve(b, e, precision=args.precision, max_it=5000)
        times.append((time.perf_counter() - t) * 1e3)
    ms = float(np.median(times))
    line = {"metric": METRIC, "value": ms, "unit": "ms", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.config, "precond": args.precond, "precision": args.precision,
                       "pcg_iterations": C.iterations, "setup_s": setup_s,
                       "converged": bool(C.final_norm < C.tol)},
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": ncores, "kind": "port",
                             "sample": f"one whole FP64 dual PCG solve per step ({C.iterations} iterations: packed "
                                       f"upper S_i SPMV, projector, preconditioner) by the OpenMP C++ restatement "
                                       f"of the reference's CPU solver on {ncores} threads; preprocessing untimed"},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_ours(args):
    if args.explicit == 0:
        args.schur, args.nrhs = "fp64", 0
    rank, world, local, dist = dist_init(args)
    import torch
    torch.cuda.set_device(local)
    from espreso_b200 import feti4i as F
    from espreso_b200 import problems
    t0 = time.time()
    P = problems.build_config(args.config)
    rhs = rank_load_case(P.rhs(), rank)
    inst = problems.make_instance(P, iopts={F.PRECONDITIONER: args.precond, F.VERBOSE_LEVEL: 0,
                                            F.MAX_ITERATIONS: 5000, F.FETI_METHOD: args.method},
                                  ropts={F.PRECISION: args.precision},
                                  ext={F.EXT_SCHUR_PRECISION: SCHUR[args.schur],
                                       F.EXT_TILE_KERNEL: max(0, args.tile_kernel),
                                       F.EXT_AUTOTUNE: 1 if args.tile_kernel < 0 else 0,
                                       F.EXT_RELIABLE_DELTA: args.delta,
                                       F.EXT_SYMM_TENSOR: args.symm_tensor,
                                       F.EXT_DEVICE_PREP: args.device_prep,
                                       F.EXT_SCHUR_EXPLICIT: args.explicit},
                                  clusters=P.sub_cluster() if args.method == 1 else None)
    setup_s = time.time() - t0
    st0 = inst.stats()
    sol = np.zeros(P.ndofs)
    if rank > 0:
        inst.update_rhs(rhs)
    # warm-up: full solves through the C ABI (also uploads the right-hand side)
    for _ in range(max(1, args.warmup)):
        inst.solve(sol)
    # FP64 GPU reference solve time (same config, same kernels, FP64 Schur tiles)
    inst.set_solve_precision(0)
    inst.solve_resident()
    fp64_ms = inst.solve_resident()
    st64 = inst.stats()
    inst.set_solve_precision(SCHUR[args.schur])
    inst.solve_resident()
    # timed region: K device-resident solves
    dist_barrier(dist)
    torch.cuda.synchronize()
    dev_ms = []
    with Clocks(local) as clk:
        tw = time.perf_counter()
        for _ in range(args.steps):
            dev_ms.append(inst.solve_resident())
        torch.cuda.synchronize()
        wall = (time.perf_counter() - tw) * 1e3 / args.steps
    dist_barrier(dist)
    st = inst.stats()
    step_ms = dist_max(dist, float(np.mean(dev_ms)))
    # end-to-end through FETI4ISolve with host buffers
    e2e = []
    for _ in range(max(2, args.steps // 2)):
        t = time.perf_counter()
        inst.solve(sol)
        e2e.append((time.perf_counter() - t) * 1e3)
    e2e_ms = dist_max(dist, float(np.median(e2e)))
    u_mixed, conv_mixed = sol.copy(), bool(inst.stats()["converged"])
    inst.set_solve_precision(0)
    u_fp64 = inst.solve(np.zeros(P.ndofs))
    conv_fp64 = bool(inst.stats()["converged"])
    inst.set_solve_precision(SCHUR[args.schur])
    # batched leg: nrhs seeded load cases solved together (block PCG, tile SYMM)
    batched = None
    R = U = U64 = None
    if args.nrhs > 0:
        rng = np.random.default_rng(1 + rank)
        if args.loads == "traction":
            R = problems.traction_loads(P, args.nrhs, seed=1 + rank)
        else:
            R = np.stack([rhs * rng.uniform(0.5, 2.0) for _ in range(args.nrhs)])
        inst.solve_multi(R)
        bms = [inst.solve_multi_resident(args.nrhs) for _ in range(max(1, args.steps))]
        stb = inst.stats()
        inst.set_solve_precision(0)
        U64 = inst.solve_multi(R)
        conv_b64 = bool(inst.stats()["converged"])
        b64 = inst.solve_multi_resident(args.nrhs)
        inst.set_solve_precision(SCHUR[args.schur])
        t = time.perf_counter()
        U = inst.solve_multi(R)
        e2e_b = (time.perf_counter() - t) * 1e3
        conv_b = bool(inst.stats()["converged"])
        bmed = float(np.median(bms))
        batched = {"nrhs": args.nrhs, "ms_per_batch": bmed, "ms_per_solve": bmed / args.nrhs,
                   "pcg_iterations": int(stb["iterations"]), "replacements": int(stb["replacements"]),
                   "fp64_ms_per_batch": b64, "fp64_single_ms_per_solve": fp64_ms,
                   "speedup_vs_fp64_single": fp64_ms / (bmed / args.nrhs), "e2e_ms_per_batch": e2e_b,
                   "symm": "tcgen05 3xTF32" if args.symm_tensor else "CUDA cores FP32"}
    NL = int(sum(inst.subdomain_info(d)["rows"] for d in range(int(st["subdomains"]))))
    nK = int(st["kernel_size"])
    # roofline of the F apply kernel (events on the library stream)
    t_f = inst.time_F(SCHUR[args.schur], 20)
    alg = float(st["fapply_bytes"])
    achieved = alg / (t_f * 1e-3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    traffic_src = None
    tp = os.path.join(ROOT, "profiles", "fapply_traffic.json")
    if args.explicit and os.path.exists(tp):
        tj = json.load(open(tp))
        key = f"{args.config}:{args.schur}"
        if key in tj:
            traffic = tj[key]["dram_bytes_per_launch"]
            traffic_src = tj[key]["source"]
    fp64_f = inst.time_F(0, 10)
    # parity of every solution timed above: primal residual on the assembled system (every rank) and,
    # on rank 0 at N=1, the error against the oracle's FP64 solve of the same mesh and loads
    parity = {"precision": args.precision,
              "mixed": {"residual": P.relative_residual(u_mixed, rhs), "converged": conv_mixed},
              "fp64": {"residual": P.relative_residual(u_fp64, rhs), "converged": conv_fp64}}
    if U is not None:
        parity["batched"] = {"residual_max": max(P.relative_residual(U[j], R[j]) for j in range(len(R))),
                             "converged": conv_b,
                             "fp64_residual_max": max(P.relative_residual(U64[j], R[j]) for j in range(len(R))),
                             "fp64_converged": conv_b64}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, uo, ucols = cpu_baseline_and_oracle(P, args, R)
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        parity["mixed"]["err_vs_oracle"] = rel(u_mixed, uo)
        parity["fp64"]["err_vs_oracle"] = rel(u_fp64, uo)
        if U is not None:
            parity["batched"]["err_vs_oracle"] = {str(j): rel(U[j], uc) for j, uc in ucols.items()}
            parity["batched"]["fp64_err_vs_oracle"] = {str(j): rel(U64[j], uc) for j, uc in ucols.items()}
        parity["oracle"] = (f"oracle FP64 Total-FETI solve of the same mesh and loads (own factorisations and "
                            f"S_i, OpenMP C++ PCG) to precision {ORACLE_PRECISION:g}; batched columns "
                            f"{sorted(ucols)} checked")
        errs = [parity["mixed"]["err_vs_oracle"], parity["fp64"]["err_vs_oracle"]]
        if U is not None:
            errs += list(parity["batched"]["err_vs_oracle"].values())
            errs += list(parity["batched"]["fp64_err_vs_oracle"].values())
        convs = [conv_mixed, conv_fp64] + ([conv_b, conv_b64] if U is not None else [])
        parity["max_err_vs_oracle"] = max(errs)
        parity["ok"] = bool(max(errs) <= args.precision and all(convs))
        if not parity["ok"]:
            print(f"PARITY FAILURE: max error vs oracle {max(errs):.3e}, converged {convs}", file=sys.stderr)
    clocks = clk.summary()
    launches = int(st["kernel_launches"]) * args.steps
    line = {
        "metric": METRIC, "value": step_ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (fp32 Schur storage)" if args.schur == "fp32" else
        ("f64 (bf16 Schur storage)" if args.schur == "bf16" else "f64"),
        "data": "synthetic",
        "config": {"workload": args.config, "subdomains": int(st["subdomains"]), "dual_size": int(st["dual_size"]),
                   "kernel_size": nK, "precond": args.precond, "schur": args.schur, "precision": args.precision,
                   "pcg_iterations": int(st["iterations"]), "replacements": int(st["replacements"]),
                   "method": ["TOTAL_FETI", "HYBRID_FETI"][args.method], "loads": args.loads,
                   "parallelism": f"load-cases{world}",
                   "l2": (f"working set > L2 (Schur tiles {alg / 1e9:.2f} GB per apply, 126 MB L2)" if alg > 126e6
                          else f"working set {alg / 1e6:.0f} MB fits in the 126 MB L2 (no flush)"),
                   "wall_ms_per_step": wall,
                   "setup_s": setup_s, "prep_s": st0["prep_seconds"],
                   "prep": ("device" if args.device_prep else "host"),
                   "prep_device_ms": st0["prep_device_ms"],
                   "prep_device_tflops": (st0["prep_device_flops"] / st0["prep_device_ms"] * 1e-9
                                          if st0["prep_device_ms"] > 0 else None),
                   "tuning": inst.tuning(),
                   "kplus_tiles_applied": st0["kplus_tiles"],
                   "reliable_delta": args.delta,
                   "f_apply": "explicit S_i tiles" if args.explicit else "implicit through the K+ factors",
                   "device_bytes": st["device_bytes"]},
        "fp64_gpu": {"ms": fp64_ms, "pcg_iterations": int(st64["iterations"]), "speedup_mixed": fp64_ms / step_ms,
                     "fapply_ms": fp64_f},
        "solves_per_s": world * 1e3 / step_ms,
        "batched": batched,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(rhs.nbytes),
                "d2h_bytes_per_step": int(sol.nbytes)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "kernel": "tile_symv_kernel" if args.explicit else "kplus_dual_kernel",
                     "launch_ms": t_f, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg},
        "cpu_baseline": cpu,
        "parity": parity,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line))
    inst.destroy()
    if dist is not None:
        dist.destroy_process_group()


ORACLE_PRECISION = 1e-11


def run_partitioned(args):
    """One dual problem split over the ranks: rank r prepares the r-th contiguous block of the
    subdomains on its GPU; the PCG runs replicated with one NCCL allreduce of the dual vector per F
    apply and per preconditioner apply (espreso_b200.partitioned).  Total work is fixed: strong scaling."""
    rank, world, local, dist = dist_init(args)
    import torch
    torch.cuda.set_device(local)
    from espreso_b200 import feti4i as F
    from espreso_b200 import problems
    from espreso_b200.partitioned import LibraryBlock, PartitionedSolver, owned_range
    P = problems.build_config(args.config)
    nsub = int(P.elem_domain.max()) + 1
    first, count = owned_range(nsub, rank, world)
    t0 = time.time()
    blk = LibraryBlock(P, first, count,
                       iopts={F.PRECONDITIONER: args.precond, F.VERBOSE_LEVEL: 0, F.MAX_ITERATIONS: 5000},
                       ropts={F.PRECISION: args.precision}, ext={F.EXT_DEVICE_PREP: args.device_prep})
    group = dist.group.WORLD if dist is not None else None
    S = PartitionedSolver(blk, group=group)
    setup_s = time.time() - t0
    for _ in range(args.warmup):
        S.solve(precision=args.precision, max_it=5000, prec=args.precond)
    dist_barrier(dist)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            S.solve(precision=args.precision, max_it=5000, prec=args.precond)
        ev1.record()
        torch.cuda.synchronize()
    dist_barrier(dist)
    ms = dist_max(dist, ev0.elapsed_time(ev1) / args.steps)
    u = S.primal()
    res = P.relative_residual(u)
    line = {"metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.config, "subdomains": nsub, "dual_size": S.n_lambda, "kernel_size": S.n_kern,
                       "precond": args.precond, "precision": args.precision, "pcg_iterations": S.iterations,
                       "parallelism": f"subdomain-blocks{world}", "setup_s": setup_s,
                       "collectives_per_solve": S.collectives // max(1, args.warmup + args.steps)},
            "parity": {"residual": res, "converged": bool(S.converged)},
            "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line))
    blk.destroy()
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline_and_oracle(P, args, R):
    """CPU baseline and checker: the oracle's FP64 dual solve of the same mesh on all host cores.

    The timed part is one whole dual PCG solve (b, e -> lambda, alpha) at the bench precision, by the
    OpenMP C++ restatement of the reference's CPU solver (preprocessing untimed).  The same oracle
    then solves to ORACLE_PRECISION, so that its own error is far below the one it checks, for the
    mesh's load and for the first and last batched load case."""
    ncores = os.cpu_count() or 1
    t0 = time.perf_counter()
    OP, C = oracle_problem(P, args.precond)
    setup_s = time.perf_counter() - t0
    b, e = OP.vec_b(), OP.vec_e()
    t = time.perf_counter()
    C.solve(b, e, precision=args.precision, max_it=5000)
    ms = (time.perf_counter() - t) * 1e3
    iters = C.iterations
    uo = oracle_u(OP, C, P, ORACLE_PRECISION)
    ucols = {}
    if R is not None:
        for j in sorted({0, len(R) - 1}):
            ucols[j] = oracle_u(OP, C, P, ORACLE_PRECISION, f=R[j])
    cpu = {"value": ms, "unit": "ms", "cores": ncores, "kind": "port",
           "sample": f"one whole FP64 dual PCG solve ({iters} iterations: packed upper S_i SPMV, projector, "
                     f"preconditioner) of the same workload by the OpenMP C++ restatement of the reference's CPU "
                     f"solver on {ncores} threads; its preprocessing ({setup_s:.1f} s) untimed"}
    return cpu, uo, ucols


def run_adjoint(args):
    """Forward + backward of the adjoint workload (seeded densities, point load, compliance plus a
    seeded quadratic), timed on the host clock around the autograd calls; the two dual solves are
    reported with their device times."""
    import torch
    from espreso_b200 import adjoint, problems
    nd, ne = args.adjoint_grid
    P, rho, f = problems.adjoint_cube(domains=(nd, nd, nd), elements=(ne, ne, ne), seed=0)
    model = adjoint.SIMPModel(P, P.Ke, rhs=f, precision=args.precision, max_it=5000,
                              device_prep=bool(args.device_prep))
    q = np.random.default_rng(9).uniform(0.0, 1e10, size=P.ndofs)
    times = []
    for _ in range(args.warmup + args.steps):
        r = torch.tensor(rho, dtype=torch.float64, requires_grad=True)
        t = time.perf_counter()
        u = adjoint.solve(r, model)
        t_fwd = time.perf_counter() - t
        L = torch.dot(torch.from_numpy(f), u) + 0.5 * torch.sum(torch.from_numpy(q) * u * u)
        t = time.perf_counter()
        L.backward()
        t_bwd = time.perf_counter() - t
        times.append((t_fwd, t_bwd))
    fwd = float(np.median([a for a, _ in times[args.warmup:]])) * 1e3
    bwd = float(np.median([b for _, b in times[args.warmup:]])) * 1e3
    line = {"metric": "adjoint forward + backward wall time", "value": fwd + bwd, "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"adjoint_elasticity_{nd}^3x{ne}^3", "subdomains": nd ** 3,
                       "elements": int(P.elem_nodes.shape[0]), "dofs": int(P.ndofs)},
            "forward_ms": fwd, "backward_ms": bwd,
            "prep": "device" if args.device_prep else "host",
            "note": "forward includes the factorisation and Schur assembly of the new densities ("
                    + ("GPU" if args.device_prep else "host") + "); backward reuses them (second dual solve + "
                    "element sensitivity kernel)"}
    print(json.dumps(line))


def run_prep(args):
    """Instance creation of --config: decomposition, preprocessing (device or host) and upload; one
    JSON line with the times and the device eliminations' flops and rate."""
    from espreso_b200 import feti4i as F
    from espreso_b200 import problems
    P = problems.build_config(args.config)
    times = []
    st = {}
    for _ in range(args.warmup + args.steps):
        t = time.perf_counter()
        inst = problems.make_instance(P, iopts={F.PRECONDITIONER: args.precond, F.VERBOSE_LEVEL: 0,
                                                F.FETI_METHOD: args.method},
                                      ropts={F.PRECISION: args.precision},
                                      ext={F.EXT_SCHUR_PRECISION: SCHUR[args.schur], F.EXT_AUTOTUNE: 0,
                                           F.EXT_DEVICE_PREP: args.device_prep},
                                      clusters=P.sub_cluster() if args.method == 1 else None)
        times.append(time.perf_counter() - t)
        st = inst.stats()
        inst.destroy()
    wall = float(np.median(times[args.warmup:])) * 1e3
    line = {"metric": "instance creation wall time", "value": wall, "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.config, "subdomains": int(st["subdomains"]),
                                            "prep": "device" if args.device_prep else "host"},
            "prep_s": st["prep_seconds"], "upload_s": st["upload_seconds"],
            "prep_device_ms": st["prep_device_ms"], "prep_device_gflop": st["prep_device_flops"] * 1e-9,
            "prep_device_tflops": (st["prep_device_flops"] / st["prep_device_ms"] * 1e-9
                                   if st["prep_device_ms"] > 0 else None)}
    print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    if a.leg == "adjoint":
        run_adjoint(a)
    elif a.leg == "prep":
        run_prep(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.mode == "partitioned":
        run_partitioned(a)
    else:
        run_ours(a)
