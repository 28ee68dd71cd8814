#!/usr/bin/env python3
"""Benchmark of the plain-FP64 staggered phase-field fracture step on B200.

A step is one staggered load increment (crack_propagation.cpp:65-121): the mechanical FAS
multigrid solve (u_entire), the strain-history update, the phase-field FAS solve, the d
reductions and the reaction sum, on the 257^3 three-phase inclusion/pore specimen with a
mid-height pre-crack (seeded synthetic stand-in; every field exceeds the 126 MB L2, so no L2
flush is needed between steps).  One process per GPU; with N > 1 each rank solves its own replica
of the specimen (weak scaling, no data-path collective), timed on the device and reduced as the
max over ranks.

metric: MDoF-iter/s = (3 N_finest x mechanical finest-level smoother iterations
                       + N_finest x phase-field finest-level smoother iterations) / s

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MDoF-iter/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# Algorithmic bytes per finest node of the mechanical operator apply: u in (24), bulK, G, d (24),
# the regime (2) and the result (24) = 74 B/node, the compulsory traffic of y = K(d) u.  The roofline
# is reported on this basis.  The apply as the mechanical solves run it reads the Gauss-point moduli
# precomputed once per solve instead of bulK, G, d and the regime: p and w (24 B each) plus K_g, G_g
# (16 doubles per element = 128 B) = 176 B/node, reported beside it (the kernel trades FP64
# instructions, its bound, for bytes).
APPLY_BYTES_PER_NODE = 74
PCG_APPLY_BYTES_PER_NODE = 176
# ncu counters of the FP64 apply (one capture of the 193^3 level, the same kernel the bench times):
# FP64 pipe active 60.7 % of active cycles, issue active 56.1 %, top stall "wait" (fixed-latency
# dependencies) 1.36 per issued instruction.
APPLY_FP64_PIPE_ACTIVE = 0.607
MECH_SOLVERS = {"fas": 0, "fcg": 1, "mixed": 2}

# DRAM bytes (read + write) per launch of the finest PCG apply: one ncu capture of the kernel on the
# 193^3 level (7,189,057 nodes) measured 1339.8 MB read + 165.9 MB written, 209.4 B/node (the
# Gauss-point moduli of strip-edge elements are read twice); other sizes scale that per-node figure
# by their node count.
PCG_APPLY_TRAFFIC_PER_NODE = (1339.779e6 + 165.902848e6) / 193 ** 3


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", default="plain257")
    ap.add_argument("--mech-solver", choices=("fas", "fcg", "mixed"), default="fas",
                    help="fas: the reference's FAS V-cycles (plain form); fcg: flexible PCG preconditioned by one "
                         "FP64 V-cycle per iteration; mixed: the precision form (FP32 V-cycle, FP64 outer PCG)")
    ap.add_argument("--no-tma", action="store_true",
                    help="stage the finest applies' node rows with per-lane cp.async instead of tensor copies "
                         "(hpc_set_tma_staging 0)")
    ap.add_argument("--cpu-plan-runs", default="parity65:3,crack65:2,parity129:3", metavar="NAME:K[,...]",
                    help="--cpu-plan: the workloads and increment counts of its full runs")
    ap.add_argument("--cpu-plan-gpu-only", action="store_true",
                    help="--cpu-plan: only the B200 side of the full runs (the reference's side: "
                         "python -m oracle.time_reference NAME K)")
    ap.add_argument("--split", choices=("replicas", "slab"), default="replicas",
                    help="replicas: one specimen per GPU (weak scaling, the default); slab: one specimen split "
                         "along z over the GPUs, one rank each over NCCL (strong scaling)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-kernel-timing", action="store_true")
    ap.add_argument("--autotune", action="store_true",
                    help="measure the element kernels' strip shapes on first use (hpc_set_autotune) instead of "
                         "the latency model's choice")
    ap.add_argument("--tensor-apply", action="store_true",
                    help="precision form: run the FP32 V-cycle's element operator as TF32 GEMMs on the tensor "
                         "cores (hpc_set_tensor_apply) instead of the FP32 stencil kernels")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the precision-form measurement on the same increments")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-form sub-measurement (64 specimens of the uneven-size mix, plain FAS "
                         "against the precision form)")
    ap.add_argument("--kernel-only", type=int, default=0, metavar="NB",
                    help="profiling driver: set the specimen up, run one finest-level pcg_u with NB iterations "
                         "(NB launches of the dominant kernel) and exit")
    ap.add_argument("--profile-cycles", type=int, default=0, metavar="K",
                    help="profiling driver: set the specimen up and run two increments capped at K mechanical "
                         "and K phase-field V-cycles each (the step's kernel mix in a bounded launch count)")
    ap.add_argument("--serve", default="", metavar="RATE[,RATE...]",
                    help="serving form: Poisson arrivals at RATE requests/s (seed 7) through the continuous-"
                         "admission server; prints solves/s and p50/p99 latency, one line per rate (the same "
                         "requests at every rate)")
    ap.add_argument("--batch", type=int, default=0, metavar="N",
                    help="batched form: N specimens of the uneven-size mix (seeds 100..) submitted at once")
    ap.add_argument("--cpu-plan", action="store_true",
                    help="the reference's CPU path on this host's cores: one Internal_Force and one Fld apply on the "
                         "65^3, 129^3 and 257^3 pre-cracked specimens, full staggered increments of the 65^3 "
                         "configuration and of the pre-cracked 65^3 specimen, beside the same work on the GPU")
    ap.add_argument("--reference-tol", type=float, default=0.0, metavar="SQ",
                    help="--compare-forms: also solve every increment with the FP64 flexible PCG to the squared "
                         "ratio SQ (e.g. 1e-24) and report both forms' errors against that converged field")
    ap.add_argument("--compare-forms", action="store_true",
                    help="run --steps increments with the plain form and with --mech-solver (default mixed) and "
                         "report solves/s of both and the per-field error against the plain run")
    ap.add_argument("--mg-u", default="", metavar="NU0,NU1,NU2,GAMMA",
                    help="override the workload's mechanical multigrid parameters (ncy stays)")
    ap.add_argument("--requests", type=int, default=24, help="requests in a --serve sample")
    ap.add_argument("--increments", type=int, default=0, help="increments per request (default 10 serve, 5 batch)")
    ap.add_argument("--slots", type=int, default=8, help="concurrent requests on the GPU")
    ap.add_argument("--time-graphs", action="store_true",
                    help="batch engine: wait for each graph after its launch to time it (hpc_batch_timing)")
    ap.add_argument("--engine", choices=("batch", "threads"), default="batch",
                    help="serving / batched forms: batch = one engine thread advancing every active request by one "
                         "increment per batched call (hpc_batch_step: device-driven solve loops, one graph launch "
                         "per solve phase for all requests); threads = one worker thread and stream per slot")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--sizes", default="", help="serve: comma list of cubic sizes to draw from (default: the mix)")
    return ap.parse_args()


def run_serving(args, local):
    """Serving / batched forms: whole fracture runs through hpcrack_b200.serving.SolveServer."""
    import torch
    from hpcrack_b200 import serving as sv
    torch.cuda.set_device(local)
    budget = int(args.hbm_budget_gb * (1 << 30))
    if args.batch:
        inc = args.increments or 5
        reqs = [sv.Request(i, sv.batch_specimen(100 + i, inc), inc) for i in range(args.batch)]
        metric, form = "solves/s", f"batched: {args.batch} specimens (seeds 100..{99 + args.batch}), sizes per axis " \
                                   f"from {{33,65,97,129,161}}, {inc} increments each, submitted at t=0"
    else:
        rates = [float(r) for r in str(args.serve).split(",") if r]
        if len(rates) > 1:
            for r in rates:
                sub = argparse.Namespace(**vars(args))
                sub.serve = str(r)
                run_serving(sub, local)
            return
        inc = args.increments or 10
        kw = {}
        if args.sizes:
            kw = {"sizes": tuple((int(n),) * 3 for n in args.sizes.split(",")), "weights": None}
            kw["weights"] = tuple(1.0 for _ in kw["sizes"])
        reqs = sv.serve_mix(args.requests, rates[0], seed=7, increments=inc, **kw)
        metric, form = "solves/s", f"served: {args.requests} requests, Poisson arrivals at {rates[0]}/s (seed 7), " \
                                   f"{inc} increments each"
    if args.mg_u:
        v = tuple(int(x) for x in args.mg_u.split(","))
        for q in reqs:
            q.workload.mg_u = v + (q.workload.mg_u[4],)
    kw = {"time_graphs": args.time_graphs} if args.engine == "batch" else {}
    server = sv.BatchServer if args.engine == "batch" else sv.SolveServer
    srv = server(budget, args.slots, solver_factory=sv.default_factory(local, tma=not args.no_tma),
                 mech_solver=MECH_SOLVERS[args.mech_solver], precision_mg=not args.mg_u, **kw)
    from hpcrack_b200.solver import precision_mg
    mg_used = reqs[0].workload.mg_u
    if args.mech_solver != "fas" and not args.mg_u:
        mg_used = "per request: " + ", ".join(sorted({str(precision_mg(q.workload.maxlevel, q.workload.element_nb,
                                                                        q.workload.mg_u[4])) for q in reqs}))
    t0 = time.perf_counter()
    res = srv.replay(reqs)
    wall = time.perf_counter() - t0
    st = sv.latency_stats(res, wall)
    dof_iters = 0.0
    for r, q in zip(res, reqs):
        nx, ny, nz = q.workload.nodes
        dof_iters += sum(3.0 * nx * ny * nz * o[6] + nx * ny * nz * o[7] for o in r.outputs)
    line = {"metric": metric, "value": st["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic", "config": {"workload": form, "slots": args.slots, "engine": args.engine,
                                                            "hbm_budget_gb": args.hbm_budget_gb,
                                                            "mech_solver": args.mech_solver,
                                                            "mg_u": mg_used if isinstance(mg_used, str)
                                                            else list(mg_used)},
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "mean_s": st["mean_s"], "wall_s": wall,
            "batched_calls": getattr(srv, "rounds", None), "batch_timing": getattr(srv, "batch_timing", None),
            "mdof_iter_per_s": dof_iters / wall / 1e6, "peak_active": srv.peak_active,
            "peak_hbm_gb": srv.peak_used / (1 << 30)}
    print(json.dumps(line), flush=True)


def batch_measure(local, n=64, increments=5, mech_solver="mixed", hbm_budget_gb=150.0):
    """The batched form: n specimens of the uneven-size mix (seeds 100..), `increments` each, submitted
    at once to the batch engine (one engine thread; every specimen's solves as device-driven loops of
    one CUDA graph per phase).  Returns solves/s, p50/p99 latency, wall time and the engine's timing."""
    from hpcrack_b200 import serving as sv
    reqs = [sv.Request(i, sv.batch_specimen(100 + i, increments), increments) for i in range(n)]
    srv = sv.BatchServer(int(hbm_budget_gb * (1 << 30)), n, solver_factory=sv.default_factory(local, tma=TMA_STAGING),
                         mech_solver=MECH_SOLVERS[mech_solver])
    t0 = time.perf_counter()
    res = srv.replay(reqs)
    wall = time.perf_counter() - t0
    st = sv.latency_stats(res, wall)
    return {"solves_per_s": st["solves_per_s"], "p50_s": st["p50_s"], "p99_s": st["p99_s"], "wall_s": wall,
            "batched_calls": srv.rounds, "peak_hbm_gb": srv.peak_used / (1 << 30),
            "v_cycles": int(sum(o[4] for r in res for o in r.outputs))}


def workload(args):
    from hpcrack_b200 import microstructure as ms
    w = ms.make_workload(args.workload)
    if args.mg_u:
        v = tuple(int(x) for x in args.mg_u.split(","))
        w.mg_u = v + (w.mg_u[4],)
    return w


def run_kernel_only(args, local):
    """A short, bounded program for profilers: material setup, then pcg_u(NB) on the finest level."""
    from hpcrack_b200 import microstructure as ms
    w = workload(args)
    hier = load_specimen(w, local)
    hier.mp_choice()
    hier.mp_all_element(w.small_k)
    _, fn = hier.pcg_u(w.maxlevel, w.small_k, 1.0, args.kernel_only, 0, 0.0)
    hier.sync()
    print(json.dumps({"kernel_only": args.kernel_only, "workload": w.name, "f_norm": fn}), flush=True)
    hier.close()


def run_profile_cycles(args, local):
    """A short, bounded program for profilers: two increments whose V-cycle counts are capped at K."""
    from hpcrack_b200 import microstructure as ms
    w = workload(args)
    hier = load_specimen(w, local)
    K = args.profile_cycles
    mg_u = tuple(w.mg_u[:4]) + (K,)
    if args.mech_solver != "fas" and not args.mg_u:
        from hpcrack_b200.solver import precision_mg
        mg_u = precision_mg(w.maxlevel, w.element_nb, K)
    mg_d = tuple(w.mg_d[:4]) + (K,)
    from hpcrack_b200.solver import KC_MECH_PCG_FINEST, KC_MECH32_PCG_FINEST
    kc = KC_MECH_PCG_FINEST if args.mech_solver == "fas" else KC_MECH32_PCG_FINEST
    hier.kernel_timing(kc)  # CUDA-event times of the finest PCG apply (FP64, or FP32 in the precision form)
    launches0 = hier.launch_count()
    outs = [hier.step(t, mg_u, mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, dU_factor=w.du_factor,
                      mech_tol=w.mech_tol, pf_tol=w.pf_tol, mech_solver=MECH_SOLVERS[args.mech_solver])
            for t in range(2)]
    hier.sync()
    kn, kms = hier.kernel_time()
    print(json.dumps({"profile_cycles": K, "workload": w.name, "launches": hier.launch_count() - launches0,
                      "mech_cycles": [int(o[4]) for o in outs], "pf_cycles": [int(o[5]) for o in outs],
                      "tensor_apply": TENSOR_APPLY, "finest_pcg_apply": {"launches": kn,
                                                                         "mean_us": 1000.0 * kms / max(kn, 1)}}),
          flush=True)
    hier.close()


# ---------------------------------------------------------------------------------------------
# process group
# ---------------------------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world: int):
    from hpcrack_b200 import replicas
    replicas.barrier(world)


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"hpc_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# CPU reference sample (the reference's own pcg_u, compiled from its sources)
# ---------------------------------------------------------------------------------------------
def cpu_reference_sample(w, repeats: int = 1, nb_relax: int = 4, slab: int = 5):
    """Times the reference's finest-level mechanical smoother pcg_u(NB_relax=nb_relax) on a
    nx*ny*slab-node slab taken at mid-height of the workload's image, one rank (single-rank MPI
    stand-in) with every host core as OpenMP threads.  Returns (MDoF-iter/s, info)."""
    import numpy as np
    from oracle import bindings as B
    from hpcrack_b200 import microstructure as ms

    nx, ny, nz = w.nodes
    z0 = (nz - slab) // 2
    img = np.ascontiguousarray(w.image[z0:z0 + slab])
    enb = (nx - 1, ny - 1, slab - 1)
    cores = os.cpu_count() or 1
    kind = "reference" if B.RefOracle.available() else "port"
    impl = B.RefOracle(0, enb) if kind == "reference" else B.COracle(0, enb)
    if kind == "reference":
        impl.set_threads(cores)
        with tempfile.TemporaryDirectory() as td:
            os.makedirs(os.path.join(td, "data"))
            raw = os.path.join(td, "data", "slab.raw")
            img.tofile(raw)
            ms.write_material_csv(os.path.join(td, "data", "Material_Property.csv"), w.table())
            impl.input_total(td, raw, (nx, ny, slab), w.voxel_size)
    else:
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        impl.image_material(img, (nx, ny, slab), w.table(), w.voxel_size)
    impl.mp_choice()
    impl.mp_all_element(w.small_k)
    n = nx * ny * slab
    times = []
    for _ in range(repeats):
        impl.set(B.U, 0, np.zeros((3, n)))
        impl.set(B.FU, 0, np.zeros((3, n)))
        t0 = time.perf_counter()
        impl.pcg_u(0, w.small_k, 1.0, nb_relax, 0, 0.0)
        times.append(time.perf_counter() - t0)
    impl.close()
    dt = min(times)
    value = 3.0 * n * nb_relax / dt / 1e6
    info = {"value": value, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"pcg_u(NB_relax={nb_relax}) on the finest level of a {nx}x{ny}x{slab}-node mid-height slab "
                      f"of the {w.name} image, 1 rank x {cores} OpenMP threads, {dt:.2f} s"}
    return value, info


def run_reference(args, rank, world):
    from hpcrack_b200 import microstructure as ms
    if rank != 0:
        return
    w = workload(args)
    vals = []
    for _ in range(max(args.warmup, 0)):
        cpu_reference_sample(w)
    for _ in range(args.steps):
        v, info = cpu_reference_sample(w)
        vals.append(v)
    value = statistics.mean(vals)
    info["value"] = value
    nx, ny, nz = w.nodes
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, world),
            "cpu_baseline": info,
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------------------------
def workload_config(w, world, mech_solver="fas"):
    nx, ny, nz = w.nodes
    return {"workload": f"{w.name}: {nx}x{ny}x{nz}-node three-phase inclusion/pore specimen, pre-cracked, "
                        f"staggered increments (mechanical + phase-field FAS V-cycles, plain FP64)",
            "nodes": nx * ny * nz, "mech_dof": 3 * nx * ny * nz, "levels": w.maxlevel + 1,
            "element_nb": list(w.element_nb), "mg_u": list(w.mg_u), "mg_d": list(w.mg_d),
            "mech_tol_sq": w.mech_tol, "pf_tol_sq": w.pf_tol, "replicas": world, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (each finest field 136 MB > 126 MB), no flush",
            "mech_solver": {"fas": "FAS V-cycles with restarted Jacobi-PCG smoothers (the reference's method)",
                            "fcg": "flexible PCG (FP64) preconditioned by one V-cycle per iteration",
                            "mixed": "precision form: flexible PCG (FP64 residual, dots, updates) preconditioned by "
                                     "one FP32 V-cycle (FP64 coarsest solve)"}[mech_solver]}


TENSOR_APPLY = False  # --tensor-apply
TMA_STAGING = True    # --no-tma turns it off


def load_specimen(w, device):
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200.solver import Hierarchy, H, D
    hier = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start, device=device)
    if TENSOR_APPLY:
        hier.set_tensor_apply(True)
    if not TMA_STAGING:
        hier.set_tma_staging(False)
    hier.image_material(w.image, w.nodes, w.table(), w.voxel_size)
    if w.crack:
        Hc, dc = ms.precrack_fields(w)
        hier.set(H, w.maxlevel, Hc)
        hier.set(D, w.maxlevel, dc)
        hier.voigt_all_level(H)
    return hier


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def run_slab(args, rank, world, local):
    """--split slab: one specimen split along z over the job's ranks (hpc_create_slab, one GPU each, ghost
    planes and reductions over NCCL): strong scaling, the same work at every N.  value = the specimen's
    DoF-iterations / the slowest rank's device time."""
    import torch
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200 import slab
    from hpcrack_b200.solver import KC_MECH_PCG_FINEST, D, H, Hierarchy

    torch.cuda.set_device(local)
    w = workload(args)
    nx, ny, nz = w.nodes
    N = nx * ny * nz
    if world > 1:
        h = slab.from_process_group(w.maxlevel, w.element_nb, w.x_start, device=local)
    else:  # one rank: a one-rank communicator on this host
        os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")
        h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start, device=local, slab=(1, 0))
        slab.join_nccl(h, slab.nccl_unique_id())
    Lf = w.maxlevel
    h.image_material(w.image, w.nodes, w.table(), w.voxel_size)
    if w.crack:
        Hc, dc = ms.precrack_fields(w)
        h.set(H, Lf, slab.local_part(h, Lf, Hc))
        h.set(D, Lf, slab.local_part(h, Lf, dc))
        h.voigt_all_level(H)
    stream = torch.cuda.ExternalStream(h.stream())
    solver = MECH_SOLVERS[args.mech_solver]

    def step(t):
        return h.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, dU_factor=w.du_factor,
                      mech_tol=w.mech_tol, pf_tol=w.pf_tol, mech_solver=solver)

    for t in range(args.warmup):
        step(t)
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    h.kernel_timing(KC_MECH_PCG_FINEST)
    launches0 = h.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = [step(args.warmup + i) for i in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    launches = h.launch_count() - launches0
    kn, kms = h.kernel_time()
    h.kernel_timing(-1)
    ms_rank = e0.elapsed_time(e1)
    max_ms = ms_rank
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms_rank], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        max_ms = float(tt.item())
    dof_iters = sum(3.0 * N * o[6] + 1.0 * N * o[7] for o in outs)  # every rank reports the specimen's counts
    local_nodes = nx * ny * h.dims[Lf][2]
    h.close()
    if rank == 0:
        peak, src = peaks()
        achieved = local_nodes * APPLY_BYTES_PER_NODE / (kms / max(kn, 1) / 1e3) / 1e9 if kn else None
        cfg = workload_config(w, world, args.mech_solver)
        plans = [slab.slab_level(w.maxlevel, w.element_nb, world, r, Lf) for r in range(world)]
        cfg.update({"parallelism": f"slab-z{world}", "replicas": 1,
                    "split": "z slabs of the specimen, one per rank; owned finest planes per rank: "
                             f"{[p[3] - p[2] for p in plans]}"})
        line = {"metric": METRIC, "value": dof_iters / (max_ms / 1e3) / 1e6, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": cfg, "clocks": clocks, "gpu_launches": launches,
                "roofline": ({"bound": "hbm", "kernel": "finest PCG apply on rank 0's slab", "achieved": achieved,
                              "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": src,
                              "bytes_per_node": APPLY_BYTES_PER_NODE, "nodes": local_nodes, "launches": kn,
                              "avg_launch_ms": kms / kn, "traffic": None} if kn else None),
                "e2e": None, "cpu_baseline": None,
                "steps_detail": [{"mech_cycles": int(o[4]), "pf_cycles": int(o[5]), "F": o[1]} for o in outs]}
        print(json.dumps(line), flush=True)


def run_b200(args, rank, world, local):
    import torch
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200 import replicas
    from hpcrack_b200.solver import KC_MECH_PCG_FINEST, U, D, H, FU, DOLDF, Hierarchy

    torch.cuda.set_device(local)
    w = workload(args)
    nx, ny, nz = w.nodes
    N = nx * ny * nz
    hier = load_specimen(w, local)
    if args.autotune:
        hier.set_autotune(True)
    stream = torch.cuda.ExternalStream(hier.stream())

    solver = MECH_SOLVERS[args.mech_solver]

    def step(t):
        return hier.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du,
                         dU_factor=w.du_factor, mech_tol=w.mech_tol, pf_tol=w.pf_tol, mech_solver=solver)

    t = 0
    for _ in range(args.warmup):
        step(t)
        t += 1

    # ------------------------------------------------------------ timed region (device-resident)
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    if not args.no_kernel_timing:
        hier.kernel_timing(KC_MECH_PCG_FINEST)
    launches0 = hier.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = []
    t_first = t
    for _ in range(args.steps):
        outs.append(step(t))
        t += 1
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    launches = hier.launch_count() - launches0
    ms_total = e0.elapsed_time(e1)
    plain_final = ({k: hier.get(f, w.maxlevel) for k, f in (("u", U), ("d", D), ("H", H))}
                   if (not args.no_forms and args.mech_solver == "fas") else None)
    kn, kms = hier.kernel_time() if not args.no_kernel_timing else (0, 0.0)
    hier.kernel_timing(-1)

    dof_iters = sum(3.0 * N * o[6] + 1.0 * N * o[7] for o in outs)
    mech_cycles = sum(o[4] for o in outs)
    max_ms, tot_dof_iters = replicas.aggregate(ms_total, dof_iters, world)
    value = tot_dof_iters / (max_ms / 1e3) / 1e6

    # roofline of the dominant kernel: the finest-level PCG apply w = K(d) p with the (p, w) reduction
    # (PCG_APPLY_BYTES_PER_NODE algorithmic bytes per finest node).
    roofline = None
    if kn > 0:
        alg = APPLY_BYTES_PER_NODE
        read = PCG_APPLY_BYTES_PER_NODE
        achieved = N * alg / (kms / kn / 1e3) / 1e9
        achieved_read = N * read / (kms / kn / 1e3) / 1e9
        peak, src = peaks()
        kname = ("mech_kernel<finest, PCG, Gauss-point moduli, " +
                 ("rows staged by TMA tensor copies" if TMA_STAGING else "rows staged by per-lane cp.async") +
                 "> (w = K(d) p, (p, w))")
        basis = "algorithmic: u 24 + bulK,G,d 24 + regime 2 + out 24 B per finest node"
        roofline = {"bound": "hbm", "kernel": kname,
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": src, "bytes_per_node": alg, "bytes_basis": basis,
                    "traffic": PCG_APPLY_TRAFFIC_PER_NODE * N,
                    "traffic_note": "bytes per launch: ncu dram bytes per node of the 193^3 capture x nodes; above "
                                    "the algorithmic bytes because the kernel reads precomputed Gauss-point moduli",
                    "read_layout": {"bytes_per_node": read, "achieved": achieved_read,
                                    "frac": achieved_read / peak,
                                    "what": "the vectors and the precomputed Gauss-point moduli the kernel reads "
                                            "and writes"},
                    "fp64_pipe_active_ncu": APPLY_FP64_PIPE_ACTIVE,
                    "limiter": "FP64 pipe (dependent FP64 latency), not HBM",
                    "launches": kn, "avg_launch_ms": kms / kn}

    # ------------------------------------------------------------ end to end through the C ABI
    e2e = None
    if not args.no_e2e:
        Lf = w.maxlevel
        pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True)  # noqa: E731
        hu, hfu = pin(3 * N), pin(3 * N)
        hd, hH, hdo = pin(N), pin(N), pin(N)
        # start from the current state, held on the host
        dptr = lambda ten: C.cast(ten.data_ptr(), C.POINTER(C.c_double))  # noqa: E731
        lib = hier.lib

        def down(field, ten, ncomp):
            for c in range(ncomp):
                lib.hpc_download(hier.h, field, Lf, c, C.cast(ten.data_ptr() + 8 * c * N, C.POINTER(C.c_double)))

        def up(field, ten, ncomp):
            for c in range(ncomp):
                lib.hpc_upload(hier.h, field, Lf, c, C.cast(ten.data_ptr() + 8 * c * N, C.POINTER(C.c_double)))

        down(U, hu, 3); down(FU, hfu, 3); down(D, hd, 1); down(H, hH, 1); down(DOLDF, hdo, 1)
        barrier(world)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        e2e_iters = 0.0
        for _ in range(args.steps):
            up(U, hu, 3); up(FU, hfu, 3); up(D, hd, 1); up(H, hH, 1); up(DOLDF, hdo, 1)
            o = step(t)
            t += 1
            down(U, hu, 3); down(FU, hfu, 3); down(D, hd, 1); down(H, hH, 1)
            e2e_iters += 3.0 * N * o[6] + 1.0 * N * o[7]
        f1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        e2e_ms, e2e_work = replicas.aggregate(f0.elapsed_time(f1), e2e_iters, world)
        e2e_val = e2e_work / (e2e_ms / 1e3) / 1e6
        e2e = {"value": e2e_val, "unit": METRIC, "h2d_bytes_per_step": 8 * N * 9, "d2h_bytes_per_step": 8 * N * 8,
               "ms_per_step": e2e_ms / args.steps}
        del hu, hfu, hd, hH, hdo

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            _, cpu = cpu_reference_sample(w)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"failed: {exc}"}

    hier.close()

    # ------------------------------------------------------------ the precision form on the same increments
    forms = None
    if not args.no_forms and args.mech_solver == "fas":
        wp = workload(args)
        from hpcrack_b200.solver import precision_mg
        wp.mg_u = precision_mg(wp.maxlevel, wp.element_nb, wp.mg_u[4])
        hp = load_specimen(wp, local)
        sp = torch.cuda.ExternalStream(hp.stream())

        def pstep(tt):
            return hp.step(tt, wp.mg_u, wp.mg_d, wp.small_k, wp.lc, wp.voxel_size, ut0=wp.ut0, dU=wp.du,
                           dU_factor=wp.du_factor, mech_tol=wp.mech_tol, pf_tol=wp.pf_tol,
                           mech_solver=MECH_SOLVERS["mixed"])
        for tt in range(args.warmup):
            pstep(tt)
        barrier(world)
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(sp)
        pouts = [pstep(args.warmup + i) for i in range(args.steps)]
        g1.record(sp)
        torch.cuda.synchronize()
        barrier(world)
        p_ms, _ = replicas.aggregate(g0.elapsed_time(g1), 0.0, world)
        mixed_final = {k: hp.get(f, wp.maxlevel) for k, f in (("u", U), ("d", D), ("H", H))}
        hp.close()
        forms = {"plain": {"solves_per_s": world * args.steps / (max_ms / 1e3),
                           "v_cycles": [int(o[4]) for o in outs]},
                 "mixed": {"solves_per_s": world * args.steps / (p_ms / 1e3), "ms_per_step": p_ms / args.steps,
                           "v_cycles": [int(o[4]) for o in pouts], "mg_u": list(wp.mg_u),
                           "what": "flexible PCG in FP64 (true residual, dots, updates) preconditioned by one "
                                   "FP32 V-cycle per iteration (FP64 coarsest solve); same increments, same "
                                   "FP64 stopping test |r|/|f| <= 1e-8"},
                 "speedup_mixed_vs_plain": max_ms / p_ms}
        if plain_final is not None:
            forms["mixed"]["u_rel_l2_vs_plain"] = field_errors(mixed_final["u"], plain_final["u"])["rel_l2"]
            forms["mixed"]["error_vs_plain"] = {k: field_errors(mixed_final[k], plain_final[k]) for k in ("u", "d", "H")}
            forms["mixed"]["error_note"] = (f"fields after increment {t_first + args.steps - 1} of both forms, each "
                                            "solved to |r|/|f| <= 1e-8; rel_l2 = |a-b|/|b|, max_abs = max|a-b|")
    # ------------------------------------------------------------ the batched form (64-specimen mix)
    batch = None
    if not args.no_batch and world == 1:
        try:
            bp = batch_measure(local, mech_solver="fas")
            bm = batch_measure(local, mech_solver="mixed")
            batch = {"workload": "64 specimens, seeds 100-163, nodes per axis from {33,65,97,129,161}, inclusion "
                                 "volume fraction in [5%,35%], 5 increments each, submitted at once",
                     "engine": "one engine thread; each increment of all specimens is one hpc_batch_step: per solve "
                               "phase one CUDA graph launch whose per-specimen WHILE loops run to convergence",
                     "plain": bp, "mixed": bm, "speedup_mixed_vs_plain": bm["solves_per_s"] / bp["solves_per_s"]}
        except Exception as exc:  # reported, never required for the headline line
            batch = {"error": str(exc)}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(w, world, args.mech_solver), "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu, "forms": forms, "batch": batch,
                "strip_shapes": ({"autotuned": [list(x) for x in Hierarchy.tuned_shapes()]} if args.autotune
                                 else "latency model (choose_strips)"),
                "solves_per_s": world * args.steps / (max_ms / 1e3),
                "v_cycles_per_s": world * sum(o[4] + o[5] for o in outs) / (max_ms / 1e3),
                "steps_detail": [{"t": t_first + i, "mech_cycles": int(o[4]), "pf_cycles": int(o[5]),
                                  "mech_iters": int(o[6]), "pf_iters": int(o[7]), "F": o[1], "dmax": o[3]}
                                 for i, o in enumerate(outs)]}
        print(json.dumps(line), flush=True)


def field_errors(a, b) -> dict:
    """Relative L2 and maximum absolute difference of field a against field b."""
    import numpy as np
    nb = float(np.linalg.norm(b))
    return {"rel_l2": float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0),
            "max_abs": float(np.max(np.abs(a - b))), "max_ref": float(np.max(np.abs(b)))}


def run_compare_forms(args, local):
    """Precision form against the plain FP64 form on the same specimen: both run the same increments
    to the same FP64 stopping test; prints solves/s of each and the per-field L2 / max error of the
    precision form's u, d, H relative to the plain run."""
    import numpy as np
    import torch
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200.solver import U, D, H
    torch.cuda.set_device(local)
    w = workload(args)
    res = {}
    names = ["fas", args.mech_solver if args.mech_solver != "fas" else "mixed"]
    if args.reference_tol > 0:
        names.append("reference")
    for name in names:
        hier = load_specimen(w, local)
        solver_id = MECH_SOLVERS["fcg"] if name == "reference" else MECH_SOLVERS[name]
        tol = args.reference_tol if name == "reference" else w.mech_tol
        mg_u = w.mg_u
        if name != "fas":
            from hpcrack_b200.solver import precision_mg
            mg_u = precision_mg(w.maxlevel, w.element_nb, w.mg_u[4])
        stream = torch.cuda.ExternalStream(hier.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        outs = [hier.step(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du,
                          dU_factor=w.du_factor, mech_tol=tol, pf_tol=w.pf_tol,
                          mech_solver=solver_id) for t in range(args.steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms_tot = e0.elapsed_time(e1)
        res[name] = {"outs": outs, "ms": ms_tot, "fields": {k: hier.get(f, w.maxlevel) for k, f in
                                                              (("u", U), ("d", D), ("H", H))}}
        hier.close()
    form_name = names[1]
    plain, other = res["fas"], res[form_name]
    errs = {k: field_errors(other["fields"][k], plain["fields"][k]) for k in ("u", "d", "H")}
    ncy = w.mg_u[4]
    line = {"metric": "solves/s", "workload": w.name, "increments": args.steps, "mech_tol_sq": w.mech_tol,
            "plain": {"solves_per_s": args.steps / (plain["ms"] / 1e3), "ms": plain["ms"],
                      "v_cycles": [int(o[4]) for o in plain["outs"]],
                      "hit_cycle_cap": [int(o[4]) >= ncy for o in plain["outs"]]},
            "form": {"name": form_name, "solves_per_s": args.steps / (other["ms"] / 1e3),
                     "ms": other["ms"], "v_cycles": [int(o[4]) for o in other["outs"]]},
            "speedup": plain["ms"] / other["ms"], "field_error_vs_plain": errs,
            "reaction_rel_diff": [abs(a[1] - b[1]) / abs(b[1]) for a, b in zip(other["outs"], plain["outs"])]}
    if "reference" in res:
        ref = res["reference"]
        line["reference"] = {"what": f"FP64 flexible PCG to |r|^2/|f|^2 <= {args.reference_tol:g} on every increment",
                             "ms": ref["ms"], "v_cycles": [int(o[4]) for o in ref["outs"]]}
        line["plain_error_vs_reference"] = {k: field_errors(plain["fields"][k], ref["fields"][k]) for k in ("u", "d", "H")}
        line["form_error_vs_reference"] = {k: field_errors(other["fields"][k], ref["fields"][k]) for k in ("u", "d", "H")}
    print(json.dumps(line), flush=True)


def run_cpu_plan(args, local):
    """The reference compiled from its sources (oracle/_ref), 1 rank x every host core as OpenMP
    threads, on the benchmark's specimens: per-apply times of Internal_Force (mechanical_pcg.cpp:
    174-191) and Fld (phase_field_pcg.cpp:93-103) with the specimen's real material, pre-crack and a
    displacement field, and full staggered increments (crack_propagation.cpp:65-121) at the reference's
    own thresholds, each beside the same work on the GPU."""
    import numpy as np
    import torch
    from oracle import bindings as B
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200.solver import Hierarchy, U, D, H, RU, FD
    torch.cuda.set_device(local)
    cores = os.cpu_count() or 1
    B.RefOracle._load().ref_set_threads(cores)
    out = {"cpu_plan": True, "cores": cores, "kind": "reference", "layout": f"1 rank x {cores} OpenMP threads",
           "applies": [], "runs": []}

    def ref_for(w):
        ref = B.RefOracle(w.maxlevel, w.element_nb, x0=w.x_start)
        with tempfile.TemporaryDirectory() as td:
            paths = ms.write_inputs(w, td)
            t0 = time.perf_counter()
            ref.input_total(td, paths["raw"], w.nodes, w.voxel_size)
            t_in = time.perf_counter() - t0
        if w.crack:
            Hc, dc = ms.precrack_fields(w)
            ref.set(H, w.maxlevel, Hc)
            ref.set(D, w.maxlevel, dc)
            ref.voigt_all_level(H)
        return ref, t_in

    for name in (() if args.cpu_plan_gpu_only else ("crack65", "mid129", "plain257")):
        w = ms.make_workload(name)
        L = w.maxlevel
        gpu = load_specimen(w, local)
        gpu.u_entire(tuple(w.mg_u[:4]) + (4,), w.small_k, 1.0, 0, 0.0)  # a displacement field of this specimen
        u = gpu.get(U, L)
        ref, t_in = ref_for(w)
        ref.set(U, L, u)
        ref.mp_choice()
        ref.mp_all_element(w.small_k)
        t0 = time.perf_counter()
        ref.internal_force(L, U, RU, w.small_k)
        t_if = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.fld(L, D, FD, w.lc)
        t_fld = time.perf_counter() - t0
        gpu.mp_choice()
        gpu.mp_all_element(w.small_k)
        gpu.internal_force(L, U, RU, w.small_k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            gpu.internal_force(L, U, RU, w.small_k)
        g_if = (time.perf_counter() - t0) / 10
        nx, ny, nz = w.nodes
        n = nx * ny * nz
        out["applies"].append({"workload": name, "nodes": n, "input_total_s": t_in, "internal_force_s": t_if,
                               "fld_s": t_fld, "internal_force_mdof_s": 3 * n / t_if / 1e6,
                               "gpu_internal_force_s": g_if,
                               "gpu_note": "hpc_internal_force: the nodal-form apply through the C ABI (one call, "
                                           "host-synchronised), not the benchmark's precomputed-moduli kernel"})
        ref.close()
        gpu.close()
        print(json.dumps(out["applies"][-1]), flush=True)

    runs = [(r.split(":")[0], int(r.split(":")[1])) for r in args.cpu_plan_runs.split(",") if r]
    for name, steps in runs:
        w = ms.make_workload(name)
        L = w.maxlevel
        ref = None if args.cpu_plan_gpu_only else ref_for(w)[0]
        gpu = load_specimen(w, local)
        rec = {"workload": name, "increments": steps, "tolerance": "the reference's own: |r|^2/|f|^2 <= 1e-6, "
                                                                    "|R|^2/|fd|^2 <= 1e-12", "cpu": [], "gpu": []}
        for t in range(steps):
            if ref is not None:
                t0 = time.perf_counter()
                o = ref.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du)
                rec["cpu"].append({"t": t, "s": time.perf_counter() - t0, "mech_cycles": int(o[4]),
                                   "pf_cycles": int(o[5]), "mech_iters": int(o[6]), "pf_iters": int(o[7])})
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            og = gpu.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du)
            rec["gpu"].append({"t": t, "s": time.perf_counter() - t0, "mech_cycles": int(og[4]),
                               "pf_cycles": int(og[5])})
        nx, ny, nz = w.nodes
        n = nx * ny * nz
        if ref is not None:
            ct = sum(r["s"] for r in rec["cpu"])
            cit = sum(3.0 * n * r["mech_iters"] + n * r["pf_iters"] for r in rec["cpu"])
            rec["cpu_mdof_iter_per_s"] = cit / ct / 1e6
            rec["cpu_s_per_v_cycle"] = ct / max(1, sum(r["mech_cycles"] + r["pf_cycles"] for r in rec["cpu"]))
            rec["cpu_s"] = ct
            ref.close()
        rec["gpu_s"] = sum(r["s"] for r in rec["gpu"])
        out["runs"].append(rec)
        gpu.close()
        print(json.dumps(rec), flush=True)
    print(json.dumps(out), flush=True)


def main():
    global TENSOR_APPLY, TMA_STAGING
    args = parse_args()
    TENSOR_APPLY = args.tensor_apply
    TMA_STAGING = not args.no_tma
    rank, world, local = dist_setup()
    try:
        if args.kernel_only:
            run_kernel_only(args, local)
        elif args.profile_cycles:
            run_profile_cycles(args, local)
        elif (args.serve and any(float(r) > 0 for r in str(args.serve).split(",") if r)) or args.batch:
            run_serving(args, local)
        elif args.compare_forms:
            run_compare_forms(args, local)
        elif args.cpu_plan:
            run_cpu_plan(args, local)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        elif args.split == "slab":
            run_slab(args, rank, world, local)
        else:
            run_b200(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
