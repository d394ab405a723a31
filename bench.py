"""FDV step throughput on B200: mixed precision vs FP64 at equal residual.

Workload (default): the 2D supersonic flat plate, 200x100 quad4 (20,000 elements,
81,204 DOF), Mach 3, Re 1e4, each step = CFL + element formation (+ApplyBC) +
restarted GMRES(30) to a 1e-8 true relative residual + update.  One "step" of the
metric is one such FDV step.  Both forms run: FP64 and mixed (FP32 element matrices
and products inside FP64 iterative refinement); ``value`` is the mixed form's
steps/s, the FP64 figure is reported beside it.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events on the
solver's stream; between timed steps L2 is flushed by writing a 512 MiB buffer
(the plate's matrices fit in L2).  Under torchrun every rank runs its own replica
(the path is not partitioned: "replicas only"), the time is the max over ranks.

``--impl reference`` times the reference's own CPU path (oracle/_ref/cfdv_ref, the
CFDV sources built unmodified) on the same case on the host, one core.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FDV steps/s & EBE matvec GB/s: mixed vs FP64 on 1 B200 at equal residual"
# Each workload states where it departs from the configuration it stands for.
WORKLOADS = {
    "plate": dict(desc="2D supersonic flat plate 200x100 quad4, M=3, Re=1e4, GMRES(30) to 1e-8",
                  make=lambda mg: mg.plate(200, 100), m=30, cfl=1.0,
                  deviations=["initial state: uniform freestream with the seeded 1e-3 Gaussian density noise, except "
                              "over the plate, which starts from a tanh boundary-layer profile (u = tanh(y/0.005), "
                              "Crocco-Busemann T): with an exact linear solve the impulsive start drives the density "
                              "negative in the first step",
                              "CFL 1.0 (the configuration names none)",
                              "timed steps return to the post-warm-up state every 10 steps, outside the timed "
                              "regions: with converged solves the plate becomes unstable near t = 0.015 (step ~16), "
                              "on the oracle's CPU solve too, so the 2000-step run is not reached"]),
    "lid": dict(desc="2D lid-driven cavity 32x32 quad4, M=0.1, Re=100, GMRES(20) to 1e-8",
                make=lambda mg: mg.lid(32), m=20, cfl=0.5,
                deviations=["a few timed steps of the 200; the full 200-step run is a GPU parity test "
                            "(reference-mode solver against the oracle)"]),
    "ramp": dict(desc="3D compression ramp 128x64x32 hex8, M=2.5, Re=1e5, GMRES(50) to 1e-8",
                 make=lambda mg: mg.ramp(128, 64, 32), m=50, cfl=0.25,
                 deviations=["3 timed steps of the 500", "CFL 0.25 (the configuration names none)"]),
    "ramp64": dict(desc="3D compression ramp 64x32x32 hex8 (profiling size), M=2.5, Re=1e5, GMRES(50) to 1e-8",
                   make=lambda mg: mg.ramp(64, 32, 32), m=50, cfl=0.25, deviations=["profiling size"]),
    "duct": dict(desc="3D duct 200x100x50 hex8 (1,000,000 elements, jittered), M=0.8, Re=5e4, GMRES(40) to 1e-8",
                 make=lambda mg: mg.duct(200, 100, 50), m=40, cfl=0.5,
                 deviations=["3 timed steps of the 100", "stored element matrices (FP64 and FP32); the "
                             "on-the-fly recomputation is measured separately"]),
}
ADJOINT_DEVIATIONS = ["span: 16 node layers with symmetry planes (bc 2), not periodic by connectivity (elements take "
                      "their geometry from absolute coordinates, so a wrapped layer would be inverted)"]


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# The timed steps march from the state after the warm-up steps and go back to it every
# RESTART_EVERY steps (between steps, outside the timed regions): with converged solves at
# CFL 1 the synthetic plate develops an instability after about 20 steps (the oracle's
# converged solve shows it too), and a longer --steps run would then time stalled solves.
RESTART_EVERY = 10

# CPU-baseline sample of the reference build per workload: (timed steps, warm-up steps), about
# 15-20 s of one core
CPU_SAMPLE = {"plate": (20, 5), "lid": (40, 5), "ramp": (1, 0), "duct": (1, 0)}

# orthogonalisation of the persistent solve (cfdv_gmres_opts.orth)
ORTH = {"cgs2": 0, "mgs": 1, "dcgs2": 2, "dcgs2-grid": 3}  # dcgs2-grid: grid barriers only


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Ranks:
    """Replica bookkeeping across ranks (the path is not partitioned: every rank runs its own
    replica).  The barrier and the max over ranks use the process group when there is one:
    NCCL with CUDA tensors on the GPU box, gloo with CPU tensors in the tests."""

    def __init__(self, ws, device):
        self.ws, self.device = ws, device

    def barrier(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v):
        if self.ws == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, steps, seconds_max):
        """Whole-job steps per second: every replica's steps over the slowest replica's time."""
        return self.ws * steps / seconds_max


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_cpu(case, steps, warmup):
    """Time the reference build on the host: (seconds per step list, sample description)."""
    from oracle import oracle as O
    from cfdv_b200 import meshgen as mg
    with tempfile.TemporaryDirectory() as d:
        mg.write_case(case, d)
        rec = O.run_reference(d, os.path.join(d, "ref.rec"), steps=warmup + steps)
    times = [float(rec[f"steptime@{k}"][0]) for k in range(warmup, warmup + steps)]
    return times


def measure_workload(args, name, steps, warmup, flush, ws, barrier, max_over_ranks, sampler=None, warm=None):
    """Time FP64 and mixed FDV steps of one workload; returns per-form results and the
    live EBE element-pass roofline (one extra host-driven step with CUDA events).  warm: start
    each solve from the previous step's dU (default: --warm-start)."""
    warm = args.warm_start if warm is None else warm
    import numpy as np
    import torch
    from cfdv_b200 import gpu as G, meshgen as mg

    W = WORKLOADS[name]
    case = W["make"](mg)
    m, cfl, rtol = W["m"], W["cfl"], 1e-8
    solver = G.FDVSolver(case)
    ext = torch.cuda.ExternalStream(solver.stream)
    forms = [("fp64", G.PREC_FP64), ("mixed", G.PREC_MIXED)]
    if args.only:
        forms = [f for f in forms if f[0] == args.only]
    out = {"case": case, "solver": solver, "ext": ext, "m": m, "cfl": cfl, "rtol": rtol, "desc": W["desc"]}
    for prec_name, prec in forms:
        solver.load_node_records()
        for _ in range(warmup):
            solver.step(cfl, mode=G.GMRES_CORRECT, m=m, restarts=200, rtol=rtol, precision=prec,
                        orth=ORTH[args.orth], warm_start=warm)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        if sampler is not None and prec_name == forms[0][0]:
            sampler.start()  # runs across every timed region of the run (both forms, e2e)
        solver.profile(True)
        step_ms, res, mvs = [], [], []
        snap = solver.get_state()
        for i in range(steps):
            if i and i % RESTART_EVERY == 0:
                torch.cuda.synchronize()
                solver.set_state(snap)
            with torch.cuda.stream(ext):
                flush.fill_(1.0)  # evict the previous step's matrices from L2
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(ext)
            rep = solver.step(cfl, mode=G.GMRES_CORRECT, m=m, restarts=200, rtol=rtol, precision=prec,
                              orth=ORTH[args.orth], warm_start=warm)
            with torch.cuda.stream(ext):
                e1.record(ext)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            res.append(rep["true_rel_res"])
            mvs.append(rep["matvecs"])
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        stats = solver.profile_read()
        solver.profile(False)
        total_s = max_over_ranks(sum(step_ms) / 1e3)
        # live roofline of the EBE element pass: one more step with the host-driven engine,
        # whose element passes are separate launches bracketed by CUDA events
        solver.profile(True)
        solver.step(cfl, mode=G.GMRES_CORRECT, m=m, restarts=200, rtol=rtol, precision=prec, engine=1)
        ebe = solver.profile_read()
        solver.profile(False)
        out[prec_name] = dict(steps_per_s=ws * steps / total_s, ms_per_step=1e3 * total_s / steps,
                              true_rel_res_max=max(res), matvecs_per_step=sum(mvs) / len(mvs), stats=stats,
                              ebe=ebe, state=solver.get_state(),
                              form_ms=stats["form_ms"] / max(stats["form_launches"], 1),
                              solve_ms=stats["solve_ms"] / max(stats["solves"], 1))
    out["sampler"] = sampler
    return out


def solve_roofline(r, peak, peak_kind, label, traffic=None):
    """The single-launch GMRES solve (the step's dominant kernel): algorithmic bytes of its
    products and Krylov passes over its CUDA-event time."""
    st = r["stats"]
    if st["solve_ms"] <= 0 or st["solves"] == 0:
        return None
    achieved = st["solve_bytes"] / (st["solve_ms"] / 1e3) / 1e9
    return {"kernel": label, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "bytes_per_launch": st["solve_bytes"] / st["solves"], "launches": st["solves"],
            "avg_launch_us": 1e3 * st["solve_ms"] / st["solves"]}


class MemPeak:
    """Device memory in use (total - free, every process on the GPU), sampled every 50 ms."""

    def __init__(self):
        import torch
        self.torch, self.peak, self.run = torch, 0, True
        self.t = threading.Thread(target=self._loop, daemon=True)
        self.t.start()

    def _loop(self):
        while self.run:
            free, total = self.torch.cuda.mem_get_info()
            self.peak = max(self.peak, total - free)
            time.sleep(0.05)

    def stop(self):
        self.run = False
        self.t.join()
        return self.peak


def measure_adjoint(args, ws, max_over_ranks):
    """Discrete adjoint on the O-grid cylinder: forward run with checkpoints, reverse sweep;
    device time of each phase from the library's own CUDA events."""
    from cfdv_b200 import gpu as G, meshgen as mg
    case = mg.cylinder(96, 128, 16)
    s = G.FDVSolver(case)
    k = args.adj_every
    out = {"workload": f"3D cylinder O-grid 96x128x16 hex8 ({case.n_elements} elements), M=0.3, Re=150, isothermal "
                       "wall; J = mean_n wall x-force; gradient w.r.t. Mach, wall temperature and each wall-node "
                       "temperature", "elements": case.n_elements, "steps": args.adj_steps,
           "checkpoint_every": k, "gmres": "GMRES(40) to 1e-8 (forward, tangent and adjoint solves)",
           "deviations": ADJOINT_DEVIATIONS + ([] if (args.adj_steps, k) == (1000, 50) else
                                              [f"{args.adj_steps} steps with checkpoints every {k} (the configuration: "
                                               "1000 steps, every 50)"])}
    for name, prec in (("fp64", G.PREC_FP64), ("mixed", G.PREC_MIXED)):
        s.load_node_records()
        s.adjoint(2, 0.5, checkpoint_every=1, m=40, rtol=1e-8, precision=prec)  # warm-up
        s.load_node_records()
        mem = MemPeak()
        r = s.adjoint(args.adj_steps, 0.5, checkpoint_every=k, m=40, rtol=1e-8, precision=prec)
        peak_bytes = mem.stop()
        f, b = max_over_ranks(r["forward_ms"]), max_over_ranks(r["backward_ms"])
        out[name] = {"forward_ms_per_step": f / args.adj_steps, "backward_ms_per_step": b / args.adj_steps,
                     "backward_over_forward": b / f, "forward_matvecs": r["forward_matvecs"],
                     "adjoint_matvecs": r["adjoint_matvecs"], "J": r["J"], "dJ_dmach": r["dJ_dmach"],
                     "dJ_dtwall": r["dJ_dtwall"], "wall_nodes": int(len(r["wall_nodes"])),
                     "kept_matrix_sets": r["kept_matrix_sets"], "reverse_forms": r["reverse_forms"],
                     "device_memory_peak_gb": peak_bytes / 1e9}
    s.close()
    return out


def matvec_roofline(r, peak, peak_kind, label):
    """The whole EBE product (element pass + node pass: gather, multiply, scatter) of the
    host-driven step's products: E*Ke^2*s_R + DOF*(8 + 8) bytes each over their device time."""
    e = r["ebe"]
    if e.get("matvec_ms", 0) <= 0 or e["launches"] == 0:
        return None
    achieved = e["matvec_bytes"] / (e["matvec_ms"] / 1e3) / 1e9
    return {"kernel": label, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "bytes_per_launch": e["matvec_bytes"] / e["launches"],
            "launches": e["launches"], "avg_us": 1e3 * e["matvec_ms"] / e["launches"]}


def summarize(sec, name, steps, warmup, peak, peak_kind, tile=None):
    """One more workload beside the headline: both forms, their ratio and rooflines."""
    s_m, s_f = sec["mixed"], sec["fp64"]
    return {
        "workload": sec["desc"], "elements": sec["case"].n_elements,
        "dof": sec["case"].n_nodes * sec["case"].neqn, "steps": steps, "warmup": warmup,
        "deviations": WORKLOADS[name]["deviations"],
        "mixed": {"value": s_m["steps_per_s"], "ms_per_step": s_m["ms_per_step"],
                  "true_rel_res_max": s_m["true_rel_res_max"], "matvecs_per_step": s_m["matvecs_per_step"],
                  "form_ms": s_m["form_ms"], "solve_ms": s_m["solve_ms"]},
        "fp64": {"value": s_f["steps_per_s"], "ms_per_step": s_f["ms_per_step"],
                 "true_rel_res_max": s_f["true_rel_res_max"], "matvecs_per_step": s_f["matvecs_per_step"],
                 "form_ms": s_f["form_ms"], "solve_ms": s_f["solve_ms"]},
        "mixed_over_fp64": s_m["steps_per_s"] / s_f["steps_per_s"],
        "roofline": solve_roofline(s_m, peak, peak_kind, "gmres_persistent_kernel, mixed (" + name + ")", tile),
        "roofline_ebe": ebe_roofline(s_m, peak, peak_kind, "ebe_elem_kernel, FP32 matrices (" + name + ")"),
        "roofline_ebe_fp64": ebe_roofline(s_f, peak, peak_kind, "ebe_elem_kernel, FP64 matrices (" + name + ")"),
        "roofline_matvec": matvec_roofline(s_m, peak, peak_kind, "EBE product, element + node pass, FP32 matrices"),
        "roofline_matvec_fp64": matvec_roofline(s_f, peak, peak_kind,
                                                "EBE product, element + node pass, FP64 matrices"),
    }


def ebe_roofline(r, peak, peak_kind, label, traffic=None):
    e = r["ebe"]
    if e["total_ms"] <= 0 or e["launches"] == 0:
        return None
    achieved = e["bytes"] / (e["total_ms"] / 1e3) / 1e9
    return {"kernel": label, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "bytes_per_launch": e["bytes"] / e["launches"], "launches": e["launches"],
            "avg_launch_us": 1e3 * e["total_ms"] / e["launches"]}


def bench_gpu(args, ws, rank, local):
    import numpy as np
    import torch
    from cfdv_b200 import gpu as G

    torch.cuda.set_device(local)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ranks = Ranks(ws, "cuda")
    barrier, max_over_ranks = ranks.barrier, ranks.max

    peak, peak_kind = peaks()
    sampler = ClockSampler(local)
    if args.only == "adjoint":  # profiling runs of the adjoint leg alone
        out = measure_adjoint(args, ws, max_over_ranks)
        if rank == 0:
            print(json.dumps(out))
        return
    head = measure_workload(args, args.workload, args.steps, args.warmup, flush, ws, barrier, max_over_ranks, sampler)
    solver, case = head["solver"], head["case"]
    if args.only:  # profiling runs: one form, no end-to-end loop, no JSON line
        sampler.stop()
        solver.close()
        if rank == 0:
            r = head[args.only]
            print(json.dumps({"form": args.only, "steps_per_s": r["steps_per_s"], "ms_per_step": r["ms_per_step"],
                              "true_rel_res_max": r["true_rel_res_max"], "matvecs_per_step": r["matvecs_per_step"],
                              "form_ms": r["form_ms"], "solve_ms": r["solve_ms"], "ebe": r["ebe"]}))
        return

    # end-to-end through the C ABI with host buffers: H2D state, step, D2H state every step
    m, cfl, rtol, ext = head["m"], head["cfl"], head["rtol"], head["ext"]
    n = solver.n_dof
    host = torch.empty(n, dtype=torch.float64, pin_memory=True)
    outb = torch.empty(n, dtype=torch.float64, pin_memory=True)
    solver.load_node_records()
    host.numpy()[:] = solver.get_state()
    solver.profile(True)
    for _ in range(2):
        solver.step_host(cfl, host.numpy(), outb.numpy(), mode=G.GMRES_CORRECT, m=m, restarts=200, rtol=rtol,
                         precision=G.PREC_MIXED, orth=ORTH[args.orth])
        host.copy_(outb)
    torch.cuda.synchronize()
    barrier()
    solver.profile(True)
    e2e_ms = []
    snap = host.numpy().copy()
    for i in range(args.steps):
        if i and i % RESTART_EVERY == 0:
            host.numpy()[:] = snap
        with torch.cuda.stream(ext):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
        # H2D of the state, the step, D2H of the new state: one C ABI call, one host wait
        solver.step_host(cfl, host.numpy(), outb.numpy(), mode=G.GMRES_CORRECT, m=m, restarts=200, rtol=rtol,
                         precision=G.PREC_MIXED, orth=ORTH[args.orth])
        with torch.cuda.stream(ext):
            e1.record(ext)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        host.copy_(outb)
    launches_per_step = solver.profile_read()["kernel_launches"] / args.steps
    solver.profile(False)
    clocks = sampler.stop()
    e2e_s = max_over_ranks(sum(e2e_ms) / 1e3)
    solver.close()

    mixed, fp64 = head["mixed"], head["fp64"]
    err = float(np.abs(mixed["state"] - fp64["state"]).max() / np.abs(fp64["state"]).max())
    # per conserved field: max |U_mixed - U_fp64| / max |U_fp64| over the nodes
    neq = case.neqn
    names = ["rho", "rho_u", "rho_v", "rho_w", "rho_E"] if neq == 5 else ["rho", "rho_u", "rho_v", "rho_E"]
    per_field = {nm: float(np.abs(mixed["state"][k::neq] - fp64["state"][k::neq]).max() /
                           max(np.abs(fp64["state"][k::neq]).max(), 1e-300)) for k, nm in enumerate(names)}
    traffic = None
    # DRAM bytes per launch of the solve kernel from an ncu capture (profiles/*.md)
    tfile = os.path.join(ROOT, "profiles", "solve_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            traffic = json.load(f).get(args.workload)
    line = {
        "metric": METRIC,
        "value": mixed["steps_per_s"],
        "unit": "FDV steps/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": mixed["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 matrices/f64 vectors (mixed); f64",
        "data": "synthetic",
        "config": {"workload": head["desc"], "elements": case.n_elements, "dof": n,
                   "gmres": f"restarted GMRES({m}), {args.orth.upper()}, right node-block Jacobi, to true relative "
                            f"residual {rtol:g}",
                   "initial_guess": "the previous step's dU" if args.warm_start else "zero (as the reference)",
                   "l2": "flushed between timed steps (512 MiB write)", "parallelism": f"replicas x{ws}",
                   "deviations": WORKLOADS[args.workload]["deviations"]},
        "fp64": {"value": fp64["steps_per_s"], "ms_per_step": fp64["ms_per_step"],
                 "true_rel_res_max": fp64["true_rel_res_max"], "matvecs_per_step": fp64["matvecs_per_step"],
                 "form_ms": fp64["form_ms"], "solve_ms": fp64["solve_ms"]},
        "mixed": {"true_rel_res_max": mixed["true_rel_res_max"], "matvecs_per_step": mixed["matvecs_per_step"],
                  "form_ms": mixed["form_ms"], "solve_ms": mixed["solve_ms"], "max_field_diff_vs_fp64": err,
                  "field_diff_vs_fp64": per_field,
                  "after_steps": args.warmup + args.steps},
        "mixed_over_fp64": mixed["steps_per_s"] / fp64["steps_per_s"],
        "roofline": solve_roofline(mixed, peak, peak_kind,
                                   "gmres_persistent_kernel, mixed (" + args.workload + "; data L2-resident)"
                                   if args.workload in ("plate", "lid") else
                                   "gmres_persistent_kernel, mixed (" + args.workload + ")", traffic),
        "roofline_ebe": ebe_roofline(mixed, peak, peak_kind, "ebe_elem_kernel, FP32 matrices (" + args.workload + ")"),
        "roofline_ebe_fp64": ebe_roofline(fp64, peak, peak_kind,
                                          "ebe_elem_kernel, FP64 matrices (" + args.workload + ")"),
        "roofline_matvec": matvec_roofline(mixed, peak, peak_kind, "EBE product, element + node pass, FP32 matrices"),
        "roofline_matvec_fp64": matvec_roofline(fp64, peak, peak_kind,
                                                "EBE product, element + node pass, FP64 matrices"),
        "e2e": {"value": ws * args.steps / e2e_s, "unit": "FDV steps/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "clocks": clocks,
    }
    del head
    tiles = {}
    if os.path.exists(tfile):
        with open(tfile) as f:
            tiles = json.load(f)
    if args.secondary in WORKLOADS and args.secondary != args.workload:
        sec = measure_workload(args, args.secondary, 3, 3, flush, ws, barrier, max_over_ranks)
        sec["solver"].close()
        line["secondary"] = summarize(sec, args.secondary, 3, 3, peak, peak_kind, tiles.get(args.secondary))
        del sec
    for name in [w for w in args.extra.split(",") if w in WORKLOADS and w not in (args.workload, args.secondary)]:
        k, w = (10, 3) if name == "lid" else (3, 3)
        ex = measure_workload(args, name, k, w, flush, ws, barrier, max_over_ranks)
        ex["solver"].close()
        line[name] = summarize(ex, name, k, w, peak, peak_kind, tiles.get(name))
        del ex
    if not args.warm_start and args.secondary != "none":
        # the same workloads with each solve started from the previous step's dU (the same
        # stopping test); the headline above starts from zero, as the reference does
        warm = {"initial_guess": "the previous step's dU", "note": "same stopping test; headline starts from zero"}
        for name, k, w in ((args.workload, args.steps, args.warmup), (args.secondary, 3, 3)):
            if name not in WORKLOADS:
                continue
            r = measure_workload(args, name, k, w, flush, ws, barrier, max_over_ranks, warm=True)
            r["solver"].close()
            warm[name] = {f: {"value": r[f]["steps_per_s"], "matvecs_per_step": r[f]["matvecs_per_step"],
                              "true_rel_res_max": r[f]["true_rel_res_max"], "solve_ms": r[f]["solve_ms"]}
                          for f in ("mixed", "fp64") if f in r}
            del r
        line["warm_start"] = warm
    if args.adj_steps > 0:
        line["adjoint"] = measure_adjoint(args, ws, max_over_ranks)
    if rank == 0:
        if not args.no_cpu_baseline:
            # the same sample as the reference arm's default: warm-up steps, then timed steps
            k, w = CPU_SAMPLE.get(args.workload, (2, 1))
            from cfdv_b200 import meshgen as mg
            times = run_reference_cpu(WORKLOADS[args.workload]["make"](mg), k, w)
            line["cpu_baseline"] = {"value": k / sum(times), "unit": "FDV steps/s", "cores": 1, "kind": "reference",
                                    "cpu": cpu_model(),
                                    "sample": f"{k} timed steps after {w} warm-up steps of the same case through "
                                              f"oracle/_ref/cfdv_ref (reference sources, 1 core, the reference's "
                                              f"GMRES({m}) with one restart: not equal residual)"}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def bench_reference(args, ws, rank):
    if rank != 0:
        return
    from cfdv_b200 import meshgen as mg
    W = WORKLOADS[args.workload]
    case = W["make"](mg)
    times = run_reference_cpu(case, args.steps, args.warmup)
    v = args.steps / sum(times)
    line = {
        "metric": METRIC, "impl": "reference", "value": v, "unit": "FDV steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": W["desc"], "elements": case.n_elements, "dof": case.n_nodes * case.neqn,
                   "gmres": f"reference MPI_GMRES({W['m']}), 1 restart (its own stopping rule)"},
        "cpu_baseline": {"value": v, "unit": "FDV steps/s", "cores": 1, "kind": "reference", "cpu": cpu_model(),
                         "sample": f"{args.steps} timed steps after {args.warmup} warm-up steps of the full case"},
        "e2e": {"value": v, "unit": "FDV steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cfdv_b200", choices=["cfdv_b200", "reference"])
    ap.add_argument("--workload", default="plate", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", choices=["fp64", "mixed", "adjoint"], help="time one form or the adjoint leg only "
                                                                         "(profiling runs)")
    ap.add_argument("--secondary", default="ramp", help="second workload reported beside the headline ('none' to skip)")
    ap.add_argument("--warm-start", action="store_true",
                    help="start each step's solve from the previous step's dU instead of zero (the same 1e-8 "
                         "stopping test)")
    ap.add_argument("--adj-steps", type=int, default=4, help="steps of the adjoint leg on the cylinder (0 to skip)")
    ap.add_argument("--adj-every", type=int, default=2, help="checkpoint spacing of the adjoint leg")
    ap.add_argument("--extra", default="lid,duct", help="further workloads reported beside the headline "
                                                         "(comma-separated; 'none' to skip)")
    ap.add_argument("--orth", default="dcgs2", choices=sorted(ORTH), help="Gram-Schmidt of the persistent GMRES solve")
    args = ap.parse_args()
    ws, rank, local = dist_info()
    if args.impl == "reference":
        bench_reference(args, ws, rank)
    else:
        bench_gpu(args, ws, rank, local)


if __name__ == "__main__":
    main()
