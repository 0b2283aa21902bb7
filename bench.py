"""Benchmark: capacitance solves/s on the 256x256x128 8-terminal extraction.

One step = one full Maxwell capacitance extraction of the layered-dielectric,
8-conductor-box workload (256x256x128 nodes, 10 nm pitch, grounded bottom
plane, 8 right-hand sides solved to FP64 relres 1e-10): edge masses built on
the device, Dirichlet elimination, block CG, FP64 charge integration.

* ``value``  -- solves/s with inputs (permittivity, terminal node lists)
  already in HBM when the timed region starts.
* ``e2e``    -- solves/s through the public API
  ``fieldspice_b200.extraction.capacitance_matrix`` with host inputs in
  pinned memory; host->device copies and the C-matrix readback are inside
  the timed region.
* ``roofline`` -- the dominant CG kernel's algorithmic bytes per launch over
  its CUDA-event duration sampled inside the timed region, against the
  measured HBM copy bandwidth.
* ``cpu_baseline`` -- the CPU oracle (SciPy Jacobi-CG, the reference's
  algorithm) timed on a bounded sample of the same workload.

Multi-GPU: one process per GPU (torchrun); every rank extracts its own
geometry (seed = rank), no data-path collective ("scaling": "weak");
timing is the max over ranks.  ``--impl reference`` times the CPU oracle
(the reference's algorithm) on the host cores instead.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHAPE = (256, 256, 128)
NBOX = 8
TOL = 1e-10
FULLSIZE_JSON = ROOT / "tests" / "golden" / "layered_256x256x128_s0.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # defaults: 20 timed steps after 5 warm-up ones for this implementation;
    # 5 after 3 for the reference arm, whose every step is a ~14 s call
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "mixed", "fp64"])
    ap.add_argument("--preconditioner", default="mg", choices=["mg", "jacobi"])
    ap.add_argument("--shape", default=",".join(map(str, SHAPE)))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--cpu-sample-iters", type=int, default=40)
    ap.add_argument("--unet-forward", action="store_true",
                    help="time the U-Net forward pass alone at the learned level of the "
                         "256x256x128 workload (64x64x32 nodes, 8 RHS), random weights")
    ap.add_argument("--single", action="store_true",
                    help="one device-resident extraction only (profiler runs)")
    args = ap.parse_args()
    ref = args.impl == "reference"
    if args.steps is None:
        args.steps = 5 if ref else 20
    if args.warmup is None:
        args.warmup = 3 if ref else 5
    return args


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """Per-node DRAM bytes of each kernel (by name) from the committed ncu
    summary: ``{"kernels": {name: {"bytes_per_node": ...}}}``."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        return json.loads(p.read_text()).get("kernels", {})
    return {}


def kernel_names(s: int, k: int, stencil_kind: int) -> dict:
    """The kernel each timed role runs as (template names as ncu lists them)."""
    t = "float" if s == 4 else "double"
    stencil = {4: "k_stencil_split", 3: "k_stencil_tma_s", 2: "k_stencil_tma_m",
               1: "k_stencil_tma"}.get(stencil_kind, "k_apply_pq")
    # the fused direction-update stencil carries its tile height (0: 32x8)
    pz = {5: 0, 6: 4, 7: 16}
    split = k * s == 32  # 32-byte nodes: the two-threads-per-node smoothing pass
    return {"stencil": (f"k_stencil_pz<{t}, {k}, {pz[stencil_kind]}>" if stencil_kind in pz
                        else f"{stencil}<{t}, {k}>"),
            "pupdate": f"k_pnew<{t}, {k}>",
            "update": f"k_update<{t}, {k}>",
            "smoother": (f"k_mg_smooth_split<{t}, {k}, 1>" if split
                         else f"k_mg_post_fused<{t}, {k}>")}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed regions.

    NVML queries take driver locks that this process's CUDA calls can wait
    on, so the sampler asks only for the six fields the bench line reports,
    every 500 ms (40 end-to-end extractions: worst call 57 ms against a
    47.7 ms median with this sampler running)."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 500

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[2:6]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


def e2e_phase_report(calls, allocs):
    """Per-phase host times of the end-to-end calls: the worst call (by wall
    time) and the median call, each phase's wall and process-CPU ms (wall
    well above CPU means the host thread waited: on the GPU, the driver or
    the OS), and the device allocations the call made."""
    def one(i):
        ph = calls[i]
        out = {"wall_ms": 1e3 * (ph[-1][1] - ph[0][1]),
               "cpu_ms": 1e3 * (ph[-1][2] - ph[0][2]), "phases": {}}
        for (_, w0, c0), (name, w1, c1) in zip(ph[:-1], ph[1:]):
            d = out["phases"].setdefault(name, [0.0, 0.0])
            d[0] += 1e3 * (w1 - w0)
            d[1] += 1e3 * (c1 - c0)
        out["phases"] = {k: [round(v[0], 3), round(v[1], 3)] for k, v in out["phases"].items()}
        slow = max(out["phases"], key=lambda k: out["phases"][k][0])
        out["slowest_phase"] = slow
        out["allocs"] = allocs[i] if i < len(allocs) else None
        out["summary"] = {"wall_ms": round(out["wall_ms"], 3), "cpu_ms": round(out["cpu_ms"], 3),
                          "slowest_phase": slow, "slowest_phase_ms": out["phases"][slow]}
        return out
    if not calls:
        return {"worst": None, "median": None}
    walls = [c[-1][1] - c[0][1] for c in calls]
    order = sorted(range(len(calls)), key=lambda i: walls[i])
    return {"worst": one(order[-1]), "median": one(order[len(order) // 2])}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def kernel_bytes(N: int, k: int, s: int, stencil_kind: int = 2) -> dict:
    """Algorithmic bytes per launch of the CG kernels (each array once)."""
    return {"pupdate": 3 * N * k * s,                 # read r|z, p_old; write p
            # read p, 3 masses; write q -- with the direction update inside
            # (kinds 5-7) read z and p_old, write p and q
            "stencil": N * ((4 if stencil_kind >= 5 else 2) * k * s + 3 * s),
            "update": 6 * N * k * s,                  # read p, q, x, r; write x, r
            # fine-level post-smoothing, one fused pass (k_mg_smooth_split):
            # read x, b and the masses; write x2 = x + a r0 + b A~r0
            "smoother": N * (3 * k * s + 3 * s)}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from fieldspice_b200 import device as D
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.poisson import capacitance_report, extract_capacitance

    shape = tuple(int(v) for v in args.shape.split(","))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = W.layered_boxes(shape, nbox=NBOX, seed=rank)
    grid = w.grid()
    bc = w.boundary_spec()
    terms = w.terminal_objects()
    # device-resident inputs for `value`
    eps_dev = torch.as_tensor(w.eps_cell, device=dev)
    term_dev = [torch.as_tensor(np.asarray(t, np.int64), device=dev) for t in w.terminals]
    from fieldspice_b200.boundaries import dirichlet_nodes
    wall = dirichlet_nodes(bc, grid)[0].astype(np.int64)
    shield = np.setdiff1d(wall, np.concatenate(w.terminals)).astype(np.int64)
    wall_dev = torch.as_tensor(wall, device=dev)
    shield_dev = torch.as_tensor(shield, device=dev)
    # pinned host inputs for `e2e`
    eps_pinned = torch.from_numpy(np.ascontiguousarray(w.eps_cell)).pin_memory().numpy()
    for t in terms:
        t.nodes = torch.from_numpy(np.ascontiguousarray(t.nodes, dtype=np.int64)).pin_memory().numpy()

    def step_device(precision, pc=args.preconditioner, learned=None):
        op = D.DeviceOperator(grid, eps_dev)
        C, qs, info = extract_capacitance(op, term_dev, wall_dev, shield_dev,
                                          tol=TOL, precision=precision,
                                          preconditioner=pc, learned=learned)
        info["gpu_launches"] += 1 + 2  # mass build + plan setup kernels
        return C, qs, info

    e2e_phases = []  # per e2e call: [(phase, wall s, CPU s)] from the library's marks
    alloc_stats = []  # per e2e call: device allocations and allocator retries

    def step_e2e(precision):
        rep = {}
        m0 = torch.cuda.memory_stats()
        D.PHASES = [("start", time.perf_counter(), time.process_time())]
        C = EX.capacitance_matrix(grid, eps_pinned, terms, bc, SolverConfig(tol=TOL),
                                  report=rep, gpu=GPUConfig(precision=precision,
                                                            preconditioner=args.preconditioner))
        D.mark("return")
        e2e_phases.append(D.PHASES)
        D.PHASES = None
        m1 = torch.cuda.memory_stats()
        alloc_stats.append({k: m1.get(k, 0) - m0.get(k, 0)
                            for k in ("num_device_alloc", "num_device_free", "num_alloc_retries")})
        return C, rep

    def barrier():
        if world > 1:
            dist.barrier()

    step_wall_ms = []  # host wall time of each timed step (the last timed() call)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            out = fn()
        barrier()
        torch.cuda.synchronize()
        stream = torch.cuda.current_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        outs = []
        step_wall_ms.clear()
        e0.record(stream)
        for _ in range(steps):
            t0 = time.perf_counter()
            outs.append(fn())
            step_wall_ms.append(1e3 * (time.perf_counter() - t0))
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, outs

    if args.single:
        for i in range(args.warmup + args.steps):
            last = i == args.warmup + args.steps - 1
            if last:  # the range a profiler can select: one steady-state extraction
                torch.cuda.nvtx.range_push("extraction")
            C, qs, info = step_device(args.precision)
            if last:
                torch.cuda.synchronize()
                torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"single": True, "shape": shape, "iterations": info["iterations"],
                              "reliable_updates": info.get("reliable_updates"),
                              "kernel_ms": info["kernel_ms"],
                              "gpu_launches": info["gpu_launches"]}), flush=True)
        return

    # clocks sampled over both timed regions (device-resident and end to end)
    sampler = ClockSampler(local_rank)
    sampler.start()
    ms_dev, outs = timed(lambda: step_device(args.precision), args.steps, args.warmup)
    C, qs, info = outs[-1]
    launches = sum(o[2]["gpu_launches"] for o in outs)
    k_rhs = NBOX
    n_solves_step = k_rhs * world
    value = n_solves_step * args.steps / (ms_dev / 1000.0)

    D.TRANSFERS.update(h2d=0, d2h=0)
    ms_e2e, outs_e2e = timed(lambda: step_e2e(args.precision), args.steps, 1)
    # every public call ends with C on the host, so each step's host wall time
    # is that call's end-to-end time: the median and the worst show whether a
    # few steps (the host thread off-CPU) set the mean
    e2e_steps = sorted(step_wall_ms)
    h2d = D.TRANSFERS["h2d"] / (args.steps + 1)
    d2h = D.TRANSFERS["d2h"] / (args.steps + 1)
    e2e_value = n_solves_step * args.steps / (ms_e2e / 1000.0)
    clocks = sampler.stop()
    timed_calls = e2e_phases[-args.steps:]
    timed_allocs = alloc_stats[-args.steps:]
    e2e_detail = e2e_phase_report(timed_calls, timed_allocs)

    variants = {}
    if not args.no_variants:
        nv = max(2, args.steps // 2)
        runs = []
        if args.preconditioner == "mg":
            runs.append(("plain_pcg_jacobi", args.precision, "jacobi"))
        other = "fp64" if args.precision != "fp64" else "mixed"
        runs.append((f"{args.preconditioner}_{other}", other, args.preconditioner))
        for name, prec, pc in runs:
            ms_o, outs_o = timed(lambda: step_device(prec, pc), nv, 1)
            Co = outs_o[-1][0]
            variants[name] = {
                "value": n_solves_step * nv / (ms_o / 1000.0),
                "ms_per_step": ms_o / nv,
                "precision": prec, "preconditioner": pc,
                "iterations": outs_o[-1][2]["iterations"],
                "C_rel_diff_vs_default": float(np.abs(Co - C).max() / np.abs(np.diag(C)).max()),
            }

    if not args.no_variants and world == 1:
        variants["batch64"] = batch_variant(timed)
        variants["learned_fcg"] = learned_variant(timed, step_device, C, args)
        variants["eqs_transient"] = eqs_variant()
        variants["field_region"] = field_region_variant()
        variants["rlgc_2d"] = rlgc_variant()
        variants["ac_admittance"] = ac_variant()

    if rank != 0:
        return
    N = int(np.prod(shape))
    s = 8 if (args.precision == "fp64" or info.get("fp64_fallback")) else 4
    km = info["kernel_ms"]
    kb = kernel_bytes(N, 8, s, km.get("stencil_kind", 2))
    names = kernel_names(s, 8, km.get("stencil_kind", 2))
    times = {"pupdate": km["pupdate_ms"], "stencil": km["stencil_ms"],
             "update": km["update_ms"]}
    if args.preconditioner == "mg":
        times["smoother"] = km["smoother_ms"]
    dom = max(times, key=times.get)
    peak, peak_kind = measured_peaks()
    gbs = {k: kb[k] / (times[k] * 1e-3) / 1e9 for k in times if times[k] > 0}
    traffic = committed_traffic().get(names[dom], {}).get("bytes_per_node")
    rep = capacitance_report(C, qs, info)
    # parity against the committed full-size oracle result (same seed-0 input)
    err_vs_oracle = None
    if FULLSIZE_JSON.exists() and rank == 0 and shape == SHAPE:
        ref = json.loads(FULLSIZE_JSON.read_text())
        Cref = np.asarray(ref["C_tol1e-12_unsymmetrised"])
        err_vs_oracle = float(np.abs(C - Cref).max() / np.abs(np.diag(Cref)).max())
    line = {
        "metric": "C solves/s @relres 1e-10",
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_dev / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if s == 8 else "f32+f64",
        "data": "synthetic (seeded layered dielectric + 8 conductor boxes per rank)",
        "config": {
            "workload": f"layered_boxes {shape[0]}x{shape[1]}x{shape[2]} nodes, "
                        f"{NBOX} terminals, zlo grounded, seed=rank",
            "nodes": N, "nrhs": NBOX, "tol": TOL, "precision": args.precision,
            "fp64_fallback": info.get("fp64_fallback"),
            "preconditioner": ("mg (geometric multigrid V-cycle, Chebyshev smoothing)"
                               if args.preconditioner == "mg" else "jacobi (equilibrated CG)"),
            "l2": "inputs larger than L2: every CG vector is N*8*4 B = 268 MB",
            "parallelism": f"dp{world} (independent geometries)",
        },
        "e2e": {"value": e2e_value, "unit": "solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": ms_e2e / args.steps,
                "step_ms_median": e2e_steps[len(e2e_steps) // 2] if e2e_steps else None,
                "step_ms_max": e2e_steps[-1] if e2e_steps else None,
                "worst_call": e2e_detail["worst"]["summary"] if e2e_detail["worst"] else None},
        "roofline": {
            "bound": "hbm", "kernel": names[dom], "role": dom, "achieved": gbs.get(dom),
            "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s",
            "frac": (gbs.get(dom) or 0.0) / peak,
            "traffic": (traffic * N if traffic else None),
            "algorithmic_bytes_per_launch": kb[dom],
            "ms_per_launch": times[dom], "samples": km["samples"],
            "precond_ms_per_iteration": km.get("precond_ms"),
        },
        "stencil_gbs": gbs.get("stencil"),
        "gpu_launches": int(launches),
        "clocks": clocks,
        "iterations": info["iterations"],
        "reliable_updates": info.get("reliable_updates"),
        "plan_setup_ms": 1e3 * info.get("setup_time", 0.0),
        "relres_fp64_max": info["residual"],
        "asymmetry_rel": rep["asymmetry_rel"],
        "C_err_vs_fp64_oracle": err_vs_oracle,
    }
    line.update(variant_scalars(variants))
    if args.preconditioner == "mg":
        line["mg_value"] = value
        if line["learned_value"]:
            line["learned_vs_mg"] = line["learned_value"] / value
    if line["learned_value"] and line["plain_pcg_value"]:
        line["learned_vs_plain_pcg"] = line["learned_value"] / line["plain_pcg_value"]
    if world == 1 and not args.no_cpu_baseline:
        jac = variants.get("plain_pcg_jacobi", {}).get("iterations")
        line["cpu_baseline"] = cpu_baseline(shape, jac, max(2, args.cpu_sample_iters // NBOX))
    # the variants and the e2e phase record in full on their own line first;
    # the headline line last
    print(json.dumps({"variants": variants, "e2e_calls": e2e_detail,
                      "roofline_all_kernels": {"gbs": gbs, "ms": times}}), flush=True)
    print(json.dumps(line), flush=True)


def variant_scalars(v: dict) -> dict:
    """The variants' headline figures as top-level scalars of the bench line."""
    def get(name, key="value"):
        return (v.get(name) or {}).get(key)
    out = {"mg_value": None, "plain_pcg_value": get("plain_pcg_jacobi"),
           "fp64_mg_value": get("mg_fp64"),
           "learned_value": get("learned_fcg"),
           "learned_iterations_max": max(get("learned_fcg", "iterations") or [0]) or None,
           "learned_vs_plain_pcg": None, "learned_vs_mg": None,
           "batch64_value": get("batch64"),
           "batch64_C_err_vs_oracle_max": get("batch64", "C_err_vs_oracle_max"),
           "eqs_steps_per_s": get("eqs_transient"),
           "eqs_current_err_vs_oracle_max": get("eqs_transient", "current_err_vs_oracle_max"),
           "eqs_iterations_per_step": get("eqs_transient", "iterations_per_step_mean"),
           "eqs_fp64_fallback": get("eqs_transient", "fp64_fallback")}
    return out


EPOCHS = 5
LEVEL = 3


def learned_variant(timed, step_device, C_default, args):
    """The learned preconditioner (U-Net coarse-level correction inside
    flexible CG) on this workload: trained here on 4096 residual-to-error
    pairs from Jacobi-PCG iterates on 64 seeded 128^3 geometries of the same
    family (seeds disjoint from the timed one), then timed like the default
    extraction.  Reports solves/s, iterations, training cost, and the same
    extraction with the network's output zeroed (what the network gains)."""
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.learned import LearnedPreconditioner
    t0 = time.perf_counter()
    train = [W.layered_boxes((128, 128, 128), nbox=NBOX, seed=1000 + s) for s in range(64)]
    net = LearnedPreconditioner.train(train, level=LEVEL, epochs=EPOCHS, batch=8, lr=1e-3,
                                      seed=0, mode="replace")
    t_train = time.perf_counter() - t0
    nv = max(2, args.steps // 2)
    ms, outs = timed(lambda: step_device("mixed", "learned", net), nv, 1)
    Cl, _, info = outs[-1]
    ms0, outs0 = timed(lambda: step_device("mixed", "learned", net.zero()), 1, 0)
    # the same V-cycle with its own multigrid recursion below the network's
    # level: plain multigrid PCG, the honest "method without the network"
    ms_mg, outs_mg = timed(lambda: step_device("mixed", "mg"), nv, 1)
    scale = float(np.abs(np.diag(C_default)).max())
    err = None
    if FULLSIZE_JSON.exists() and tuple(int(v) for v in args.shape.split(",")) == SHAPE:
        ref = json.loads(FULLSIZE_JSON.read_text())
        Cref = np.asarray(ref["C_tol1e-12_unsymmetrised"])
        err = float(np.abs(Cl - Cref).max() / np.abs(np.diag(Cref)).max())
    return {"value": NBOX / (ms / nv / 1000.0), "ms_per_step": ms / nv,
            "iterations": info["iterations"], "learned_fallback": info.get("learned_fallback"),
            "relres_fp64_max": info["residual"],
            "C_err_vs_fp64_oracle": err,
            "C_rel_diff_vs_default": float(np.abs(Cl - C_default).max() / scale),
            "kernel_ms": info["kernel_ms"],
            "mode": f"replace: V-cycle smoothing on levels 0-{LEVEL - 1}, the network's "
                    f"output as the level-{LEVEL} correction",
            "network_zeroed": {"value": NBOX / (ms0 / 1000.0),
                               "iterations": outs0[-1][2]["iterations"]},
            "multigrid_recursion": {"value": NBOX / (ms_mg / nv / 1000.0),
                                    "iterations": outs_mg[-1][2]["iterations"],
                                    "precond_ms": outs_mg[-1][2]["kernel_ms"]["precond_ms"]},
            "vs_multigrid_recursion": (NBOX / (ms / nv / 1000.0)) / (NBOX / (ms_mg / nv / 1000.0)),

            "training": {"pairs": net.pairs, "geometries": len(train), "shape": [128, 128, 128],
                         "level": net.level, "epochs": EPOCHS, "batch": 8,
                         "data_seconds": net.data_time, "fit_seconds": net.train_time,
                         "total_seconds": t_train,
                         "loss_first": net.history[0] if net.history else None,
                         "loss_last": net.history[-1] if net.history else None}}


def eqs_variant(shape=(192, 192, 96), steps=200):
    """Backward-Euler EQS transient: copper boxes in oxide over doped
    silicon, two ports driven by a 1 V ramp (10 ps rise), dt = 1 ps, 200
    steps.  The default path (mixed precision, multigrid, warm-started steps)
    against the same transient in FP64 at relres 1e-12 (the FP64 reference
    method): per-step port-current error and time per step."""
    import torch
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    w = W.eqs_interconnect(shape, nbox=6, nports=2, seed=0)
    g = w.grid()
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", w.terminals[0], voltage=ramp),
             Terminal("port1", w.terminals[1], voltage=0.0)]
    bc = BoundarySpec(zlo=Dirichlet(0.0))

    def run(precision, tol):
        s = EQSSolver(g, w.eps_cell, w.sigma_cell, SolverConfig(tol=tol),
                      gpu=GPUConfig(precision=precision, preconditioner="mg"))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = s.solve(terms, t_end=steps * 1e-12, dt=1e-12, bc=bc)
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0
    r, t = run("auto", TOL)
    rf, tf = run("fp64", 1e-12)
    i0, i1 = np.asarray(r.i("port0")), np.asarray(r.i("port1"))
    f0, f1 = np.asarray(rf.i("port0")), np.asarray(rf.i("port1"))
    scale = max(np.abs(f0).max(), np.abs(f1).max())
    err = np.maximum(np.abs(i0 - f0), np.abs(i1 - f1)) / scale
    its = np.asarray(r.meta.get("iterations") or [0])
    out = {"metric": "EQS steps/s (192x192x96, 200 steps, dt 1 ps)",
           "value": steps / t, "seconds": t, "fp64_seconds": tf,
           "nodes": int(np.prod(shape)),
           "iterations_per_step_mean": float(its.mean()),
           "iterations_per_step_max": int(its.max()),
           "iterations_first_steps": [int(v) for v in its[:8]],
           "fp64_fallback": bool(r.meta.get("fp64_fallback")),
           "current_err_vs_fp64_max": float(err.max()),
           "current_err_vs_fp64_final": float(err[-1]),
           "per_step_err_quantiles": [float(np.quantile(err, q)) for q in (0.5, 0.9, 1.0)],
           "precision": "auto (mixed, FP64 continuation on stall)", "tol": TOL}
    out.update(eqs_vs_reference())
    return out


def eqs_vs_reference():
    """The same transient at the largest grid the reference itself finished
    here (tests/golden/eqs_<shape>_s0.npz, made by tests/golden/make_scale.py:
    the reference's EQSSolver, Jacobi-CG forced, tol 1e-12): port currents of
    the default GPU path against the reference's at every step."""
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    fx = sorted((ROOT / "tests" / "golden").glob("eqs_*x*x*_s0.npz"),
                key=lambda p: int(np.prod(np.load(p)["shape"])))
    if not fx:
        return {"current_err_vs_oracle_max": None}
    d = np.load(fx[-1])
    shape = tuple(int(v) for v in d["shape"])
    steps = int(d["steps"])
    w = W.eqs_interconnect(shape, nbox=6, nports=2, seed=0)
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", w.terminals[0], voltage=ramp),
             Terminal("port1", w.terminals[1], voltage=0.0)]
    s = EQSSolver(w.grid(), w.eps_cell, w.sigma_cell, SolverConfig(tol=TOL),
                  gpu=GPUConfig(precision="auto", preconditioner="mg"))
    r = s.solve(terms, t_end=steps * 1e-12, dt=1e-12, bc=BoundarySpec(zlo=Dirichlet(0.0)))
    i0, i1 = np.asarray(r.i("port0")), np.asarray(r.i("port1"))
    scale = max(np.abs(d["i0"]).max(), np.abs(d["i1"]).max())
    err = np.maximum(np.abs(i0 - d["i0"]), np.abs(i1 - d["i1"])) / scale
    return {"oracle_shape": list(shape), "oracle_steps": steps,
            "current_err_vs_oracle_max": float(err.max()),
            "current_err_vs_oracle_quantiles": [float(np.quantile(err, q))
                                                for q in (0.5, 0.9, 1.0)],
            "oracle": "reference EQSSolver, Jacobi-CG forced, tol 1e-12 (tests/golden)"}


def field_region_variant(shape=(128, 128, 64), steps=100, dt=1e-12):
    """A meshed EQS region as a netlist element (circuit/coupling.py): copper
    boxes in oxide over doped silicon, every box plus the bottom plane an
    electrode.  Time of the Schur-complement reduction at dt = 1 ps (one
    block solve of all unit excitations) and of the per-step device work
    (history solve, stamp, back-substitution) with the electrode voltages of
    a 10 ps ramp; Y and the history currents against the same region solved
    in FP64 at relres 1e-12."""
    import torch
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.circuit import FieldRegion
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    w = W.eqs_interconnect(shape, nbox=6, nports=6, seed=1)
    g = w.grid()
    nx, ny, nz = shape
    nid = np.arange(nx * ny * nz).reshape(shape)
    terms = [Terminal(f"box{i}", t) for i, t in enumerate(w.terminals)]
    terms.append(Terminal("sub", nid[:, :, 0].ravel()))
    names = [t.name for t in terms]
    nmap = {n: i for i, n in enumerate(names[:-1])}      # "sub" is ground
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)

    def run(precision, tol):
        fr = FieldRegion("FR", g, w.eps_cell, w.sigma_cell, terms,
                         circuit_nodes=names[:-1] + ["0"], config=SolverConfig(tol=tol),
                         gpu=GPUConfig(precision=precision, preconditioner="mg"))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Y = fr.terminal_admittance(dt).copy()
        torch.cuda.synchronize()
        t_red = time.perf_counter() - t0
        nE = len(names) - 1
        fs = []
        t0 = time.perf_counter()
        for k in range(1, steps + 1):
            G = np.zeros((nE, nE))
            I = np.zeros(nE)
            fr.stamp_tran(G, I, None, None, dt, nmap)
            fs.append(I.copy())
            x = np.zeros(nE)
            x[0] = ramp(k * dt)
            fr.accept_timestep(x, None, dt, nmap)
        torch.cuda.synchronize()
        t_steps = time.perf_counter() - t0
        fr.close()
        return Y, np.array(fs), t_red, t_steps
    Y, f, t_red, t_steps = run("auto", TOL)
    Yf, ff, t_redf, t_stepsf = run("fp64", 1e-12)
    return {"metric": f"field-region steps/s ({shape[0]}x{shape[1]}x{shape[2]}, "
                      f"{len(terms)} electrodes, dt 1 ps)",
            "value": steps / t_steps, "reduction_s": t_red, "steps": steps,
            "fp64_reduction_s": t_redf, "fp64_value": steps / t_stepsf,
            "Y_err_vs_fp64": float(np.abs(Y - Yf).max() / np.abs(Yf).max()),
            "f_eff_err_vs_fp64": float(np.abs(f - ff).max() / max(np.abs(ff).max(), 1e-300)),
            "nodes": int(np.prod(shape)), "tol": TOL}


def rlgc_variant(nx=1201, ny=801):
    """Per-unit-length RLGC of a coupled-microstrip cross-section
    (extraction.rlgc_2d): three 2-D extractions (dielectric, vacuum,
    conductivity) batched on one GPU with the semi-coarsened multigrid
    (x and y halved, the two z planes kept); C and L against the same call in
    FP64 at relres 1e-12."""
    import torch
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    w = W.cross_section(nx, ny, nlines=3, seed=0)
    g = w.grid()
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]

    def run(precision, tol):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = EX.rlgc_2d(g, w.eps_cell, w.sigma_cell, terms, config=SolverConfig(tol=tol),
                       gpu=GPUConfig(precision=precision, preconditioner="mg"))
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0
    run("auto", TOL)                      # warm-up (plans, allocator)
    times = []
    for _ in range(3):
        r, t = run("auto", TOL)
        times.append(t)
    t = float(np.median(times))
    rf, tf = run("fp64", 1e-12)
    return {"metric": f"rlgc_2d calls/s ({nx}x{ny}x2 nodes, 4 conductors)",
            "value": 1.0 / t, "seconds": t, "seconds_each": times, "fp64_seconds": tf,
            "C_err_vs_fp64": float(np.abs(r["C"] - rf["C"]).max() / np.abs(rf["C"]).max()),
            "L_err_vs_fp64": float(np.abs(r["L"] - rf["L"]).max() / np.abs(rf["L"]).max()),
            "Z0": [float(z) for z in r["Z0"]], "nodes": int(nx * ny * 2), "tol": TOL}


def ac_variant(shape=(128, 128, 64), freqs=(1e6, 1e9, 1e10)):
    """Harmonic EQS (solvers/ac.py): the 7x7 complex admittance of copper
    boxes in oxide over doped silicon (every box and the bottom plane a
    terminal) at three frequencies, each one complex-symmetric block solve
    (COCG with the multigrid V-cycle of |A| + |B|).  Accuracy: reciprocity
    of Y (the reference's own check) and row sums (no terminal current is
    lost: every wall insulating)."""
    import torch
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.ac import ACSolver
    from fieldspice_b200.solvers.base import Terminal
    w = W.eqs_interconnect(shape, nbox=6, nports=6, seed=2)
    g = w.grid()
    nx, ny, nz = shape
    nid = np.arange(nx * ny * nz).reshape(shape)
    terms = [Terminal(f"box{i}", t) for i, t in enumerate(w.terminals)]
    terms.append(Terminal("sub", nid[:, :, 0].ravel()))
    ac = ACSolver(g, w.eps_cell, w.sigma_cell)
    ac.admittance_matrix(terms, freqs[:1])            # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Y = ac.admittance_matrix(terms, freqs)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    asym = max(float(np.abs(y - y.T).max() / np.abs(y).max()) for y in Y)
    rows = max(float(np.abs(y.sum(axis=1)).max() / np.abs(np.diag(y)).max()) for y in Y)
    its = [[s["iterations"] for s in st] for st in ac.last_stats]
    return {"metric": f"AC admittance matrices/s ({shape[0]}x{shape[1]}x{shape[2]}, "
                      f"{len(terms)} terminals)",
            "value": len(freqs) / t, "seconds": t, "freqs": list(freqs),
            "iterations": its, "asymmetry_max": asym, "row_sum_rel_max": rows,
            "nodes": int(np.prod(shape))}


def batch_variant(timed):
    """64 uneven seeded geometries (32^3 .. 160x160x96 nodes, 2-16 terminals,
    eps_r from {2.5, 3.9, 7.0, 11.7}) extracted as one batch: C-matrices/s
    over the whole job (host set-up included), the same batch one geometry at
    a time, and each C against an FP64 multigrid solve at relres 1e-12."""
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.batch import capacitance_matrices
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    ws = W.batch_geometries(64, seed=0)
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    probs = [(w.grid(), w.eps_cell, [Terminal(n, t) for n, t in zip(w.names, w.terminals)], bc)
             for w in ws]
    cfg = SolverConfig(tol=TOL)
    gcfg = GPUConfig(precision="auto", preconditioner="mg")
    reps = [None] * len(probs)
    ms_b, outs = timed(lambda: capacitance_matrices(probs, cfg, gpu=gcfg, reports=reps), 1, 1)
    Cs = outs[-1]
    ms_s, _ = timed(lambda: [EX.capacitance_matrix(p[0], p[1], p[2], p[3], cfg, gpu=gcfg)
                             for p in probs], 1, 0)
    nodes = [int(np.prod(p[0].shape_nodes)) for p in probs]
    out = {"metric": "C-matrices/s (64 uneven geometries)",
           "value": len(probs) / (ms_b / 1000.0), "ms_per_batch": ms_b,
           "one_at_a_time_value": len(probs) / (ms_s / 1000.0),
           "solves_per_batch": int(sum(len(p[2]) for p in probs)),
           "nodes_total": int(sum(nodes)), "nodes_min": min(nodes), "nodes_max": max(nodes),
           "max_iterations": max(max(r["linear"]["iterations"]) for r in reps)}
    # each C against the reference's own extraction of the same geometry
    # (Jacobi-CG forced, tol 1e-12; tests/golden/batch64_s0.json from
    # tests/golden/make_scale.py)
    fx = ROOT / "tests" / "golden" / "batch64_s0.json"
    if fx.exists():
        ref = json.loads(fx.read_text())["geometries"]
        errs = [None if r is None else
                float(np.abs(C - np.asarray(r["C"])).max() / np.abs(np.diag(r["C"])).max())
                for C, r in zip(Cs, ref)]
        have = [e for e in errs if e is not None]
        out.update({"C_err_vs_oracle_max": max(have) if have else None,
                    "oracle_geometries": len(have),
                    "C_err_vs_oracle_per_geometry": errs,
                    "oracle": "reference PoissonSolver.capacitance_matrix, Jacobi-CG "
                              "forced, tol 1e-12 (tests/golden)"})
    return out


# ---------------------------------------------------------------------------
# CPU timing of the reference's own path (cpu_baseline and the reference arm)
# ---------------------------------------------------------------------------
REF_DIR = ROOT / "baseline" / "_ref"


def _reference_package():
    """The unmodified reference package installed in baseline/_ref, or None."""
    if not (REF_DIR / "fieldspice" / "__init__.py").is_file():
        return None
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import fieldspice
    # the solver modules probe scipy's CG signature when first imported:
    # import them before any bounded-CG context replaces the function
    import fieldspice.extraction  # noqa: F401
    import fieldspice.solvers.poisson  # noqa: F401
    return fieldspice


class _BoundedReferenceCG:
    """Context for a bounded sample of the reference's Jacobi-CG path.

    ``spilu`` raises, so ``LinearSystem`` takes its Jacobi-preconditioned
    CG branch (``fieldspice/solvers/poisson.py:472-484``; the incomplete-LU
    branch stalls on this system), and every ``scipy.sparse.linalg.cg``
    call the reference makes runs exactly ``sample`` iterations (relative
    tolerance 1e-300), timed.  The reference's own residual check, relative
    to a right-hand side that includes the unit Dirichlet rows, lets every
    right-hand side through, so one call runs all eight bounded solves (the
    resulting C is discarded)."""

    def __init__(self, sample: int):
        self.sample = sample
        self.cg_seconds: list[float] = []

    def __enter__(self):
        import scipy.sparse.linalg as spla
        self._spla = spla
        self._ilu, self._cg = spla.spilu, spla.cg
        orig_cg, sample, log = self._cg, self.sample, self.cg_seconds

        def no_ilu(*a, **k):
            raise MemoryError("incomplete LU disabled: Jacobi branch forced")

        def cg(A, b, **kw):
            if sample is not None:  # None: the reference's own stopping rule
                kw["maxiter"] = sample
                for key in ("rtol", "tol"):
                    if key in kw:
                        kw[key] = 1e-300
            t0 = time.perf_counter()
            out = orig_cg(A, b, **kw)
            log.append(time.perf_counter() - t0)
            return out
        spla.spilu, spla.cg = no_ilu, cg
        return self

    def __exit__(self, *exc):
        self._spla.spilu, self._spla.cg = self._ilu, self._cg
        return False


def _reference_iterations(shape, jacobi_iters=None):
    """Jacobi-CG iterations to 1e-10 of the 8 right-hand sides of ``shape``,
    and where they come from; (None, reason) when none are known."""
    if tuple(shape) == SHAPE and FULLSIZE_JSON.exists():
        d = json.loads(FULLSIZE_JSON.read_text())
        return [int(v) for v in d["iterations_1e-10"]], "oracle full-size run (tests/golden)"
    if jacobi_iters:
        return ([int(v) for v in jacobi_iters],
                "the GPU's Jacobi PCG of the same system (mixed precision; its FP64 "
                "iteration counts equal the reference's)")
    return None, f"no Jacobi-CG iteration counts recorded for {tuple(shape)}"


#: Below this many nodes a reference extraction runs to convergence in a few
#: seconds and is measured whole instead of projected.
WHOLE_REFERENCE_NODES = 1 << 17


def reference_sample(shape, sample_iters, seed=0):
    """One call of the reference's public ``extraction.capacitance_matrix``
    (``fieldspice/extraction.py:41-56``) on the seeded workload with the
    Jacobi branch forced and each right-hand side bounded to
    ``sample_iters`` CG iterations (None: the reference's own stopping rule,
    a whole extraction).  Returns (call seconds, seconds in CG, CG
    iterations run, 0 when unbounded)."""
    fs = _reference_package()
    from fieldspice.boundaries import BoundarySpec, Dirichlet
    from fieldspice.grid import RectilinearGrid
    from fieldspice.solvers.base import ConvergenceError, SolverConfig, Terminal
    from fieldspice_b200 import workloads as W
    w = W.layered_boxes(shape, nbox=NBOX, seed=seed)
    g = RectilinearGrid(w.x, w.y, w.z)
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    ctx = _BoundedReferenceCG(sample_iters)
    t0 = time.perf_counter()
    with ctx, warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        try:
            fs.extraction.capacitance_matrix(g, w.eps_cell, terms, bc,
                                             SolverConfig(linear_solver="cg", tol=TOL))
        except ConvergenceError:
            pass
    n_cg = sample_iters * len(ctx.cg_seconds) if sample_iters else 0
    return time.perf_counter() - t0, sum(ctx.cg_seconds), n_cg


def _project(t_call, t_cg, n_cg, iters):
    """Extraction time of the reference = everything outside CG in the
    sampled call (assembly, elimination, equilibration, each right-hand
    side's set-up and charge integration) plus the measured seconds per CG
    iteration times the iterations each of the eight right-hand sides needs
    to reach relres 1e-10."""
    t_iter = t_cg / max(n_cg, 1)
    t_setup = t_call - t_cg
    return t_setup + t_iter * sum(iters), t_setup, t_iter


def cpu_baseline(shape, jacobi_iters, sample_iters):
    if _reference_package() is None:
        return {"value": None, "unit": "solves/s", "kind": "reference",
                "sample": "reference not installed in baseline/_ref"}
    iters, src = _reference_iterations(shape, jacobi_iters)
    if iters is None:
        if int(np.prod(shape)) > WHOLE_REFERENCE_NODES:
            return {"value": None, "unit": "solves/s", "kind": "reference",
                    "sample": f"not projected: {src}"}
        t_call, _, _ = reference_sample(shape, None)
        return {"value": NBOX / t_call, "unit": "solves/s", "cores": 1, "kind": "reference",
                "projected": False,
                "sample": (f"one whole reference extraction.capacitance_matrix (baseline/_ref, "
                           f"SciPy Jacobi-CG forced, relres 1e-10) of the {shape} workload: "
                           f"{t_call:.2f} s"),
                "seconds_per_extraction": t_call, "measured_call_seconds": t_call}
    t_call, t_cg, n_cg = reference_sample(shape, sample_iters)
    t_ext, t_setup, t_iter = _project(t_call, t_cg, n_cg, iters)
    return {"value": NBOX / t_ext, "unit": "solves/s", "cores": 1, "kind": "reference",
            "projected": True,
            "sample": (f"reference extraction.capacitance_matrix (baseline/_ref, SciPy "
                       f"Jacobi-CG forced) on the same {shape} workload, each RHS bounded to "
                       f"{n_cg // NBOX} CG iterations: call {t_call:.2f} s, set-up outside CG "
                       f"{t_setup:.2f} s, {t_iter*1e3:.1f} ms/iteration (SciPy's CSR SpMV "
                       f"is single-threaded); extraction = set-up + ms/iteration x "
                       f"iterations to 1e-10 of the 8 RHS ({src}: {iters})"),
            "seconds_per_extraction": t_ext, "measured_call_seconds": t_call}


def run_reference(args, rank, world):
    """The reference arm: the unmodified reference package (baseline/_ref)
    through its public API on this box's host cores, one bounded sample per
    step, projected to whole extractions.  Ranks other than 0 do nothing."""
    if rank != 0:
        return
    shape = tuple(int(v) for v in args.shape.split(","))
    if _reference_package() is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference package not installed in baseline/_ref"}),
              flush=True)
        return
    iters, src = _reference_iterations(shape)
    whole = iters is None and int(np.prod(shape)) <= WHOLE_REFERENCE_NODES
    if iters is None and not whole:
        print(json.dumps({"impl": "reference", "metric": "C solves/s @relres 1e-10",
                          "value": None, "unit": "solves/s",
                          "reason": f"not projected: {src}; measured whole only up to "
                                    f"{WHOLE_REFERENCE_NODES} nodes"}), flush=True)
        return
    sample = None if whole else max(2, args.cpu_sample_iters // 16)
    calls = []
    for s_ in range(args.warmup + args.steps):
        r = reference_sample(shape, sample)
        if s_ >= args.warmup:
            calls.append(r)
    t_call = statistics.median(c[0] for c in calls)
    t_cg = statistics.median(c[1] for c in calls)
    n_cg = calls[0][2]
    ncores = os.cpu_count() or 1
    if whole:
        t_ext, t_setup, t_iter = t_call, t_call - t_cg, 0.0
        sample_txt = (f"one whole reference extraction.capacitance_matrix from baseline/_ref "
                      f"(SciPy Jacobi-CG forced, relres 1e-10) per step: median {t_call:.2f} s; "
                      f"BLAS threads unrestricted on {ncores} cores, SpMV single-threaded")
    else:
        t_ext, t_setup, t_iter = _project(t_call, t_cg, n_cg, iters)
        sample_txt = (f"reference extraction.capacitance_matrix from baseline/_ref (SciPy "
                      f"Jacobi-CG forced), one call per step with each of the 8 RHS bounded to "
                      f"{n_cg // NBOX} CG iterations: median call {t_call:.2f} s (set-up outside "
                      f"CG {t_setup:.2f} s, {t_iter*1e3:.1f} ms/iteration); projected extraction "
                      f"= set-up + ms/iteration x iterations to 1e-10 of the 8 RHS ({src}: "
                      f"{iters}); BLAS threads unrestricted on {ncores} cores, SpMV "
                      f"single-threaded")
    value = NBOX / t_ext
    line = {
        "impl": "reference",
        "metric": "C solves/s @relres 1e-10",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_call * 1e3,
        "projected": not whole,
        "projected_ms_per_extraction": t_ext * 1e3,
        "measured": {"call_s": t_call, "setup_outside_cg_s": t_setup,
                     "ms_per_cg_iteration": t_iter * 1e3, "cg_iterations_per_call": n_cg},
        "extrapolated": (None if whole else
                         {"iterations_per_rhs": iters, "cg_s": t_iter * sum(iters)}),
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded layered dielectric + 8 conductor boxes)",
        "config": {"workload": f"layered_boxes {shape[0]}x{shape[1]}x{shape[2]} nodes, "
                               f"{NBOX} terminals, zlo grounded, seed=0",
                   "nodes": int(np.prod(shape)), "nrhs": NBOX, "tol": TOL,
                   "precision": "fp64", "preconditioner": "jacobi (SciPy CG)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": ncores,
                         "kind": "reference", "sample": sample_txt},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_unet_forward(args, dims=(64, 64, 32), batch=8):
    """U-Net forward timing (CUDA events) and its tensor-core FLOP rate."""
    import ctypes
    import torch
    from fieldspice_b200 import _lib as L
    from fieldspice_b200.learned import CIN, COUT, init_theta
    lib = L.lib()
    dev = torch.device("cuda", 0)
    N = int(np.prod(dims))
    th = torch.as_tensor(init_theta(0), device=dev)
    nb = ctypes.c_size_t()
    L.check("ws", lib.fs_unet_workspace_bytes(*dims, batch, 0, ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
    net = ctypes.c_void_p()
    L.check("create", lib.fs_unet_create(*dims, batch, 0, L.ptr(th), L.ptr(ws), nb.value,
                                         ctypes.byref(net), L.stream_ptr()))
    g = torch.Generator(device=dev).manual_seed(0)
    rhs = torch.randn((batch, N), device=dev, generator=g)
    em = torch.rand((batch, 3, N), device=dev, generator=g) * 0.16
    lab = (torch.rand((batch, N), device=dev, generator=g) < 0.05).to(torch.uint8)
    out = torch.empty((batch, N), device=dev)

    def fwd():
        L.check("fwd", lib.fs_unet_forward(net, L.ptr(rhs), 1, N, L.ptr(em), 3 * N, L.ptr(lab), N,
                                           L.ptr(out), 1, N, L.stream_ptr()))
    for _ in range(args.warmup):
        fwd()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fwd()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    flops = 0.0
    X, Y, Z = dims
    vox = []
    for l in range(4):
        vox.append(X * Y * Z * batch)
        X, Y, Z = (X + 1) // 2, (Y + 1) // 2, (Z + 1) // 2
    lev = (0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0)
    for l in range(14):
        flops += 2.0 * 27 * CIN[l] * COUT[l] * vox[lev[l]]
    lib.fs_unet_destroy(net)
    print(json.dumps({"unet_forward": True, "dims": dims, "batch": batch, "ms": ms,
                      "conv_tflop": flops / 1e12, "tflops": flops / (ms * 1e-3) / 1e12}),
          flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.unet_forward:
        run_unet_forward(args)
        return
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
