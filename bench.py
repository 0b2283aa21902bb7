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
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
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
    return ap.parse_args()


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """Per-node DRAM bytes of the CG kernels from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
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
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def kernel_bytes(N: int, k: int, s: int) -> dict:
    """Algorithmic bytes per launch of the CG kernels (each array once)."""
    return {"pupdate": 3 * N * k * s,                 # read r|z, p_old; write p
            "stencil": N * (2 * k * s + 3 * s),       # read p, 3 masses; write q
            "update": 6 * N * k * s,                  # read p, q, x, r; write x, r
            # fine-level post-smoothing, one fused pass (k_mg_post_fused):
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

    def step_e2e(precision):
        rep = {}
        C = EX.capacitance_matrix(grid, eps_pinned, terms, bc, SolverConfig(tol=TOL),
                                  report=rep, gpu=GPUConfig(precision=precision,
                                                            preconditioner=args.preconditioner))
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

    sampler = ClockSampler(local_rank)
    sampler.start()
    ms_dev, outs = timed(lambda: step_device(args.precision), args.steps, args.warmup)
    clocks = sampler.stop()
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
    kb = kernel_bytes(N, 8, s)
    km = info["kernel_ms"]
    times = {"pupdate": km["pupdate_ms"], "stencil": km["stencil_ms"],
             "update": km["update_ms"]}
    if args.preconditioner == "mg":
        times["smoother"] = km["smoother_ms"]
    dom = max(times, key=times.get)
    peak, peak_kind = measured_peaks()
    gbs = {k: kb[k] / (times[k] * 1e-3) / 1e9 for k in times if times[k] > 0}
    traffic = committed_traffic().get(f"{dom}_{args.precision}_bytes_per_node")
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
                "step_ms_max": e2e_steps[-1] if e2e_steps else None},
        "roofline": {
            "bound": "hbm", "kernel": dom, "achieved": gbs.get(dom), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s",
            "frac": (gbs.get(dom) or 0.0) / peak,
            "traffic": (traffic * N if traffic else None),
            "algorithmic_bytes_per_launch": kb[dom],
            "ms_per_launch": times[dom], "samples": km["samples"],
            "all_kernels_gbs": gbs, "all_kernels_ms": times,
            "precond_ms_per_iteration": km.get("precond_ms"),
        },
        "stencil_gbs": gbs.get("stencil"),
        "learned_vs_plain_pcg": (variants["learned_fcg"]["value"] / variants["plain_pcg_jacobi"]["value"]
                                 if "learned_fcg" in variants and "plain_pcg_jacobi" in variants
                                 else None),
        "gpu_launches": int(launches),
        "clocks": clocks,
        "iterations": info["iterations"],
        "reliable_updates": info.get("reliable_updates"),
        "plan_setup_ms": 1e3 * info.get("setup_time", 0.0),
        "relres_fp64_max": info["residual"],
        "asymmetry_rel": rep["asymmetry_rel"],
        "C_err_vs_fp64_oracle": err_vs_oracle,
        "variants": variants,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(shape, info["iterations"], args.cpu_sample_iters)
    print(json.dumps(line), flush=True)


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
    return {"metric": "EQS steps/s (192x192x96, 200 steps, dt 1 ps)",
            "value": steps / t, "seconds": t, "fp64_seconds": tf,
            "nodes": int(np.prod(shape)),
            "current_err_vs_fp64_max": float(err.max()),
            "current_err_vs_fp64_final": float(err[-1]),
            "per_step_err_quantiles": [float(np.quantile(err, q)) for q in (0.5, 0.9, 1.0)],
            "precision": "auto (mixed, FP64 continuation on stall)", "tol": TOL}


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
    ref = capacitance_matrices(probs, SolverConfig(tol=1e-12),
                               gpu=GPUConfig(precision="fp64", preconditioner="mg"))
    errs = [float(np.abs(a - b).max() / np.abs(np.diag(b)).max()) for a, b in zip(Cs, ref)]
    nodes = [int(np.prod(p[0].shape_nodes)) for p in probs]
    return {"metric": "C-matrices/s (64 uneven geometries)",
            "value": len(probs) / (ms_b / 1000.0), "ms_per_batch": ms_b,
            "one_at_a_time_value": len(probs) / (ms_s / 1000.0),
            "solves_per_batch": int(sum(len(p[2]) for p in probs)),
            "nodes_total": int(sum(nodes)), "nodes_min": min(nodes), "nodes_max": max(nodes),
            "max_iterations": max(max(r["linear"]["iterations"]) for r in reps),
            "C_err_vs_fp64_max": max(errs), "C_err_vs_fp64_per_geometry": errs}


# ---------------------------------------------------------------------------
# CPU oracle timing (cpu_baseline and the reference arm)
# ---------------------------------------------------------------------------
_CPU = {}


def _cpu_setup(shape, seed=0):
    from oracle import fs_oracle as O
    from fieldspice_b200 import workloads as W
    import scipy.sparse as sp
    w = W.layered_boxes(shape, nbox=NBOX, seed=seed)
    g = O.Grid(w.x, w.y, w.z)
    t0 = time.perf_counter()
    m = O.edge_mass_vector(g, O.cell_to_edge(g, w.eps_cell))
    Lm = O.nodal_laplacian(g, m)
    wall = O.wall_nodes(g, "zlo")
    terms = [np.asarray(t, np.intp) for t in w.terminals]
    fixed = np.unique(np.concatenate([wall] + terms))
    A, _ = O.apply_dirichlet(Lm, np.zeros(g.n_nodes), fixed, 0.0)
    ls = O.LinearSystemCPU(A, method="cg", tol=TOL)
    t_setup = time.perf_counter() - t0
    _CPU.update(Lm=Lm, ls=ls, terms=terms, fixed=fixed, n=g.n_nodes, t_setup=t_setup)
    return t_setup


def _cpu_iterate(j, iters):
    """Run `iters` iterations of the reference's Jacobi CG on RHS j."""
    import scipy.sparse.linalg as spla
    Lm, ls, terms, fixed, n = (_CPU[k] for k in ("Lm", "ls", "terms", "fixed", "n"))
    x0 = np.zeros(n)
    x0[terms[j]] = 1.0
    b = -(Lm @ x0)
    b[fixed] = x0[fixed]
    bs = (b[ls.free] if ls.split else b) * ls.dinv
    t0 = time.perf_counter()
    spla.cg(ls.A, bs, rtol=1e-30, atol=0.0, maxiter=iters, M=ls.M)
    return (time.perf_counter() - t0) / iters


def _reference_iterations(gpu_iters=None):
    if FULLSIZE_JSON.exists():
        d = json.loads(FULLSIZE_JSON.read_text())
        return [int(v) for v in d["iterations_1e-10"]], "oracle full-size run (tests/golden)"
    if gpu_iters:
        return [int(v) for v in gpu_iters], "GPU solve of the same system"
    return [1765] * NBOX, "survey measurement"


def cpu_baseline(shape, gpu_iters, sample_iters):
    from threadpoolctl import threadpool_limits
    with threadpool_limits(limits=1):
        t_setup = _cpu_setup(shape)
        t_iter = _cpu_iterate(0, sample_iters)
    iters, src = _reference_iterations(gpu_iters)
    t_ext = t_setup + sum(t_iter * it for it in iters)
    return {"value": NBOX / t_ext, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": (f"CPU oracle (SciPy Jacobi-CG on the equilibrated system): "
                       f"assembly ({t_setup:.2f} s) + {sample_iters} CG iterations on "
                       f"RHS 0 of the same {shape} workload ({t_iter*1e3:.1f} ms/iter); "
                       f"extraction time = assembly + sum over 8 RHS of ms/iter x "
                       f"iterations to 1e-10 ({src}: {iters})"),
            "seconds_per_extraction": t_ext}


def run_reference(args, rank, world):
    if rank != 0:
        return
    import multiprocessing as mp
    shape = tuple(int(v) for v in args.shape.split(","))
    ncores = os.cpu_count() or 1
    nproc = max(1, min(NBOX, ncores))
    sample = max(5, args.cpu_sample_iters // 2)
    from threadpoolctl import threadpool_limits
    with threadpool_limits(limits=1):
        t_setup = _cpu_setup(shape)
    iters, src = _reference_iterations()
    ctx = mp.get_context("fork")  # no CUDA in this process
    step_times = []
    with threadpool_limits(limits=1), ctx.Pool(nproc) as pool:
        for s in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            per = pool.starmap(_cpu_iterate, [(j, sample) for j in range(NBOX)])
            wall = time.perf_counter() - t0
            if s >= args.warmup:
                # RHS run concurrently on nproc cores: the extraction takes the
                # assembly plus the longest per-process chain of solves.
                chains = [0.0] * nproc
                for j in range(NBOX):
                    chains[j % nproc] += per[j] * iters[j]
                step_times.append(t_setup + max(chains))
    t_ext = statistics.median(step_times)
    value = NBOX / t_ext
    line = {
        "impl": "reference",
        "metric": "C solves/s @relres 1e-10",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ext * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded layered dielectric + 8 conductor boxes)",
        "config": {"workload": f"layered_boxes {shape[0]}x{shape[1]}x{shape[2]} nodes, "
                               f"{NBOX} terminals, zlo grounded, seed=0",
                   "nodes": int(np.prod(shape)), "nrhs": NBOX, "tol": TOL,
                   "precision": "fp64", "preconditioner": "jacobi (SciPy CG)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nproc, "kind": "port",
                         "sample": (f"CPU oracle (the reference's SciPy Jacobi-CG, restated): "
                                    f"assembly ({t_setup:.2f} s) once, then per step {sample} "
                                    f"CG iterations on each of the 8 RHS in {nproc} "
                                    f"processes; extraction time = assembly + longest chain "
                                    f"of (s/iter x iterations to 1e-10 [{src}: {iters}])")},
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
