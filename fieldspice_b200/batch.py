"""Capacitance extraction of many independent geometries at once.

The reference extracts one geometry per ``capacitance_matrix`` call
(``fieldspice/extraction.py:41-56`` -> ``solvers/poisson.py:1100-1249``).
:func:`capacitance_matrices` takes a batch of uneven geometries, builds one
CG plan per geometry (all of its terminals as one block of right-hand sides)
and runs them together on a pool of CUDA streams with the library's
non-blocking solve (``fs_pcg_plan_solve_begin`` / ``fs_pcg_plan_solve_poll``):
largest geometry first, each plan's next graph chunk enqueued as soon as its
previous one has finished, and the host building the next plans while the GPU
solves the ones already built.  A geometry with more terminals than one block
of 32-byte nodes holds (8 FP32 / 4 FP64 RHS) solves its column blocks one
after another on its plan.  Charges are integrated per geometry in FP64
exactly as in a single extraction.

With a process group of several ranks (one per GPU), the geometries are
shared out by estimated cost (nodes x padded RHS, longest first onto the
least-loaded rank), every rank extracts its share, and one all-gather of the
small C matrices returns the whole batch, in input order, on every rank.
"""

from __future__ import annotations

import ctypes
import time
from typing import Any, Callable, Sequence

import numpy as np

from . import _lib as L
from .boundaries import dirichlet_nodes
from .device import (DeviceOperator, EliminatedSystem, block_rhs, h2d, pad_rhs,
                     rhs_blocks, upload_groups)
from .solvers.base import GPUConfig, SolverConfig, resolve_preconditioner
from .solvers.poisson import (capacitance_report, check_terminals, prepare_bc, raise_on_status,
                              shield_nodes, upload_cell_property)

__all__ = ["capacitance_matrices", "shard_by_cost", "problem_cost"]

#: CG vectors at or above this size (bytes) make a new plan time the stencil
#: kernels when it is created (the library's autotuner threshold).
TUNE_MIN_BYTES = 32 << 20


def problem_cost(problem, width: int = 8) -> float:
    """Work estimate of one extraction: nodes x the padded RHS widths of its
    column blocks."""
    grid, _, terms = problem[:3]
    blocks = rhs_blocks(len(terms), width)
    return float(np.prod(grid.shape_nodes)) * pad_rhs(len(blocks[0])) * len(blocks)


def shard_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of items to ``world`` ranks.

    Returns, per rank, the item indices it owns (ascending).  Ties go to the
    lower rank, so every rank computes the same assignment.
    """
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda w: (load[w], w))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(o) for o in out]


class _Extraction:
    """One geometry's extraction: the eliminated system (one plan, as wide
    as its largest column block), the charge groups of every terminal, and
    its terminals' unit excitations in column blocks solved one after
    another on that plan."""

    def __init__(self, grid, eps_cell, terminals, bc, cfg, gcfg, width):
        import torch
        self.grid = grid
        _, eps, eps_min, eps_max = upload_cell_property(eps_cell, grid, "eps_cell")
        if eps_min <= 0.0:
            raise ValueError("eps_cell must be strictly positive [F/m]")
        if eps_min >= 1e-6:
            raise ValueError("eps_cell looks like a RELATIVE permittivity; "
                             "pass the absolute value in F/m")
        self.terms = check_terminals(terminals, grid)
        nt = len(self.terms)
        if nt == 0:
            raise ValueError("capacitance extraction needs at least one terminal")
        self.blocks = rhs_blocks(nt, width)
        self.block = 0
        bc = prepare_bc(bc, grid)
        self.op = DeviceOperator(grid, eps, prop_range=(eps_min, eps_max))
        dev = self.op.dev
        wall_idx, _ = dirichlet_nodes(bc, grid, 0.0)
        term_nodes = [np.asarray(t.nodes, np.int64) for t in self.terms]
        self.term_dev = [h2d(n, torch.int64, dev) for n in term_nodes]
        wall_dev = h2d(wall_idx.astype(np.int64), torch.int64, dev)
        shield_dev = shield_nodes(wall_dev, self.term_dev, self.op.N)
        label = torch.zeros(self.op.N, dtype=torch.uint8, device=dev)
        if wall_idx.size:
            label[wall_dev] = L.LABEL_FIXED
        for n in self.term_dev:
            label[n] = L.LABEL_FIXED
        self.has_shield = shield_dev.numel() > 0
        groups = self.term_dev + ([shield_dev] if self.has_shield else [])
        self.groups = groups
        self.gdev = upload_groups(groups, dev)
        self.tol = float(cfg.tol)
        self.system = EliminatedSystem(
            self.op, label, len(self.blocks[0]), precision=gcfg.precision,
            preconditioner=resolve_preconditioner(cfg, gcfg), learned=gcfg.learned,
            coarsening=gcfg.coarsening, mg_params=gcfg.mg_params)
        # 0: the reference's cap max(500, 10 sqrt(n_free)), per plan on the device
        self.maxiter = 0 if gcfg.maxiter is None else int(gcfg.maxiter)
        self.group = torch.empty(self.op.N, dtype=torch.int16, device=dev)
        self.C = np.zeros((nt, nt))
        self.q_shield = np.zeros(nt)
        self.stats: list[dict] = []
        self.excite(0)

    def excite(self, b: int) -> None:
        """Unit excitations of column block b into the plan's phi (on the
        current stream)."""
        self.block = b
        self.system.nrhs = len(self.blocks[b])
        self.group.fill_(-1)
        for c, j in enumerate(self.blocks[b]):
            self.group[self.term_dev[j]] = c
        nx, ny, nz = self.op.shape
        L.check("fs_fill_unit_excitation", L.lib().fs_fill_unit_excitation(
            L.ptr(self.group), L.ptr(self.system.label_in), L.ptr(self.system.phi),
            nx, ny, nz, self.system.k, L.stream_ptr()))

    def collect(self, stats: list[dict]) -> bool:
        """The current block's columns of C and of the shield charge; True
        when every block is in."""
        nt = len(self.terms)
        cols = self.blocks[self.block]
        Q = self.op.group_sums(self.system.phi, self.groups, nrhs=self.system.k,
                               nodes_dev=self.gdev)
        self.C[:, cols] = np.asarray(Q[:nt, :len(cols)], dtype=float)
        if self.has_shield:
            self.q_shield[cols] = np.asarray(Q[nt, :len(cols)])
        self.stats.extend(stats)
        return self.block + 1 == len(self.blocks)

    def result(self) -> tuple[np.ndarray, dict]:
        info = {"method": f"gpu-cg-{self.system.preconditioner}-{self.system.mode}",
                "n": self.op.N, "iterations": [s["iterations"] for s in self.stats],
                "relres_fp64": [s["relres"] for s in self.stats],
                "residual": max(s["relres"] for s in self.stats),
                "fp64_fallback": bool(self.system.fell_back),
                "symmetric": True, "equilibrated": True, "blocks": len(self.blocks)}
        rep = capacitance_report(self.C, self.q_shield, info)
        rep["terminals"] = tuple(t.name for t in self.terms)
        return 0.5 * (self.C + self.C.T), rep

    def close(self):
        self.system.close()


def _stats_list(arr, n):
    return [{"iterations": s.iterations, "status": s.status, "relres": s.relres,
             "bnorm": s.bnorm, "reliable_updates": s.reliable_updates}
            for s in arr[:n]]


def extract_local(problems, cfg, gcfg, streams: int, reports: list | None):
    """Extract every problem on this GPU; returns the list of C matrices."""
    import torch
    out: list[Any] = [None] * len(problems)
    if not problems:
        return out
    lib = L.lib()
    tol = float(cfg.tol)
    # each geometry's terminals in column blocks of at most `width` (32-byte
    # nodes: the widest the fused multigrid passes serve), one plan per
    # geometry solving its blocks in turn
    width = block_rhs(gcfg.precision)
    # Largest first (longest-processing-time order).  Plans whose CG vectors
    # reach the stencil autotuner's 32 MB threshold (nodes x padded RHS x the
    # element size) time kernels when they are created, so they are all built
    # before any solve runs; after that each plan starts as soon as it is
    # built and the host builds the next while the GPU solves.
    order = sorted(range(len(problems)), key=lambda i: (-problem_cost(problems[i], width), i))
    es = 8 if gcfg.precision == "fp64" else 4

    def vector_bytes(i):
        p = problems[i]
        return float(np.prod(p[0].shape_nodes)) * pad_rhs(len(rhs_blocks(len(p[2]), width)[0])) * es
    tuned = [i for i in order if vector_bytes(i) >= TUNE_MIN_BYTES]
    rest = [i for i in order if vector_bytes(i) < TUNE_MIN_BYTES]
    pool = [torch.cuda.Stream() for _ in range(max(1, min(streams, len(problems))))]
    ex: dict[int, _Extraction] = {}
    running: dict[int, Any] = {}
    stream_of: dict[int, Any] = {}

    def build(i):
        p = problems[i]
        ex[i] = _Extraction(p[0], p[1], p[2], p[3] if len(p) > 3 else None, cfg, gcfg, width)
        stream_of[i] = pool[len(stream_of) % len(pool)]

    def start(i):
        s = stream_of[i]
        ready = torch.cuda.Event()
        ready.record(torch.cuda.current_stream())  # set-up and excitation kernels
        s.wait_event(ready)
        stats = (L.FsRhsStats * ex[i].system.k)()
        L.check("fs_pcg_plan_solve_begin", lib.fs_pcg_plan_solve_begin(
            ex[i].system.plan, 0, tol, ex[i].maxiter, s.cuda_stream))
        running[i] = stats

    def finish(i, st, stats_arr):
        e = ex[i]
        stats = _stats_list(stats_arr, e.system.nrhs)
        if st not in (L.FS_OK, L.FS_NOT_CONVERGED, L.FS_NAN, L.FS_STALLED):
            L.check("fs_pcg_plan_solve_poll", st)
        if e.system.preconditioner == "learned":
            st, stats = e.system.finish_learned(st, stats, tol, e.maxiter)
        _, stats = e.system.finish_auto(st, stats, tol, e.maxiter)
        raise_on_status(stats, tol, "gpu-cg")
        if e.collect(stats):
            out[i], rep = e.result()
            if reports is not None:
                reports[i] = rep
        else:  # the next column block on the same plan
            e.excite(e.block + 1)
            start(i)

    def poll() -> bool:
        progressed = False
        done = ctypes.c_int()
        for i in list(running):
            stats_arr = running[i]
            st = lib.fs_pcg_plan_solve_poll(ex[i].system.plan, stats_arr, ctypes.byref(done))
            if done.value:
                del running[i]
                finish(i, st, stats_arr)
                progressed = True
            elif st != L.FS_OK:
                del running[i]
                L.check("fs_pcg_plan_solve_poll", st)
        return progressed

    try:
        for i in tuned:
            build(i)
        for i in tuned:
            start(i)
        for i in rest:
            build(i)
            start(i)
            poll()
        while running:
            if not poll():
                time.sleep(5e-5)
    finally:
        # a failed batch may leave solves in flight: let them land before
        # the plans and their buffers go
        torch.cuda.synchronize()
        for e in ex.values():
            e.close()
    missing = [i for i, c in enumerate(out) if c is None]
    if missing:
        raise RuntimeError(f"batched extraction left geometries {missing} unsolved")
    return out


def capacitance_matrices(problems: Sequence, config: SolverConfig | None = None, *,
                         gpu: GPUConfig | None = None, streams: int = 16,
                         reports: list | None = None, group=None,
                         local: Callable | None = None) -> list[np.ndarray]:
    """Maxwell capacitance matrices of a batch of independent geometries.

    ``problems``: sequence of ``(grid, eps_cell, terminals)`` or
    ``(grid, eps_cell, terminals, bc)`` -- the arguments of
    ``extraction.capacitance_matrix`` per geometry.  Returns the symmetrised
    C matrices in input order.  ``reports``: optional list, filled with one
    report dict per geometry (the keys of a single extraction's report).

    ``group``: a ``torch.distributed`` process group (or ``None`` for the
    default group when one is initialised): geometries are sharded by cost
    over its ranks and the results all-gathered.  ``local``: the per-rank
    extraction, ``local(problems, config, gpu, streams, reports)``
    (defaults to the GPU one).
    """
    cfg = config or SolverConfig()
    gcfg = gpu or GPUConfig()
    problems = list(problems)
    run = local or extract_local
    t0 = time.perf_counter()
    import torch.distributed as dist
    world, rank = 1, 0
    if dist.is_available() and dist.is_initialized():
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
    if world == 1:
        return run(problems, cfg, gcfg, streams, reports)
    shards = shard_by_cost([problem_cost(p, block_rhs(gcfg.precision)) for p in problems],
                           world)
    mine = shards[rank]
    my_reports = [None] * len(mine) if reports is not None else None
    res = run([problems[i] for i in mine], cfg, gcfg, streams, my_reports)
    gathered: list[Any] = [None] * world
    payload = (mine, [np.asarray(c) for c in res], my_reports)
    dist.all_gather_object(gathered, payload, group=group)
    out: list[Any] = [None] * len(problems)
    for idx, mats, reps in gathered:
        for j, i in enumerate(idx):
            out[i] = mats[j]
            if reports is not None and reps is not None:
                reports[i] = reps[j]
    if reports is not None:
        for r in reports:
            if isinstance(r, dict):
                r.setdefault("batch_time", time.perf_counter() - t0)
    return out
