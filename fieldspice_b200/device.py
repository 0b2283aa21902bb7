"""Device-resident operators and the eliminated CG system.

:class:`DeviceOperator` holds the edge masses of one ``G^T diag(m) G`` in HBM
(FP64, node-padded, see ``include/fieldspice_b200.h``) and offers the FP64
applies, charge sums and energies.  :class:`EliminatedSystem` binds one
operator, one Dirichlet label array and one potential buffer to a CG plan of
the C library and solves in place.
"""

from __future__ import annotations

import ctypes
import math
import time
import weakref

import numpy as np

from . import _lib as L
from .grid import grid_metric

__all__ = ["DeviceOperator", "EliminatedSystem", "pad_rhs", "MAX_RHS", "block_rhs", "rhs_blocks",
           "device", "h2d", "d2h", "TRANSFERS", "PHASES", "mark", "upload_groups"]

#: Bytes moved between host and device by the product path (host arrays
#: uploaded, results read back); the benchmark reads it per step.
TRANSFERS = {"h2d": 0, "d2h": 0}

#: Host-side phase log of the public calls: ``None`` (off), or a list that
#: receives ``(phase, wall seconds, process CPU seconds)`` at each phase end.
PHASES: list | None = None


def mark(phase: str) -> None:
    """Record the end of ``phase`` in :data:`PHASES` when logging is on."""
    if PHASES is not None:
        PHASES.append((phase, time.perf_counter(), time.process_time()))


#: Host arrays up to this size go through a page-locked staging copy.
STAGED_H2D_BYTES = 4 << 20


def h2d(a, dtype, dev):
    """Upload a host array (counted in ``TRANSFERS``).

    Small arrays are copied into page-locked staging memory and uploaded
    asynchronously on the current stream, so the host does not wait for the
    device work queued before (a copy from pageable memory would); the
    staging block is reused only after the copy has run.  Larger arrays are
    uploaded synchronously."""
    import torch
    arr = np.ascontiguousarray(a)
    TRANSFERS["h2d"] += arr.nbytes
    src = torch.as_tensor(arr)
    if src.dtype != dtype:
        src = src.to(dtype)
    if src.numel() * src.element_size() > STAGED_H2D_BYTES:
        return src.to(device=dev)
    staged = torch.empty(src.shape, dtype=dtype, pin_memory=True)
    staged.copy_(src)
    out = torch.empty(src.shape, dtype=dtype, device=dev)
    out.copy_(staged, non_blocking=True)
    return out


def d2h(t) -> np.ndarray:
    """Read a device tensor back to a NumPy array (counted)."""
    out = t.detach().cpu().numpy()
    TRANSFERS["d2h"] += out.nbytes
    return out

MAX_RHS = 16
_SUPPORTED_K = (1, 2, 4, 8, 16)


def block_rhs(precision: str) -> int:
    """RHS block width of a multi-terminal solve: 32-byte nodes (8 FP32 or 4
    FP64 values), the widest the fused multigrid passes and the TMA
    restriction serve.  Measured with 16 terminals: two 8-RHS blocks 48.3 ms
    against 79.3 ms for one 16-RHS block at 160x160x96 (15.5 against 19.5 ms
    at 96x96x64)."""
    return 4 if precision == "fp64" else 8


def rhs_blocks(n: int, width: int) -> list[list[int]]:
    """Columns 0..n-1 in ceil(n / width) blocks of near-equal size (one
    padded RHS width serves them all, so one plan solves every block)."""
    if n <= 0:
        return []
    nb = -(-n // width)
    size = -(-n // nb)
    return [list(range(b, min(n, b + size))) for b in range(0, n, size)]


def pad_rhs(k: int) -> int:
    """Smallest supported RHS width (1, 2, 4, 8, 16) holding ``k`` columns."""
    for s in _SUPPORTED_K:
        if k <= s:
            return s
    raise ValueError(f"at most {MAX_RHS} right-hand sides per solve, got {k}")


def device():
    import torch
    L.lib()  # raises without a GPU or without the library
    return torch.device("cuda", torch.cuda.current_device())


# Device copies of each grid's metric arrays (cell widths and dual widths),
# reused while the grid's host values are unchanged.
_METRIC_CACHE: "weakref.WeakKeyDictionary" = weakref.WeakKeyDictionary()


def metric_dev(grid, dev):
    """The six FP64 metric arrays of ``grid_metric(grid)`` on ``dev``.

    Kept per grid object and reused as long as the grid's current metric
    equals the cached host copy (so a grid changed in place is uploaded
    again); grids that cannot be weakly referenced are uploaded each call."""
    import torch
    (hx, hy, hz), (hxd, hyd, hzd) = grid_metric(grid)
    host = [np.asarray(a, dtype=np.float64) for a in (hx, hy, hz, hxd, hyd, hzd)]
    try:
        hit = _METRIC_CACHE.get(grid)
    except TypeError:
        hit = None
    if hit is not None and hit[0] == dev and all(
            a.shape == b.shape and np.array_equal(a, b) for a, b in zip(hit[1], host)):
        return hit[2]
    tensors = [h2d(a, torch.float64, dev) for a in host]
    try:
        _METRIC_CACHE[grid] = (dev, [a.copy() for a in host], tensors)
    except TypeError:
        pass
    return tensors


def _as_dev(a, dtype, dev):
    import torch
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype).contiguous()
    return h2d(a, dtype, dev)


class DeviceOperator:
    """``G^T diag(m) G`` on one grid, masses resident on the GPU.

    Build from a per-cell property with the reference's averaging
    (``fieldspice/operators.py:144-237`` then ``:302-315``), or wrap masses
    that already live on the device.
    """

    def __init__(self, grid, prop_cell=None, *, mode: str = "parallel",
                 masses=None, shape=None, periodic: int = 0, prop_range=None):
        import torch
        self.grid = grid
        self.shape = (tuple(int(s) for s in grid.shape_nodes) if shape is None
                      else tuple(int(s) for s in shape))
        self.N = int(np.prod(self.shape))
        self.dev = device()
        self.periodic = int(periodic)   # wrap-around axes (bit 0 x, 1 y, 2 z)
        self.material_contrast = None   # cell-property max/min, when known
        lib = L.lib()
        if masses is not None:
            self.m = masses
            return
        if mode not in ("parallel", "arithmetic", "harmonic", "series"):
            raise ValueError(f"unknown averaging mode {mode!r}")
        avg = L.AVERAGE_HARMONIC if mode in ("harmonic", "series") else L.AVERAGE_PARALLEL
        hs = metric_dev(grid, self.dev)
        prop = _as_dev(prop_cell, torch.float64, self.dev)
        if prop.numel() != int(np.prod(grid.shape_cells)):
            raise ValueError("prop_cell does not match the grid's cell shape")
        self.m = torch.empty((3, self.N), dtype=torch.float64, device=self.dev)
        nx, ny, nz = self.shape
        st = lib.fs_build_masses(L.ptr(prop), *(L.ptr(h) for h in hs), nx, ny, nz,
                                 avg, L.ptr(self.m[0]), L.ptr(self.m[1]),
                                 L.ptr(self.m[2]), L.stream_ptr())
        L.check("fs_build_masses", st)
        # the material contrast (largest over smallest positive cell value),
        # which decides the multigrid hierarchy; geometry (grading, a
        # collapsed axis) is handled by the rediscretised levels either way,
        # and a zero-conductivity region is decoupled, not a contrast
        if prop_range is None and isinstance(prop_cell, np.ndarray):
            pos = prop_cell[prop_cell > 0]
            if pos.size:
                prop_range = (float(pos.min()), float(pos.max()))
        if prop_range is not None:
            lo, hi = (float(v) for v in prop_range)
            self.material_contrast = hi / lo if lo > 0.0 else None

    # -- mass arrays ---------------------------------------------------------
    @property
    def mx(self):
        return self.m[0]

    @property
    def my(self):
        return self.m[1]

    @property
    def mz(self):
        return self.m[2]

    def reduced(self, periodic: int) -> "DeviceOperator":
        """The operator of the wrap-around grid of periodic axes ``periodic``
        (the last node plane of each merged into the first, as the reference's
        node-merging reduction, ``poisson.py:665-719``); FP64 masses built on
        the device (``fs_periodic_masses``)."""
        import torch
        nx, ny, nz = self.shape
        shape = (nx - (periodic & 1), ny - ((periodic >> 1) & 1), nz - ((periodic >> 2) & 1))
        if min(shape) < 2:
            raise ValueError("a periodic axis needs at least 3 node planes")
        m = torch.empty((3, int(np.prod(shape))), dtype=torch.float64, device=self.dev)
        L.check("fs_periodic_masses", L.lib().fs_periodic_masses(
            L.ptr(self.m), nx, ny, nz, int(periodic), L.ptr(m), L.stream_ptr()))
        return DeviceOperator(self.grid, masses=m, shape=shape, periodic=periodic)

    def combine(self, a: float, other: "DeviceOperator", b: float) -> "DeviceOperator":
        """``a*self + b*other`` edge by edge (eqs.py:279-280)."""
        import torch
        out = torch.empty_like(self.m)
        st = L.lib().fs_combine_masses(L.ptr(self.m), L.ptr(other.m), float(a),
                                       float(b), L.ptr(out), self.m.numel(),
                                       L.stream_ptr())
        L.check("fs_combine_masses", st)
        return DeviceOperator(self.grid, masses=out, shape=self.shape, periodic=self.periodic)

    def mass_contrast(self) -> float:
        """max / min over the nonzero edge masses (1 when there are none),
        computed on the device once and kept."""
        import torch
        c = getattr(self, "_contrast", None)
        if c is None:
            hi = self.m.max()
            lo = torch.where(self.m > 0, self.m, torch.full_like(self.m[:1, :1], np.inf)).min()
            hi, lo = (float(v) for v in torch.stack([hi, lo]).cpu())
            c = hi / lo if (hi > 0 and np.isfinite(lo)) else 1.0
            self._contrast = c
        return c

    def edge_vector(self) -> np.ndarray:
        """Masses in the reference's concatenated [x|y|z] edge order (host)."""
        nx, ny, nz = self.shape
        m = self.m.cpu().numpy().reshape(3, nx, ny, nz)
        return np.concatenate([m[0, :-1].ravel(), m[1, :, :-1].ravel(),
                               m[2, :, :, :-1].ravel()])

    # -- FP64 applies ----------------------------------------------------------
    def apply(self, u, nrhs: int = 1, add=None):
        """``L u (+ add)`` in FP64 on the device (u: N*nrhs, RHS-interleaved)."""
        import torch
        out = torch.empty_like(u)
        nx, ny, nz = self.shape
        st = L.lib().fs_apply_laplacian(L.ptr(self.mx), L.ptr(self.my),
                                        L.ptr(self.mz), L.ptr(u), L.ptr(add),
                                        L.ptr(out), nx, ny, nz, nrhs,
                                        L.stream_ptr())
        L.check("fs_apply_laplacian", st)
        return out

    def quadform(self, u, nrhs: int = 1, out=None):
        """``u^T L u`` per RHS (FP64): a host array, or written into the
        device tensor ``out`` (nrhs FP64 values) without a host copy."""
        import torch
        lib = L.lib()
        nb = ctypes.c_size_t()
        L.check("fs_quadform_workspace_bytes",
                lib.fs_quadform_workspace_bytes(nrhs, ctypes.byref(nb)))
        ws = torch.empty(nb.value, dtype=torch.uint8, device=self.dev)
        dst = torch.empty(nrhs, dtype=torch.float64, device=self.dev) if out is None else out
        nx, ny, nz = self.shape
        st = lib.fs_quadform(L.ptr(self.mx), L.ptr(self.my), L.ptr(self.mz),
                             L.ptr(u), nx, ny, nz, nrhs, L.ptr(dst), L.ptr(ws),
                             nb.value, L.stream_ptr())
        L.check("fs_quadform", st)
        return d2h(dst) if out is None else out

    def group_sums(self, u, groups, nrhs: int = 1, minus=None, w=None,
                   nodes_dev=None, out=None):
        """``sum_{n in group} (L u - L_minus w)_n`` per group and RHS (FP64).

        ``groups`` is a list of node-index arrays; ``nodes_dev`` may carry the
        already-uploaded ``(nodes, offsets)`` pair to skip the copy.  Returns
        a host ``(ngroups, nrhs)`` array, or writes the device tensor ``out``
        (ngroups * nrhs FP64 values) without a host copy.
        """
        import torch
        lib = L.lib()
        if nodes_dev is None:
            nodes_dev = upload_groups(groups, self.dev)
        nodes, offsets, ng = nodes_dev
        nb = ctypes.c_size_t()
        L.check("fs_group_apply_workspace_bytes",
                lib.fs_group_apply_workspace_bytes(ng, nrhs, ctypes.byref(nb)))
        ws = torch.empty(nb.value, dtype=torch.uint8, device=self.dev)
        dst = (torch.empty(ng * nrhs, dtype=torch.float64, device=self.dev)
               if out is None else out)
        nx, ny, nz = self.shape
        mb = (None, None, None) if minus is None else (minus.mx, minus.my, minus.mz)
        st = lib.fs_group_apply(L.ptr(self.mx), L.ptr(self.my), L.ptr(self.mz),
                                L.ptr(u), *(L.ptr(t) for t in mb), L.ptr(w),
                                L.ptr(nodes), L.ptr(offsets), ng, nx, ny, nz,
                                nrhs, L.ptr(dst), L.ptr(ws), nb.value,
                                L.stream_ptr())
        L.check("fs_group_apply", st)
        return d2h(dst).reshape(ng, nrhs) if out is None else out


def upload_groups(groups, dev):
    """Concatenate node lists into (nodes, offsets, ngroups) device arrays.

    ``groups`` may hold host arrays or int64 device tensors."""
    import torch
    if groups and all(isinstance(g, torch.Tensor) for g in groups):
        sizes = [int(g.numel()) for g in groups]
        flat = torch.cat([g.reshape(-1).to(torch.int64) for g in groups])
        offsets = np.zeros(len(groups) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum(sizes)
        if flat.numel() == 0:
            flat = torch.zeros(1, dtype=torch.int64, device=dev)
        return flat, h2d(offsets, torch.int64, dev), len(groups)
    groups = [np.asarray(g, dtype=np.int64).ravel() for g in groups]
    offsets = np.zeros(len(groups) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([g.size for g in groups])
    flat = np.concatenate(groups) if groups else np.zeros(0, np.int64)
    if flat.size == 0:
        flat = np.zeros(1, np.int64)
    return h2d(flat, torch.int64, dev), h2d(offsets, torch.int64, dev), len(groups)


class EliminatedSystem:
    """One Dirichlet-eliminated system and its CG plan.

    ``label``: uint8 device array (``FS_LABEL_FREE``/``FS_LABEL_FIXED`` per
    node).  ``phi`` (N*k FP64) holds the Dirichlet values on fixed nodes and
    receives the solution; ``f`` (optional, N*k) is the source term.

    ``precision``: ``"mixed"`` (FP32 inner CG, FP64 reliable updates),
    ``"fp64"``, or ``"auto"``: mixed, and if a right-hand side stalls (a mode
    below FP32 resolution, e.g. a floating copper island in oxide) the same
    solve continues in FP64 from the mixed iterate; later solves of this
    system then stay in FP64.
    """

    #: Material contrast (the operator's cell property, max over min; the
    #: edge-mass contrast when the property is not known) above which
    #: ``coarsening="auto"`` builds the multigrid levels by aggregation with
    #: Galerkin coarse operators (copper/oxide in an EQS step is ~1e6).
    GALERKIN_CONTRAST = 1e3

    def __init__(self, op: DeviceOperator, label, nrhs: int, *,
                 precision: str = "auto", with_source: bool = False,
                 preconditioner: str = "jacobi", learned=None, diag=None,
                 coarsening: str = "auto", mg_params: dict | None = None):
        import torch
        self.mg_params = L.mg_params(mg_params)  # validated names; None = defaults
        if coarsening not in ("auto", "geometric", "galerkin"):
            raise ValueError(f"coarsening must be 'auto', 'geometric' or 'galerkin', "
                             f"got {coarsening!r}")
        if precision not in ("auto", "mixed", "fp64"):
            raise ValueError(f"precision must be 'auto', 'mixed' or 'fp64', got {precision!r}")
        if preconditioner not in ("jacobi", "mg", "learned"):
            raise ValueError(f"preconditioner must be 'jacobi', 'mg' or 'learned', "
                             f"got {preconditioner!r}")
        if preconditioner == "learned":
            if learned is None:
                raise ValueError("preconditioner='learned' needs a trained network")
            if precision == "fp64":
                raise ValueError("the learned preconditioner runs in mixed precision")
        if op.periodic and preconditioner != "jacobi":
            # of the multigrid hierarchies only the aggregation one wraps
            if preconditioner == "learned":
                raise ValueError("the learned preconditioner does not support periodic axes")
            coarsening = "galerkin"
        self.preconditioner = preconditioner
        self.learned = learned
        # optional FP64 node-diagonal term of the operator (kept alive here)
        self.diag = (None if diag is None else
                     torch.as_tensor(diag, dtype=torch.float64, device=op.dev).contiguous())
        if preconditioner == "mg" and coarsening == "auto":
            contrast = (op.material_contrast if op.material_contrast is not None
                        else op.mass_contrast())
            coarsening = "galerkin" if contrast > self.GALERKIN_CONTRAST else "geometric"
        # the learned level is trained on the geometric hierarchy
        self.coarsening = ("geometric" if preconditioner == "learned" else coarsening) \
            if preconditioner != "jacobi" else None
        self._pc = (L.PRECOND_JACOBI if preconditioner == "jacobi" else
                    L.PRECOND_MG_AGG if self.coarsening == "galerkin" else L.PRECOND_MG)
        self.op = op
        self.k = pad_rhs(nrhs)
        self.nrhs = nrhs
        self.mode = precision
        self.precision = "fp64" if precision == "fp64" else "mixed"
        dev = op.dev
        N = op.N
        self.label_in = label
        self.phi = torch.zeros(N * self.k, dtype=torch.float64, device=dev)
        self.f = (torch.zeros(N * self.k, dtype=torch.float64, device=dev)
                  if with_source else None)
        t0 = time.perf_counter()
        self._plan, self.workspace = self._make_plan(self.precision)
        self._fp64 = None
        self.fell_back = False
        # The classified labels are the first N bytes of the workspace.
        lib = L.lib()
        lab_ptr = lib.fs_pcg_plan_labels(self._plan)
        off = lab_ptr - self.workspace.data_ptr()
        self.labels = self.workspace[off:off + N]
        self._counts = None      # free / fixed / solo / pinned, read when first asked
        self._net_ws = None
        self.learned_level = None
        self.learned_fallback = False
        if preconditioner == "learned":
            self.learned_level = learned.attach(self._plan, self)
        self.setup_time = time.perf_counter() - t0
        self.launches = 0
        self._last_plan = self._plan

    def _make_plan(self, precision: str):
        import torch
        lib = L.lib()
        op = self.op
        prec = L.PRECISION_MIXED if precision == "mixed" else L.PRECISION_FP64
        nb = ctypes.c_size_t()
        nx, ny, nz = op.shape
        opt = None if self.mg_params is None else ctypes.byref(self.mg_params)
        L.check("fs_pcg_workspace_bytes",
                lib.fs_pcg_workspace_bytes_opt(nx, ny, nz, self.k, prec, self._pc, opt,
                                               ctypes.byref(nb)))
        ws = torch.empty(nb.value, dtype=torch.uint8, device=op.dev)
        if ws.data_ptr() % 256:
            raise RuntimeError("device allocation is not 256-byte aligned")
        plan = ctypes.c_void_p()
        st = lib.fs_pcg_plan_create_opt(nx, ny, nz, self.k, prec, self._pc, L.ptr(op.mx),
                                        L.ptr(op.my), L.ptr(op.mz), L.ptr(self.diag),
                                        int(op.periodic), opt, L.ptr(self.label_in),
                                        L.ptr(self.phi), L.ptr(self.f), L.ptr(ws), nb.value,
                                        ctypes.byref(plan), L.stream_ptr())
        L.check("fs_pcg_plan_create", st)
        return plan, ws

    def _label_counts(self):
        if self._counts is None:
            counts = (ctypes.c_longlong * 4)()
            L.check("fs_pcg_plan_label_counts",
                    L.lib().fs_pcg_plan_label_counts(self._plan, counts, L.stream_ptr()))
            self._counts = tuple(int(c) for c in counts)
        return self._counts

    @property
    def n_free(self) -> int:
        return self._label_counts()[0]

    @property
    def n_fixed(self) -> int:
        return self._label_counts()[1]

    @property
    def n_solo(self) -> int:
        return self._label_counts()[2]

    @property
    def n_pinned(self) -> int:
        return self._label_counts()[3]

    def default_maxiter(self) -> int:
        """The reference's cap ``max(500, 10*sqrt(n))`` (poisson.py:535-536)."""
        return max(500, int(10 * math.sqrt(max(self.n_free, 1))))

    def _run(self, plan, tol, maxiter, warm):
        lib = L.lib()
        stats = (L.FsRhsStats * self.k)()
        st = lib.fs_pcg_plan_solve(plan, 1 if warm else 0, float(tol), maxiter,
                                   stats, L.stream_ptr())
        self.launches += int(lib.fs_pcg_plan_launches(plan))
        if st not in (L.FS_OK, L.FS_NOT_CONVERGED, L.FS_NAN, L.FS_STALLED):
            L.check("fs_pcg_plan_solve", st)
        self._last_plan = plan
        return st, [{"iterations": s.iterations, "status": s.status,
                     "relres": s.relres, "bnorm": s.bnorm,
                     "reliable_updates": s.reliable_updates}
                    for s in stats[:self.nrhs]]

    def solve(self, tol: float, maxiter: int | None = None, *, warm: bool = False):
        """Solve in place into ``phi``; returns (status, per-RHS stats dicts).
        ``maxiter=None``: the reference's cap, evaluated on the device."""
        mi = 0 if maxiter is None else int(maxiter)
        self.launches = 0
        if self.fell_back:
            return self._run(self._fp64[0], tol, mi, warm)
        st, stats = self._run(self._plan, tol, mi, warm)
        if self.preconditioner == "learned":
            st, stats = self.finish_learned(st, stats, tol, mi)
        return self.finish_auto(st, stats, tol, mi)

    def finish_learned(self, st: int, stats: list, tol: float, maxiter: int):
        """If flexible CG with the network stalled or hit ``maxiter``, detach
        the network (plain multigrid PCG) and continue from the iterate."""
        bad = any(s["status"] in (L.FS_NOT_CONVERGED, L.FS_STALLED, L.FS_NAN) for s in stats)
        if not bad:
            return st, stats
        L.check("fs_pcg_plan_set_unet", L.lib().fs_pcg_plan_set_unet(
            self._plan, -1, 0, None, None, 0, L.stream_ptr()))
        self.learned_fallback = True
        st, stats2 = self._run(self._plan, tol, maxiter, True)
        for a, b in zip(stats, stats2):
            b["iterations"] += a["iterations"]
            b["reliable_updates"] += a["reliable_updates"]
            b["learned_fallback"] = True
        return st, stats2

    def finish_auto(self, st: int, stats: list, tol: float, maxiter: int):
        """In ``"auto"`` mode, continue a mixed solve whose RHS stalled or hit
        ``maxiter`` in FP64 from its iterate (this system then stays FP64)."""
        bad = any(s["status"] in (L.FS_NOT_CONVERGED, L.FS_STALLED) for s in stats)
        if self.mode == "auto" and bad and not self.fell_back:
            if self._fp64 is None:
                self._fp64 = self._make_plan("fp64")
            self.fell_back = True
            st, stats2 = self._run(self._fp64[0], tol, maxiter, True)
            for a, b in zip(stats, stats2):
                b["iterations"] += a["iterations"]
                b["reliable_updates"] += a["reliable_updates"]
                b["fp64_fallback"] = True
            stats = stats2
        return st, stats

    @property
    def plan(self):
        """The CG plan the next solve runs (the FP64 one after a fallback)."""
        return self._fp64[0] if self.fell_back else self._plan

    def kernel_times(self) -> dict:
        """Per-kernel device time sampled during the last solve (ms per
        launch): p update, stencil (A~p, p.q), update (x, r, r.r), reliable
        update, the preconditioner (V-cycle + r.z) and one fine-level
        multigrid smoothing step; ``stencil_kind`` is the CG stencil the plan
        runs (5: the direction update formed inside the stencil)."""
        ms = (ctypes.c_double * 6)()
        ns = ctypes.c_longlong()
        L.check("fs_pcg_plan_kernel_times",
                L.load_library().fs_pcg_plan_kernel_times(self._last_plan, ms,
                                                          ctypes.byref(ns)))
        n = max(ns.value, 1)
        kind = L.load_library().fs_pcg_plan_stencil_kind(self._last_plan)
        return {"samples": ns.value, "pupdate_ms": ms[0] / n, "stencil_ms": ms[1] / n,
                "update_ms": ms[2] / n, "reliable_ms": ms[3] / n,
                "precond_ms": ms[4] / n, "smoother_ms": ms[5] / n, "stencil_kind": kind}

    def close(self) -> None:
        lib = L.load_library()
        for plan in (getattr(self, "_plan", None),
                     (getattr(self, "_fp64", None) or (None,))[0]):
            if plan is not None and plan.value:
                lib.fs_pcg_plan_destroy(plan)
        self._plan = None
        self._fp64 = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
