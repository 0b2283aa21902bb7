"""ctypes binding of the C ABI in ``include/fieldspice_b200.h``.

The product path has no CPU fallback: if the shared library is missing, or
no CUDA device is visible, every entry point raises.  Device memory and
streams come from PyTorch (plumbing only); the library receives raw device
pointers and a ``cudaStream_t``.
"""

from __future__ import annotations

import ctypes
from ctypes import (POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_longlong,
                    c_size_t, c_void_p)

from ._build import LIB_PATH

__all__ = ["lib", "FsRhsStats", "check", "FsError", "stream_ptr", "ptr",
           "FS_OK", "FS_NOT_CONVERGED", "FS_TIMEOUT", "FS_BAD_ARG", "FS_NAN",
           "FS_CUDA_ERROR", "FS_STALLED", "LABEL_FREE", "LABEL_FIXED", "LABEL_SOLO",
           "LABEL_PINNED", "DTYPE_F64", "DTYPE_F32", "PRECISION_FP64",
           "PRECISION_MIXED", "PRECOND_JACOBI", "PRECOND_MG", "PRECOND_MG_AGG", "AVERAGE_PARALLEL", "AVERAGE_HARMONIC",
           "EXPORTED_SYMBOLS", "load_library"]

FS_OK, FS_NOT_CONVERGED, FS_TIMEOUT, FS_BAD_ARG, FS_NAN, FS_CUDA_ERROR, FS_STALLED = range(7)
LABEL_FREE, LABEL_FIXED, LABEL_SOLO, LABEL_PINNED = range(4)
DTYPE_F64, DTYPE_F32 = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
PRECOND_JACOBI, PRECOND_MG, PRECOND_MG_AGG = 0, 1, 2
PROP_STATS_WORKSPACE_BYTES = 16384  # FS_PROP_STATS_WORKSPACE_BYTES
PROP_STATS_RESULT_OFFSET = 14208    # FS_PROP_STATS_RESULT_OFFSET
AVERAGE_PARALLEL, AVERAGE_HARMONIC = 0, 1


class FsRhsStats(ctypes.Structure):
    _fields_ = [("iterations", c_int32), ("status", c_int32),
                ("relres", c_double), ("bnorm", c_double),
                ("reliable_updates", c_int32), ("reserved", c_int32)]


class FsMgParams(ctypes.Structure):
    """``fs_mg_params``: multigrid and stencil options of one plan."""
    _fields_ = [("smooth_deg", c_int32), ("smooth_lo", c_double),
                ("coarse_deg", c_int32), ("coarse_lo", c_double),
                ("coarsest_nodes", c_longlong), ("stencil_kind", c_int32),
                ("agg_alpha", c_double)]


def mg_params(opts: dict | None):
    """An ``FsMgParams`` from the library defaults updated by ``opts`` (keys
    as the struct fields), or None for the defaults."""
    if not opts:
        return None
    unknown = set(opts) - {f for f, _ in FsMgParams._fields_}
    if unknown:
        raise ValueError(f"unknown multigrid option(s): {sorted(unknown)}")
    p = FsMgParams()
    load_library().fs_mg_params_default(ctypes.byref(p))
    for k, v in opts.items():
        setattr(p, k, v)
    return p


class FsError(RuntimeError):
    """A library call returned a status other than FS_OK."""

    def __init__(self, where: str, status: int, detail: str = ""):
        self.status = status
        msg = f"{where}: {_status_text(status)}"
        if detail:
            msg += f" [{detail}]"
        super().__init__(msg)


_SIGNATURES = {
    "fs_version": (c_char_p, []),
    "fs_status_string": (c_char_p, [c_int]),
    "fs_last_error": (c_char_p, []),
    "fs_build_masses": (c_int, [c_void_p] * 7 + [c_int] * 4 + [c_void_p] * 4),
    "fs_combine_masses": (c_int, [c_void_p, c_void_p, c_double, c_double,
                                  c_void_p, c_longlong, c_void_p]),
    "fs_stencil_apply": (c_int, [c_void_p] * 6 + [c_int] * 5 + [c_void_p]),
    "fs_fill_unit_excitation": (c_int, [c_void_p] * 3 + [c_int] * 4 + [c_void_p]),
    "fs_set_dirichlet": (c_int, [c_void_p] * 4 + [c_int] * 3 + [c_void_p]),
    "fs_pcg_workspace_bytes": (c_int, [c_int] * 6 + [POINTER(c_size_t)]),
    "fs_pcg_plan_create": (c_int, [c_int] * 6 + [c_void_p] * 7 + [c_size_t,
                                   POINTER(c_void_p), c_void_p]),
    "fs_pcg_plan_create_diag": (c_int, [c_int] * 6 + [c_void_p] * 8 + [c_size_t,
                                        POINTER(c_void_p), c_void_p]),
    "fs_pcg_plan_create_ex": (c_int, [c_int] * 6 + [c_void_p] * 4 + [c_int] + [c_void_p] * 4
                              + [c_size_t, POINTER(c_void_p), c_void_p]),
    "fs_mg_params_default": (None, [POINTER(FsMgParams)]),
    "fs_pcg_plan_solve_begin": (c_int, [c_void_p, c_int, c_double, c_int, c_void_p]),
    "fs_pcg_plan_solve_poll": (c_int, [c_void_p, POINTER(FsRhsStats), POINTER(c_int)]),
    "fs_pcg_workspace_bytes_opt": (c_int, [c_int] * 6 + [POINTER(FsMgParams),
                                                         POINTER(c_size_t)]),
    "fs_pcg_plan_create_opt": (c_int, [c_int] * 6 + [c_void_p] * 4 + [c_int,
                               POINTER(FsMgParams)] + [c_void_p] * 4
                               + [c_size_t, POINTER(c_void_p), c_void_p]),
    "fs_periodic_masses": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "fs_pcg_plan_solve": (c_int, [c_void_p, c_int, c_double, c_int,
                                  POINTER(FsRhsStats), c_void_p]),
    "fs_pcg_plans_solve": (c_int, [POINTER(c_void_p), c_int, POINTER(c_void_p), c_int,
                                   c_double, c_int, POINTER(POINTER(FsRhsStats)),
                                   POINTER(c_int)]),
    "fs_conv3d_pack_weights": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]),
    "fs_conv3d_bf16": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p,
                               c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int,
                               c_int, c_int, c_int, c_int, c_int, c_int, c_void_p,
                               c_void_p]),
    "fs_unet_param_count": (c_int, [POINTER(c_longlong)]),
    "fs_unet_layer": (c_int, [c_int, POINTER(c_int), POINTER(c_int), POINTER(c_longlong),
                              POINTER(c_longlong)]),
    "fs_unet_workspace_bytes": (c_int, [c_int] * 5 + [POINTER(c_size_t)]),
    "fs_unet_create": (c_int, [c_int] * 5 + [c_void_p, c_void_p, c_size_t, POINTER(c_void_p),
                                             c_void_p]),
    "fs_unet_sync": (c_int, [c_void_p, c_void_p]),
    "fs_unet_forward": (c_int, [c_void_p, c_void_p, c_longlong, c_longlong, c_void_p, c_longlong,
                                c_void_p, c_longlong, c_void_p, c_longlong, c_longlong, c_void_p]),
    "fs_unet_train_step": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float,
                                   c_void_p, c_void_p]),
    "fs_unet_gradient": (c_int, [c_void_p] * 8),
    "fs_unet_adam_step": (c_int, [c_void_p, c_void_p, c_float, c_void_p]),
    "fs_unet_error": (c_int, [c_void_p, POINTER(c_int), c_void_p]),
    "fs_unet_destroy": (c_int, [c_void_p]),
    "fs_eq_apply": (c_int, [c_void_p] * 6 + [c_int] * 4 + [c_void_p]),
    "fs_pcg_plan_levels": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "fs_pcg_plan_level_data": (c_int, [c_void_p, c_int, POINTER(c_void_p), POINTER(c_void_p),
                                       POINTER(c_void_p)]),
    "fs_pcg_plan_unet_workspace_bytes": (c_int, [c_void_p, c_int, POINTER(c_size_t)]),
    "fs_pcg_plan_set_unet": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_size_t,
                                     c_void_p]),
    "fs_pcg_plan_sync_unet": (c_int, [c_void_p, c_void_p]),
    "fs_selftest_wait_timeout": (c_int, [c_longlong, POINTER(c_int), c_void_p]),
    "fs_prop_stats": (c_int, [c_void_p, c_longlong, POINTER(c_double), c_void_p, c_size_t,
                              c_void_p]),
    "fs_prop_stats_enqueue": (c_int, [c_void_p, c_longlong, c_void_p, c_size_t, c_void_p]),
    "fs_rhs_superpose": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double),
                                 c_void_p, c_void_p, c_longlong, c_void_p]),
    "fs_pcg_plan_precondition": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fs_pcg_plan_scale": (c_int, [c_void_p, POINTER(c_void_p), POINTER(c_void_p)]),
    "fs_pcg_plan_label_counts": (c_int, [c_void_p, POINTER(c_longlong), c_void_p]),
    "fs_pcg_plan_stencil_kind": (c_int, [c_void_p]),
    "fs_pcg_plan_stencil_times": (c_int, [c_void_p, POINTER(c_float)]),
    "fs_conv3d_wgrad_workspace_bytes": (c_int, [c_int, c_int, POINTER(c_size_t)]),
    "fs_conv3d_wgrad_bf16": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int,
                                     c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_size_t, c_void_p, c_void_p]),
    "fs_ac_workspace_bytes": (c_int, [c_int, c_int, c_int, c_int, c_int, POINTER(c_size_t)]),
    "fs_ac_solve": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_double, c_int, c_void_p, c_size_t,
                            POINTER(FsRhsStats), c_void_p]),
    "fs_pcg_plan_labels": (c_void_p, [c_void_p]),
    "fs_pcg_plan_launches": (c_longlong, [c_void_p]),
    "fs_pcg_plan_kernel_times": (c_int, [c_void_p, POINTER(c_double),
                                         POINTER(c_longlong)]),
    "fs_pcg_plan_destroy": (c_int, [c_void_p]),
    "fs_group_apply_workspace_bytes": (c_int, [c_int, c_int, POINTER(c_size_t)]),
    "fs_group_apply": (c_int, [c_void_p] * 10 + [c_int] * 5 + [c_void_p, c_void_p,
                               c_size_t, c_void_p]),
    "fs_group_apply_noalloc": (c_int, [c_void_p] * 10 + [c_int] * 5 + [c_void_p,
                                       c_void_p]),
    "fs_quadform_workspace_bytes": (c_int, [c_int, POINTER(c_size_t)]),
    "fs_quadform": (c_int, [c_void_p] * 4 + [c_int] * 4 + [c_void_p, c_void_p,
                            c_size_t, c_void_p]),
    "fs_apply_laplacian": (c_int, [c_void_p] * 6 + [c_int] * 4 + [c_void_p]),
}

#: Every symbol ``include/fieldspice_b200.h`` declares.
EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_LIB: ctypes.CDLL | None = None


def load_library(path=None) -> ctypes.CDLL:
    """Load the shared library and declare its signatures (no GPU needed)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = LIB_PATH if path is None else path
    if not p.exists():
        raise RuntimeError(
            f"the CUDA library {p} is not built; run "
            "`python -c 'import __graft_entry__ as g; g.build()'` first. "
            "fieldspice_b200 has no CPU fallback.")
    dll = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(dll, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = dll
    return dll


def prop_stats(t) -> tuple[float, float, float]:
    """``fs_prop_stats`` of an FP64 device tensor: (min, max, non-finite
    count), with its workspace from the framework's caching allocator."""
    import torch
    ws = torch.empty(PROP_STATS_WORKSPACE_BYTES, dtype=torch.uint8, device=t.device)
    stats = (ctypes.c_double * 3)()
    check("fs_prop_stats", lib().fs_prop_stats(ptr(t), t.numel(), stats, ptr(ws),
                                               PROP_STATS_WORKSPACE_BYTES, stream_ptr()))
    return float(stats[0]), float(stats[1]), float(stats[2])


class PendingStats:
    """An enqueued ``fs_prop_stats_enqueue``: the three results travel to a
    page-locked host buffer behind it on the same stream; ``result()`` waits
    for them."""

    def __init__(self, workspace, host, event):
        self._ws = workspace  # kept allocated until the copy has run
        self._host = host
        self._event = event

    def result(self) -> tuple[float, float, float]:
        self._event.synchronize()
        h = self._host
        return float(h[0]), float(h[1]), float(h[2])


def prop_stats_begin(t) -> PendingStats:
    """``prop_stats`` without waiting: the reduction and the copy of its three
    results are enqueued on the current stream."""
    import torch
    ws = torch.empty(PROP_STATS_WORKSPACE_BYTES, dtype=torch.uint8, device=t.device)
    check("fs_prop_stats_enqueue", lib().fs_prop_stats_enqueue(
        ptr(t), t.numel(), ptr(ws), PROP_STATS_WORKSPACE_BYTES, stream_ptr()))
    host = torch.empty(3, dtype=torch.float64, pin_memory=True)
    host.copy_(ws[PROP_STATS_RESULT_OFFSET:PROP_STATS_RESULT_OFFSET + 24].view(torch.float64),
               non_blocking=True)
    ev = torch.cuda.Event()
    ev.record()
    return PendingStats(ws, host, ev)


def lib() -> ctypes.CDLL:
    """The loaded library, after checking that a CUDA device is present."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError(
            "fieldspice_b200 needs a CUDA device (sm_100a); none is visible and "
            "there is no CPU fallback")
    return load_library()


def _status_text(status: int) -> str:
    try:
        return load_library().fs_status_string(status).decode()
    except Exception:  # pragma: no cover - only when the library is absent
        return f"status {status}"


def check(where: str, status: int) -> None:
    """Raise :class:`FsError` unless ``status`` is FS_OK."""
    if status != FS_OK:
        detail = ""
        if status == FS_CUDA_ERROR:
            detail = load_library().fs_last_error().decode()
        raise FsError(where, status, detail)


def stream_ptr(stream=None) -> c_void_p:
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return c_void_p(s.cuda_stream)


def ptr(t) -> c_void_p:
    """Raw device pointer of a tensor (``None`` -> NULL)."""
    if t is None:
        return c_void_p(0)
    return c_void_p(t.data_ptr())
