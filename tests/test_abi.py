"""The C-ABI library loads and exports what ``include/*.h`` declares (CPU).

No compute call is made here: only symbol lookup, status strings and the
argument checks that return before any CUDA call.
"""

import ctypes
import re
from pathlib import Path

import pytest

from fieldspice_b200 import _lib as L
from fieldspice_b200._build import LIB_PATH, build

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(fs_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def dll():
    build()
    return L.load_library()


def test_every_declared_symbol_is_exported(dll):
    names = declared_symbols()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(dll, n), n
    assert names == set(L.EXPORTED_SYMBOLS), names ^ set(L.EXPORTED_SYMBOLS)


def test_status_strings(dll):
    assert dll.fs_version().decode().startswith("fieldspice_b200")
    assert dll.fs_status_string(L.FS_OK).decode() == "ok"
    assert "converged" in dll.fs_status_string(L.FS_NOT_CONVERGED).decode()
    assert dll.fs_status_string(99).decode() == "unknown status"


def test_workspace_sizes_and_bad_arguments(dll):
    nb = ctypes.c_size_t()
    assert dll.fs_pcg_workspace_bytes(32, 32, 16, 8, L.PRECISION_MIXED, 0, ctypes.byref(nb)) == L.FS_OK
    n = 32 * 32 * 16
    # label + s64 + 3 FP32 masses + 4 FP32 vectors of 8 RHS
    assert nb.value >= n * (1 + 8 + 12 + 4 * 8 * 4)
    nb64 = ctypes.c_size_t()
    assert dll.fs_pcg_workspace_bytes(32, 32, 16, 8, L.PRECISION_FP64, 0, ctypes.byref(nb64)) == L.FS_OK
    assert nb64.value > nb.value
    nbmg = ctypes.c_size_t()
    assert dll.fs_pcg_workspace_bytes(32, 32, 16, 8, L.PRECISION_MIXED, L.PRECOND_MG,
                                      ctypes.byref(nbmg)) == L.FS_OK
    assert nbmg.value > nb.value
    assert dll.fs_pcg_workspace_bytes(32, 32, 16, 8, 1, 7, ctypes.byref(nb)) == L.FS_BAD_ARG
    for k in (0, 3, 5, 17):
        assert dll.fs_pcg_workspace_bytes(32, 32, 16, k, 1, 0, ctypes.byref(nb)) == L.FS_BAD_ARG
    assert dll.fs_pcg_workspace_bytes(1, 32, 16, 8, 1, 0, ctypes.byref(nb)) == L.FS_BAD_ARG
    assert dll.fs_pcg_workspace_bytes(32, 32, 16, 8, 7, 0, ctypes.byref(nb)) == L.FS_BAD_ARG
    null = ctypes.c_void_p(0)
    assert dll.fs_build_masses(*([null] * 7), 4, 4, 4, 0, null, null, null, null) == L.FS_BAD_ARG
    plan = ctypes.c_void_p()
    assert dll.fs_pcg_plan_create(8, 8, 8, 3, 1, 0, *([null] * 7), 0, ctypes.byref(plan), null) == L.FS_BAD_ARG
    assert dll.fs_pcg_plan_destroy(null) == L.FS_OK
    assert dll.fs_group_apply_workspace_bytes(0, 8, ctypes.byref(nb)) == L.FS_BAD_ARG
    assert dll.fs_quadform_workspace_bytes(17, ctypes.byref(nb)) == L.FS_BAD_ARG
    # the property statistics validate before touching the device
    one = ctypes.c_void_p(256)
    stats = (ctypes.c_double * 3)()
    ws = L.PROP_STATS_WORKSPACE_BYTES
    assert dll.fs_prop_stats_enqueue(null, 10, one, ws, null) == L.FS_BAD_ARG
    assert dll.fs_prop_stats_enqueue(one, 0, one, ws, null) == L.FS_BAD_ARG
    assert dll.fs_prop_stats_enqueue(one, 10, one, ws - 16, null) == L.FS_BAD_ARG
    assert dll.fs_prop_stats_enqueue(one, 10, ctypes.c_void_p(264), ws, null) == L.FS_BAD_ARG
    assert dll.fs_prop_stats(one, 10, None, one, ws, null) == L.FS_BAD_ARG
    assert dll.fs_prop_stats(null, 10, stats, one, ws, null) == L.FS_BAD_ARG
    # the result offset the host reads is inside the workspace, 16-byte aligned
    assert L.PROP_STATS_RESULT_OFFSET % 16 == 0
    assert L.PROP_STATS_RESULT_OFFSET + 24 <= ws


def test_multigrid_parameters_are_validated(dll):
    # per-plan options: the sizing call checks them and touches no device
    p = L.FsMgParams()
    dll.fs_mg_params_default(ctypes.byref(p))
    assert (p.smooth_deg, p.smooth_lo, p.coarse_deg, p.coarse_lo, p.coarsest_nodes,
            p.stencil_kind, p.agg_alpha) == (2, 0.3, 32, 0.06, 4096, -1, 1.7)
    nb = ctypes.c_size_t()
    args = (64, 64, 32, 8, L.PRECISION_MIXED, L.PRECOND_MG)
    assert dll.fs_pcg_workspace_bytes_opt(*args, ctypes.byref(p), ctypes.byref(nb)) == L.FS_OK
    default = nb.value
    assert dll.fs_pcg_workspace_bytes_opt(*args, None, ctypes.byref(nb)) == L.FS_OK
    assert nb.value == default
    for field, bad in [("smooth_deg", 0), ("smooth_lo", 2.0), ("coarse_deg", 65),
                       ("coarse_lo", 0.0), ("coarsest_nodes", 4), ("stencil_kind", 8),
                       ("stencil_kind", -2), ("agg_alpha", 0.0), ("agg_alpha", 2.0)]:
        q = L.FsMgParams()
        dll.fs_mg_params_default(ctypes.byref(q))
        setattr(q, field, bad)
        assert dll.fs_pcg_workspace_bytes_opt(*args, ctypes.byref(q),
                                              ctypes.byref(nb)) == L.FS_BAD_ARG, field
    # a deeper hierarchy (smaller coarsest level) needs more workspace
    q = L.mg_params({"coarsest_nodes": 64})
    assert dll.fs_pcg_workspace_bytes_opt(*args, ctypes.byref(q), ctypes.byref(nb)) == L.FS_OK
    assert nb.value > default
    with pytest.raises(ValueError, match="unknown"):
        L.mg_params({"smoothing": 3})


def test_library_is_sm100a_only():
    # the build flags target sm_100a and nothing else
    from fieldspice_b200 import _build
    assert _build.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert LIB_PATH.exists()


def test_product_path_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        L.lib()


def test_header_constants_match_the_binding():
    """The #define values the Python binding repeats."""
    text = (ROOT / "include" / "fieldspice_b200.h").read_text()
    defs = dict(re.findall(r"#define\s+(FS_[A-Z0-9_]+)\s+(\d+)", text))
    assert int(defs["FS_PROP_STATS_WORKSPACE_BYTES"]) == L.PROP_STATS_WORKSPACE_BYTES
    assert int(defs["FS_PROP_STATS_RESULT_OFFSET"]) == L.PROP_STATS_RESULT_OFFSET
