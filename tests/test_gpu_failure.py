"""Failure detection on the GPU without a GPU fault (needs a B200).

Every staged-load and tensor-core wait in the library is bounded: when its
budget runs out the thread records a timeout and returns instead of hanging.
Here a device thread waits on an mbarrier that nothing completes, with a
budget of ~1 ms of SM clocks; the host must read FS_TIMEOUT, and the context
must stay usable for a normal extraction afterwards.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(cuda):
    from fieldspice_b200 import _lib as L
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    lib = L.lib()
    st = ctypes.c_int(-1)
    L.check("selftest", lib.fs_selftest_wait_timeout(2_000_000, ctypes.byref(st), L.stream_ptr()))
    assert st.value == L.FS_TIMEOUT
    w = W.layered_boxes((24, 24, 16), nbox=3, seed=2)
    C = EX.capacitance_matrix(w.grid(), w.eps_cell, w.terminal_objects(), w.boundary_spec())
    assert C.shape == (3, 3) and np.all(np.isfinite(C)) and np.all(np.diag(C) > 0)


def test_selftest_rejects_bad_budget(cuda):
    from fieldspice_b200 import _lib as L
    st = ctypes.c_int(-1)
    assert L.lib().fs_selftest_wait_timeout(0, ctypes.byref(st), L.stream_ptr()) == L.FS_BAD_ARG
