"""Host-side pieces of ``bench.py`` (CPU): the iteration counts behind the
reference baseline's projection belong to the shape they were recorded at."""

import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_iterations_follow_the_shape(bench):
    iters, src = bench._reference_iterations(bench.SHAPE)
    assert bench.FULLSIZE_JSON.exists()
    assert len(iters) == bench.NBOX and min(iters) > 1000 and "full-size" in src
    # the recorded full-size counts are not reused at another shape
    other = (48, 48, 24)
    none, why = bench._reference_iterations(other)
    assert none is None and "48" in why
    jac = [300 + i for i in range(bench.NBOX)]
    got, src = bench._reference_iterations(other, jac)
    assert got == jac and "Jacobi" in src
    assert bench.WHOLE_REFERENCE_NODES >= 48 * 48 * 24


def test_projection_arithmetic(bench):
    # set-up outside CG plus ms per iteration times the iterations to 1e-10
    t_ext, t_setup, t_iter = bench._project(10.0, 4.0, 40, [100] * 8)
    assert t_setup == pytest.approx(6.0)
    assert t_iter == pytest.approx(0.1)
    assert t_ext == pytest.approx(6.0 + 0.1 * 800)
