"""GPU heat conduction against the reference (needs a B200).

``ThermalSolver`` steady (Dirichlet heat sink + convective walls), theta
scheme transients (backward Euler and Crank-Nicolson) and the thermal
resistance, recorded from the reference in ``tests/golden/thermal.npz``.
The reference factorises this small system; the GPU iterates to relres
1e-13, so temperatures agree to 1e-8 of the largest temperature rise.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONV = {"zhi": (2e4, 310.0), "xlo": (5e3, 295.0)}


def _solver(golden, precision="auto", preconditioner="mg"):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.thermal import ThermalSolver
    d = golden("thermal")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    s = ThermalSolver(g, d["kappa"], d["rho_cp"], SolverConfig(tol=1e-13),
                      gpu=GPUConfig(precision=precision, preconditioner=preconditioner))
    return d, s


@pytest.mark.parametrize("preconditioner", ["mg", "jacobi"])
@pytest.mark.parametrize("precision", ["auto", "fp64"])
def test_steady_matches_reference(cuda, golden, precision, preconditioner):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    d, s = _solver(golden, precision, preconditioner)
    r = s.steady(d["q"], bc=BoundarySpec(zlo=Dirichlet(300.0)), convection=CONV)
    T = r.fields["T"][0]
    rise = np.abs(d["T_steady"] - 300.0).max()
    assert np.abs(T - d["T_steady"]).max() <= 1e-8 * rise
    assert r.scalars["power_in"][0] == pytest.approx(d["q"].sum(), rel=1e-15)


@pytest.mark.parametrize("theta", [1.0, 0.5])
def test_transient_matches_reference(cuda, golden, theta):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    d, s = _solver(golden)
    r = s.transient(d["q"], t_end=2e-5, dt=1e-6, T0=300.0, bc=BoundarySpec(zlo=Dirichlet(300.0)),
                    convection=CONV, theta=theta, store=True)
    want = d[f"T_transient_theta{theta:g}"]
    assert r.fields["T"].shape == want.shape
    assert np.abs(r.fields["T"] - want).max() <= 1e-8 * np.abs(want - 300.0).max()
    assert r.scalars["T_max"][-1] == pytest.approx(want[-1].max(), rel=1e-10)


def test_thermal_resistance_matches_reference(cuda, golden):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    d, s = _solver(golden)
    R = s.thermal_resistance(d["src"], bc=BoundarySpec(zlo=Dirichlet(300.0)), convection=CONV,
                             power=1e-3)
    assert R == pytest.approx(float(d["R_th"]), rel=1e-8)


def test_thermal_input_checks(cuda, golden):
    from fieldspice_b200.solvers.thermal import ThermalSolver
    d, s = _solver(golden)
    with pytest.raises(ValueError, match="strictly positive"):
        ThermalSolver(s.grid, -d["kappa"])
    with pytest.raises(ValueError, match="rho_cp_cell"):
        ThermalSolver(s.grid, d["kappa"]).transient(0.0, 1e-6, 1e-7)
    with pytest.warns(RuntimeWarning, match="adiabatic"):
        with pytest.raises(Exception):
            s.steady(d["q"])
