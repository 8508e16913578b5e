"""The in-house direct solves that replaced cuSOLVER on the evaluation paths:

* the pivoted LU (k_lu_factor + k_lu_back) of an indefinite reduced EEQ matrix, against the
  CPU oracle (which falls back to an LU of the augmented system the way curcuma does,
  eeq_solver.cpp:1448-2086);
* the second right-hand side of the exact-gradient mode (the charge response of Coulomb pairs
  cut at 100 bohr) with that LU factor (k_lu_solve_rhs) and with a Cholesky factor
  (k_chol_solve_rhs, after the tiled Cholesky or cuSOLVER's when asked for), against central
  finite differences (h = 1e-4 bohr);
* the default solver choice of a small molecule no longer includes cuSOLVER.
"""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, workloads
from tests.indefinite_systems import h2_chain
from tests.oracle_api import Oracle

pytestmark = pytest.mark.gpu

BOHR = 0.529177210903


def _fd_worst(g, X, atoms):
    g.updateGeometry(X)
    g.calculateEnergy(True)
    G = g.getGradient()
    h = 1e-4 * BOHR
    worst = 0.0
    for a in atoms:
        for d in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[a, d] += h
            Xm[a, d] -= h
            g.updateGeometry(Xp)
            ep = g.calculateEnergy(True)
            g.updateGeometry(Xm)
            em = g.calculateEnergy(True)
            worst = max(worst, abs((ep - em) / 2e-4 - G[a, d]))
    g.updateGeometry(X)
    return worst


def test_indefinite_matrix_takes_the_lu_and_matches_the_oracle():
    Z, X = h2_chain()
    g = GFNFF()
    assert g.setMolecule(Z, X), g.getErrorMessage()
    assert g.eeqSolver() == "lu"
    e = g.calculateEnergy(True)
    assert not g.hasError(), g.getErrorMessage()
    T, G, q, cn = Oracle(Z, X).engrad(X)
    assert abs(e - T["total"]) < 1e-8
    assert np.abs(g.getGradient() - G).max() < 1e-7
    assert np.abs(g.getCharges() - q).max() < 1e-9
    # repeated evaluations (the factor is rebuilt every step)
    for k in range(2):
        Xk = X + np.random.default_rng(k).normal(scale=0.01, size=X.shape)
        assert g.updateGeometry(Xk)
        e = g.calculateEnergy(True)
        T, G, q, cn = Oracle(Z, X).engrad(Xk)
        assert abs(e - T["total"]) < 1e-8


def test_exact_gradient_with_the_lu_factor():
    Z, X = h2_chain()
    g = GFNFF(exact_gradient=True)
    assert g.setMolecule(Z, X), g.getErrorMessage()
    assert g.eeqSolver() == "lu"
    assert _fd_worst(g, X, [0, 31, 58, 70]) < 1e-6


@pytest.mark.parametrize("solver", ["tiled", "library"])
def test_exact_gradient_with_a_cholesky_factor(solver, monkeypatch):
    """C64H130 spans more than 100 bohr: the charge response is solved with the factor of
    the step's EEQ matrix (k_chol_solve_rhs)."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", solver)
    Z, X = workloads.alkane(64, 1001)
    g = GFNFF(exact_gradient=True)
    assert g.setMolecule(Z, X), g.getErrorMessage()
    assert g.eeqSolver() == solver
    assert _fd_worst(g, X, [0, 5, 100, 191]) < 1e-6


def test_default_choice_is_an_in_house_solver():
    for Z, X in (workloads.alkane(64, 1001), workloads.water_cluster(60, 4)):
        g = GFNFF()
        assert g.setMolecule(Z, X), g.getErrorMessage()
        assert g.eeqSolver() in ("tiled", "pcg", "batched")
