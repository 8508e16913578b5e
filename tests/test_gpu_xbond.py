"""Halogen bonds on the GPU (k_xbonds) against the CPU oracle's restatement of
calcHalogenBonds (ff_workspace_gfnff.cpp:1411-1524): FP64 per term and total at 1e-10 /
1e-8 Eh, gradient at 1e-7 Eh/bohr; mixed at 1e-6 / 1e-5; and the exact-gradient mode's
gradient against central finite differences of the GPU energy (h = 1e-4 bohr)."""
import numpy as np
import pytest

from curcuma_b200 import FP64, GFNFF, MIXED
from tests.halogen_dimers import dimer
from tests.oracle_api import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("x_el", [17, 35, 53])
def test_xbond_against_oracle(x_el):
    Z, X = dimer(x_el)
    T, G, q, cn = Oracle(Z, X).engrad(X)
    assert T["xbond"] < -1e-3
    for prec, te, tg in ((FP64, 1e-8, 1e-7), (MIXED, 1e-6, 1e-5)):
        g = GFNFF(precision=prec)
        assert g.setMolecule(Z, X), g.getErrorMessage()
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        d = g.getEnergyDecomposition()
        assert len(g.topology(7, 3)) == 1
        assert abs(d["xbond"] - T["xbond"]) < (1e-10 if prec == FP64 else 1e-7)
        assert abs(e - T["total"]) < te
        assert np.abs(g.getGradient() - G).max() < tg


def test_xbond_exact_gradient_finite_differences():
    Z, X = dimer(35)
    g = GFNFF(exact_gradient=True)
    assert g.setMolecule(Z, X), g.getErrorMessage()
    g.calculateEnergy(True)
    G = g.getGradient()
    h = 1e-4 * 0.529177210903
    for a in (0, 1, 5):   # C, Br, N
        for c in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[a, c] += h
            Xm[a, c] -= h
            g.updateGeometry(Xp)
            ep = g.calculateEnergy(True)
            g.updateGeometry(Xm)
            em = g.calculateEnergy(True)
            assert abs((ep - em) / 2e-4 - G[a, c]) < 1e-6, (a, c)
