"""The oracle's ALPB implicit solvation (oracle/alpb_oracle.cpp, the restatement of curcuma's
ff_methods/alpb_solvation.cpp) against curcuma's own golden totals: xtb 6.7.1
``--gfnff --alpb`` for 7 molecules in 4 solvents, which curcuma's
``validate_gfnff_solvation.py`` checks at 1e-7 Eh (fixture: tests/golden/alpb/).  The
solvation gradient (Born pairs, Born radii, surface areas, HB weights, shape term) against
central differences: its error is the one of the gas-phase gradient, because the reference
gradient's known approximations (the D4 dC6/dCN term) are the same with and without the
solvent."""
import json
from pathlib import Path

import numpy as np
import pytest

from tests.oracle_api import Oracle

FIX = json.loads((Path(__file__).parent / "golden" / "alpb" / "gfnff_alpb_xtb.json").read_text())
BOHR = 0.529177210903


@pytest.mark.parametrize("mol", list(FIX["molecules"]))
def test_alpb_totals_match_xtb(mol):
    rec = FIX["molecules"][mol]
    Z, X = np.array(rec["Z"]), np.array(rec["xyz_angstrom"])
    for solvent, e_ref in rec["total"].items():
        T, G, q, cn = Oracle(Z, X, solvent=solvent).engrad(X)
        assert abs(T["total"] - e_ref) <= FIX["tolerance"], (mol, solvent, T["total"] - e_ref)
        assert T["solvation"] < 0.0
        assert abs(q.sum()) < 1e-10


def test_solvent_aliases_and_unknown():
    rec = FIX["molecules"]["H2O"]
    Z, X = np.array(rec["Z"]), np.array(rec["xyz_angstrom"])
    a = Oracle(Z, X, solvent="h2o").engrad(X)[0]["total"]
    b = Oracle(Z, X, solvent="Water").engrad(X)[0]["total"]
    assert a == b
    assert Oracle(Z, X, solvent="none").engrad(X)[0]["solvation"] == 0.0
    with pytest.raises(RuntimeError):
        Oracle(Z, X, solvent="liquid-nitrogen")


@pytest.mark.parametrize("mol,solvent", [("H2O", "water"), ("acetic_acid_dimer", "chloroform"),
                                         ("caffeine", "dmso")])
def test_alpb_gradient_central_differences(mol, solvent):
    rec = FIX["molecules"][mol]
    Z, X = np.array(rec["Z"]), np.array(rec["xyz_angstrom"])
    h = 1e-4 * BOHR
    err = {}
    for s in (None, solvent):
        o = Oracle(Z, X, solvent=s)
        G = o.engrad(X)[1]
        e = np.zeros(G.shape)
        for a in range(min(len(Z), 5)):
            for d in range(3):
                Xp, Xm = X.copy(), X.copy()
                Xp[a, d] += h
                Xm[a, d] -= h
                fd = (o.engrad(Xp)[0]["total"] - o.engrad(Xm)[0]["total"]) / 2e-4
                e[a, d] = fd - G[a, d]
        err[s] = e
    assert np.abs(err[solvent] - err[None]).max() < 1e-7


def test_alpb_gradient_of_a_cation():
    """NH4+ beside a water: the shape term (1/2 keps alpbet / adet (sum q)^2) and its
    gradient only act on a charged solute."""
    t = 1.03 / np.sqrt(3.0)
    a = np.deg2rad(104.52 / 2)
    X = np.array([[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t], [3.5, 0, 0],
                  [3.5 + 0.9572 * np.cos(a), 0.9572 * np.sin(a), 0], [3.5 + 0.9572 * np.cos(a), -0.9572 * np.sin(a), 0]])
    Z = np.array([7, 1, 1, 1, 1, 8, 1, 1])
    h = 1e-4 * BOHR
    err = {}
    for s in (None, "water"):
        o = Oracle(Z, X, charge=1, solvent=s)
        T, G, q, cn = o.engrad(X)
        assert abs(q.sum() - 1.0) < 1e-10
        e = np.zeros(G.shape)
        for a_ in range(len(Z)):
            for d in range(3):
                Xp, Xm = X.copy(), X.copy()
                Xp[a_, d] += h
                Xm[a_, d] -= h
                e[a_, d] = (o.engrad(Xp)[0]["total"] - o.engrad(Xm)[0]["total"]) / 2e-4 - G[a_, d]
        err[s] = e
        if s:
            assert T["solvation"] < -0.2
    assert np.abs(err["water"] - err[None]).max() < 1e-8
