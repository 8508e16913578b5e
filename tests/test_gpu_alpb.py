"""ALPB implicit solvation on the device (k_alpb.cuh; the Born matrix inside the EEQ matrix)
against the CPU oracle and curcuma's golden totals:

* the 7 molecules x 4 solvents of curcuma's xtb 6.7.1 ``--gfnff --alpb`` references at the
  reference test's 1e-7 Eh, and against the oracle per term;
* larger solutes (a 200-water cluster, a solvated peptide, a charged molecule) against the
  oracle: energy 1e-8 Eh, gradient 1e-7 Eh/bohr, charges 1e-9 (FP64 form), 1e-6 / 1e-5 in the
  mixed form;
* the exact-gradient mode against central differences (h = 1e-4 bohr), including the shape
  term of a charged solute."""
import json
from pathlib import Path

import numpy as np
import pytest

from curcuma_b200 import GFNFF, MIXED, workloads
from tests.oracle_api import Oracle

pytestmark = pytest.mark.gpu

FIX = json.loads((Path(__file__).parent / "golden" / "alpb" / "gfnff_alpb_xtb.json").read_text())
BOHR = 0.529177210903


def _ammonium_water():
    t = 1.03 / np.sqrt(3.0)
    a = np.deg2rad(104.52 / 2)
    X = np.array([[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t], [3.5, 0, 0],
                  [3.5 + 0.9572 * np.cos(a), 0.9572 * np.sin(a), 0], [3.5 + 0.9572 * np.cos(a), -0.9572 * np.sin(a), 0]])
    return np.array([7, 1, 1, 1, 1, 8, 1, 1]), X


@pytest.mark.parametrize("mol", list(FIX["molecules"]))
def test_alpb_golden_totals(mol):
    rec = FIX["molecules"][mol]
    Z, X = np.array(rec["Z"]), np.array(rec["xyz_angstrom"])
    for solvent, e_ref in rec["total"].items():
        g = GFNFF(solvent=solvent)
        assert g.setMolecule(Z, X), g.getErrorMessage()
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        assert abs(e - e_ref) <= FIX["tolerance"], (mol, solvent, e - e_ref)
        T, G, q, cn = Oracle(Z, X, solvent=solvent).engrad(X)
        assert abs(g.getEnergyDecomposition()["solvation"] - T["solvation"]) < 1e-10
        assert np.abs(g.getGradient() - G).max() < 1e-8
        assert np.abs(g.getCharges() - q).max() < 1e-10


@pytest.mark.parametrize("case", ["water200", "peptide", "cation"])
@pytest.mark.parametrize("precision", [0, MIXED], ids=["fp64", "mixed"])
def test_alpb_against_oracle(case, precision):
    solvent, charge = {"water200": ("water", 0), "peptide": ("dmso", 0), "cation": ("water", 1)}[case]
    Z, X = {"water200": lambda: workloads.water_cluster(200, 21),
            "peptide": lambda: workloads.solvated_peptide(8, 60, 22),
            "cation": _ammonium_water}[case]()
    g = GFNFF(precision=precision, solvent=solvent)
    assert g.setMolecule(Z, X, charge), g.getErrorMessage()
    e = g.calculateEnergy(True)
    assert not g.hasError(), g.getErrorMessage()
    T, G, q, cn = Oracle(Z, X, charge, solvent=solvent).engrad(X)
    etol, gtol, qtol = (1e-8, 1e-7, 1e-9) if precision == 0 else (1e-6, 1e-5, 1e-6)
    assert abs(e - T["total"]) < etol, (e, T["total"])
    assert abs(g.getEnergyDecomposition()["solvation"] - T["solvation"]) < etol
    assert np.abs(g.getGradient() - G).max() < gtol
    assert np.abs(g.getCharges() - q).max() < qtol
    # a second geometry: the Born radii, surfaces and the solve follow the atoms
    X2 = X + np.random.default_rng(4).normal(scale=0.03, size=X.shape)
    assert g.updateGeometry(X2)
    e2 = g.calculateEnergy(True)
    T2, G2, q2, _ = Oracle(Z, X, charge, solvent=solvent).engrad(X2)
    assert abs(e2 - T2["total"]) < etol
    assert np.abs(g.getGradient() - G2).max() < gtol


@pytest.mark.parametrize("case", ["alkane", "cation"])
def test_alpb_exact_gradient_central_differences(case):
    Z, X = workloads.alkane(12, 3) if case == "alkane" else _ammonium_water()
    charge = 1 if case == "cation" else 0
    g = GFNFF(exact_gradient=True, solvent="water")
    assert g.setMolecule(Z, X, charge)
    g.calculateEnergy(True)
    G = g.getGradient()
    h = 1e-4 * BOHR
    worst = 0.0
    for a in range(min(len(Z), 8)):
        for d in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[a, d] += h
            Xm[a, d] -= h
            g.updateGeometry(Xp)
            ep = g.calculateEnergy(True)
            g.updateGeometry(Xm)
            em = g.calculateEnergy(True)
            worst = max(worst, abs((ep - em) / 2e-4 - G[a, d]))
    assert worst < 1e-6, worst


def test_alpb_unknown_solvent_and_batches():
    with pytest.raises(ValueError):
        GFNFF(solvent="liquid-nitrogen")
    g = GFNFF(solvent="water")
    mols = workloads.conformer_batch(3, 5, lo=20, hi=40)
    assert not g.setMoleculeBatch(mols)
