"""Periodic boundary conditions on the device (gfnff_set_unit_cell; the minimum image in the
CN, bond, angle, HB, XB, repulsion and pair kernels, the EEQ matrix on plain distances, as
in curcuma's CUDA kernels) against the oracle's restatement of the same rules
(tests/test_oracle_pbc.py): per term 1e-8 Eh, gradient 1e-7 Eh/bohr, charges 1e-9, CN 1e-12
in the FP64 form; 1e-6 / 1e-5 in the mixed form."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, MIXED, workloads
from tests.oracle_api import Oracle, OracleSequence
from tests.test_oracle_pbc import face_dimer

pytestmark = pytest.mark.gpu


def _cases():
    Z, X = workloads.water_cluster(48, 5)
    L = workloads.water_box_edge(48) + 2.8
    tri = np.eye(3) * L
    tri[1] = [0.3 * L, L, 0.0]
    tri[2] = [0.2 * L, -0.1 * L, L]
    Zd, Xd = face_dimer()
    Zb, Xb = workloads.water_cluster(1000, 9)
    Lb = workloads.water_box_edge(1000) + 2.8
    Zp, Xp = workloads.solvated_peptide(6, 60, 13)
    Lp = (Xp.max(0) - Xp.min(0)).max() + 2.5
    return {"face_dimer": (Zd, Xd, np.eye(3) * 10.0),
            "water48_cubic": (Z, X, np.eye(3) * L),
            "water48_triclinic": (Z, X, tri),
            "water1000": (Zb, Xb, np.eye(3) * Lb),
            "peptide": (Zp, Xp - Xp.min(0), np.eye(3) * Lp)}


CASES = _cases()


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("precision", [0, MIXED], ids=["fp64", "mixed"])
def test_pbc_against_oracle(case, precision):
    Z, X, cell = CASES[case]
    g = GFNFF(precision=precision, unit_cell=cell)
    assert g.setMolecule(Z, X), g.getErrorMessage()
    # the oracle with the library's HB/XB and topology refreshes (plain displacements)
    o = OracleSequence(Z, X, unit_cell=cell)
    etol, gtol, qtol, ctol = (1e-8, 1e-7, 1e-9, 1e-12) if precision == 0 else (1e-6, 1e-5, 1e-6, 1e-7)
    rng = np.random.default_rng(2)
    X2 = X + rng.normal(scale=0.02, size=X.shape)
    assert list(Z[-3:]) == [8, 1, 1]
    X2[-3:] += cell[0] - cell[2]          # the last water moved by the lattice vector a - c
    for geo in (X, X2):
        assert g.updateGeometry(geo)
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        T, G, q, cn = o.engrad(geo)
        dec = g.getEnergyDecomposition()
        for k in T:
            assert abs(dec[k] - T[k]) < etol, (case, k, dec[k] - T[k])
        assert abs(e - T["total"]) < etol
        assert np.abs(g.getGradient() - G).max() < gtol
        assert np.abs(g.getCharges() - q).max() < qtol
        assert np.abs(g.getCN() - cn).max() < ctol


def test_large_cell_equals_isolated():
    Z, X, cell = CASES["water48_cubic"]
    a = GFNFF()
    b = GFNFF(unit_cell=cell * 10.0)
    assert a.setMolecule(Z, X) and b.setMolecule(Z, X)
    ea, eb = a.calculateEnergy(True), b.calculateEnergy(True)
    assert abs(ea - eb) < 1e-9
    assert np.abs(a.getGradient() - b.getGradient()).max() < 1e-9


def test_cell_refusals():
    Z, X, cell = CASES["water48_cubic"]
    with pytest.raises(ValueError):
        GFNFF(unit_cell=cell, exact_gradient=True)
    with pytest.raises(ValueError):
        GFNFF(unit_cell=[[1, 0, 0], [2, 0, 0], [0, 0, 1]])
    g = GFNFF(unit_cell=cell, solvent="water")
    assert not g.setMolecule(Z, X)
    g = GFNFF(unit_cell=cell)
    assert not g.setMoleculeBatch(workloads.conformer_batch(2, 3, lo=20, hi=30))
    # the same handle without the cell afterwards: the isolated result
    g.setParameters({"unit_cell": None})
    assert g.setMolecule(Z, X)
    e = g.calculateEnergy(True)
    assert abs(e - Oracle(Z, X).engrad(X)[0]["total"]) < 1e-8
