"""Mixed-precision form (FP32 arithmetic in the short-range pair, CN, repulsion and
hydrogen-bond terms; FP64 positions, long-range Coulomb, EEQ and all sums) against the
CPU oracle.  Bar: |dE| <= 1e-6 Eh and max |dF| <= 1e-5 Eh/bohr, topology unchanged."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, workloads
from curcuma_b200 import MIXED as GFNFF_MIXED
from tests.oracle_api import Oracle, golden

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
G_TOL = 1e-5


def _mixed_vs_oracle(Z, X, charge=0):
    gpu = GFNFF(precision=GFNFF_MIXED)
    assert gpu.setMolecule(Z, X, charge), gpu.getErrorMessage()
    e = gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    o = Oracle(Z, X, charge)
    T, G, q, cn = o.engrad(X)
    assert abs(e - T["total"]) <= E_TOL, (e, T["total"])
    dg = np.abs(gpu.getGradient() - G).max()
    assert dg <= G_TOL, dg
    return gpu, e - T["total"], dg


@pytest.mark.parametrize("name", ["caffeine", "complex", "polymer", "acetic_acid_dimer"])
def test_mixed_golden(name):
    g = golden(name)
    _mixed_vs_oracle(np.array(g["Z"]), np.array(g["xyz_angstrom"]))


def test_mixed_water_cluster():
    Z, X = workloads.water_cluster(400, 31)
    _mixed_vs_oracle(Z, X)


def test_mixed_alkane_and_peptide():
    _mixed_vs_oracle(*workloads.alkane(64, 1001))
    _mixed_vs_oracle(*workloads.solvated_peptide(8, 60, 12))


def test_mixed_topology_matches_fp64():
    Z, X = workloads.water_cluster(50, 3)
    a, b = GFNFF(), GFNFF(precision=GFNFF_MIXED)
    assert a.setMolecule(Z, X) and b.setMolecule(Z, X)
    for kind, width in [(0, 2), (1, 3), (4, 2), (6, 4), (8, 1), (9, 1)]:
        assert np.array_equal(a.topology(kind, width), b.topology(kind, width)), kind


@pytest.mark.parametrize("system", ["water400", "peptide"])
def test_mixed_fp32_pcg_matrix(system, monkeypatch):
    """The mixed form's optional FP32-stored lower-triangle PCG matrix (GFNFF_PCG_F32=1,
    forced here on smaller systems): energy and gradient stay within the mixed bar against
    the oracle."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", "pcg")
    monkeypatch.setenv("GFNFF_PCG_SYM", "1")
    monkeypatch.setenv("GFNFF_PCG_F32", "1")
    Z, X = {"water400": lambda: workloads.water_cluster(400, 31),
            "peptide": lambda: workloads.solvated_peptide(8, 60, 12)}[system]()
    gpu, de, dg = _mixed_vs_oracle(Z, X)
    assert gpu.eeqSolver() == "pcg"
