"""Mixed form, batched EEQ on the tensor cores: FP32 Cholesky with 3xTF32 trailing updates
and FP64 iterative refinement to ||b - M y||_inf <= 1e-10 (k_eeq_tc.cuh), against the CPU
oracle per molecule (|dE| <= 1e-6 Eh, max |dF| <= 1e-5 Eh/bohr), and against the mixed form
with the FP64 batched Cholesky (GFNFF_BATCH_TC=0: the same right-hand sides, which the mixed
form's FP32 CN makes differ from the FP64 form's at ~1e-8; the charges of the two solves agree
to the refinement bar)."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, MIXED, workloads
from tests.oracle_api import Oracle, golden

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
G_TOL = 1e-5
Q_TOL = 1e-8   # same system: ||M dy||_inf <= 1e-10, lambda_min(M) >= 0.1, n <= 300
Q_TOL_ORACLE = 1e-6   # mixed form against the oracle (FP32 CN in the right-hand side)


def _ammonium_water():
    t = 1.03 / np.sqrt(3.0)
    nh4 = [[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t]]
    a = np.deg2rad(104.52 / 2)
    h2o = [[3.5, 0, 0], [3.5 + 0.9572 * np.cos(a), 0.9572 * np.sin(a), 0],
           [3.5 + 0.9572 * np.cos(a), -0.9572 * np.sin(a), 0]]
    return np.array([7, 1, 1, 1, 1, 8, 1, 1]), np.array(nh4 + h2o, dtype=float)


def _mols():
    """Sizes on both sides of the warp path (<= 70 unknowns) and at the panel edges of the
    tensor-core path: C37H76 (112 unknowns, a multiple of 16), C42H86 (127, one short of
    it), C100H202 (301, near the 303 limit); 30 waters (90 atoms, 30 fragments: the
    multi-fragment build); conformers of 20-300 atoms."""
    mols = workloads.conformer_batch(10, 91, lo=20, hi=300)
    mols += [workloads.alkane(37, 5), workloads.alkane(42, 6), workloads.alkane(100, 7),
             workloads.water_cluster(30, 8)]
    g = golden("caffeine")
    mols.append((np.array(g["Z"]), np.array(g["xyz_angstrom"])))
    return mols


def test_batch_tc_against_oracle_and_fp64(monkeypatch):
    mols = _mols()
    monkeypatch.setenv("GFNFF_BATCH_TC", "0")
    a = GFNFF(precision=MIXED)
    assert a.setMoleculeBatch(mols), a.getErrorMessage()
    monkeypatch.delenv("GFNFF_BATCH_TC")
    b = GFNFF(precision=MIXED)
    assert b.setMoleculeBatch(mols), b.getErrorMessage()
    ea, sa = a.calculateEnergyBatch()
    eb, sb = b.calculateEnergyBatch()
    assert (sa == 0).all() and (sb == 0).all(), (sa, sb)
    it = b.eeqIterations()
    assert 1 <= it <= 8, it   # refinement corrections of the slowest molecule
    assert np.abs(a.getCharges() - b.getCharges()).max() < Q_TOL
    Gb = b.getGradient()
    off = 0
    for m, (Z, X) in enumerate(mols):
        n = len(Z)
        T, Go, qo, cn = Oracle(Z, X).engrad(X)
        assert abs(eb[m] - T["total"]) <= E_TOL, (m, n, eb[m], T["total"])
        assert np.abs(Gb[off:off + n] - Go).max() <= G_TOL, (m, n)
        assert np.abs(b.getCharges()[off:off + n] - qo).max() < Q_TOL_ORACLE, (m, n)
        off += n


def test_batch_tc_repeated_and_charged():
    """Repeated evaluations reuse the scratch; a charged two-fragment molecule."""
    mols = _mols()[:6] + [_ammonium_water()]
    charges = [0] * 6 + [1]
    b = GFNFF(precision=MIXED)
    assert b.setMoleculeBatch(mols, charges), b.getErrorMessage()
    e1, s1 = b.calculateEnergyBatch()
    q1 = b.getCharges().copy()
    e2, s2 = b.calculateEnergyBatch()
    assert (s1 == 0).all() and (s2 == 0).all()
    assert np.abs(e1 - e2).max() < 1e-12
    assert np.abs(q1 - b.getCharges()).max() < 1e-12
    Z, X = mols[-1]
    T, Go, qo, cn = Oracle(Z, X, 1).engrad(X)
    assert abs(e1[-1] - T["total"]) <= E_TOL
    assert abs(b.getCharges()[-len(Z):].sum() - 1.0) < 1e-9


def test_single_molecule_tc_solver(monkeypatch):
    """A single molecule of the mixed form through the batched solver (the path a 194-atom
    alkane takes when the autotuner picks it)."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", "batched")
    Z, X = workloads.alkane(64, 1001)
    g = GFNFF(precision=MIXED)
    assert g.setMolecule(Z, X), g.getErrorMessage()
    assert g.eeqSolver() == "batched"
    e = g.calculateEnergy(True)
    assert not g.hasError(), g.getErrorMessage()
    T, Go, qo, cn = Oracle(Z, X).engrad(X)
    assert abs(e - T["total"]) <= E_TOL
    assert np.abs(g.getGradient() - Go).max() <= G_TOL
    assert np.abs(g.getCharges() - qo).max() < Q_TOL_ORACLE
