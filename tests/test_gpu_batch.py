"""Batched evaluation of independent molecules (gfnff_setup_batch /
gfnff_energy_and_gradient_batch) against the same molecules evaluated one at a time
and against the CPU oracle."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, MIXED, workloads
from tests.oracle_api import Oracle, golden

pytestmark = pytest.mark.gpu


def _mols():
    mols = workloads.conformer_batch(12, 77, lo=20, hi=120)
    g = golden("caffeine")
    mols.append((np.array(g["Z"]), np.array(g["xyz_angstrom"])))
    mols.append(workloads.water_cluster(20, 4))
    return mols


def test_batch_matches_single_and_oracle():
    mols = _mols()
    b = GFNFF()
    assert b.setMoleculeBatch(mols), b.getErrorMessage()
    e, st = b.calculateEnergyBatch()
    assert not b.hasError(), b.getErrorMessage()
    assert (st == 0).all()
    G = b.getGradient()
    q = b.getCharges()
    off = 0
    for m, (Z, X) in enumerate(mols):
        n = len(Z)
        s = GFNFF()
        assert s.setMolecule(Z, X)
        es = s.calculateEnergy(True)
        assert abs(e[m] - es) < 1e-10, (m, e[m], es)
        assert np.abs(G[off:off + n] - s.getGradient()).max() < 1e-10
        assert np.abs(q[off:off + n] - s.getCharges()).max() < 1e-10
        if m % 4 == 0:
            T, Go, qo, cn = Oracle(Z, X).engrad(X)
            assert abs(e[m] - T["total"]) < 1e-8
            assert np.abs(G[off:off + n] - Go).max() < 1e-7
        off += n


def test_batch_mixed_and_repeated_calls():
    mols = _mols()
    a, b = GFNFF(), GFNFF(precision=MIXED)
    assert a.setMoleculeBatch(mols) and b.setMoleculeBatch(mols)
    ea, _ = a.calculateEnergyBatch()
    for _ in range(2):
        eb, st = b.calculateEnergyBatch()
        assert (st == 0).all()
        assert np.abs(ea - eb).max() < 1e-6
        assert np.abs(a.getGradient() - b.getGradient()).max() < 1e-5


def test_batch_rejects_single_calls():
    b = GFNFF()
    assert b.setMoleculeBatch(_mols()[:3])
    b.calculateEnergy(True)
    assert b.hasError()
