"""Parity on the benchmark configurations at full size: the FP64 form against the CPU oracle
at |dE| <= 1e-8 Eh and max |dF| <= 1e-7 Eh/bohr, the mixed form at 1e-6 Eh / 1e-5 Eh/bohr, at
each workload's own geometry.

* 1000-water cluster (3000 atoms, 1000 fragments)
* Gly50 + 1500 waters (4853 atoms)
* 6000 waters + 40 C20H42 (20,480 atoms, 6040 fragments; the oracle's dense 20,480 x 20,480
  Schur-complement solve takes about a minute on the host)
* the 512-conformer batch (20-300 atoms each), every molecule against its own oracle run.
"""
import numpy as np
import pytest

from curcuma_b200 import FP64, GFNFF, MIXED, workloads
from tests.oracle_api import Oracle

pytestmark = pytest.mark.gpu

TOL = {FP64: (1e-8, 1e-7), MIXED: (1e-6, 1e-5)}
SINGLE = {
    "water1000": lambda: workloads.water_cluster(1000, 1002),
    "gly50_water1500": lambda: workloads.solvated_peptide(50, 1500, 1003),
    "cluster20k": lambda: workloads.large_cluster(6000, 40, 20, 1005),
}
_cache = {}


def _oracle(name):
    if name not in _cache:
        Z, X = SINGLE[name]()
        T, G, q, cn = Oracle(Z, X).engrad(X)
        _cache[name] = (Z, X, T["total"], G)
    return _cache[name]


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", list(SINGLE))
def test_single_structure_against_oracle(name, precision):
    Z, X, E, G = _oracle(name)
    gpu = GFNFF(precision=precision)
    assert gpu.setMolecule(Z, X), gpu.getErrorMessage()
    e = gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    te, tg = TOL[precision]
    assert abs(e - E) <= te, (name, e, E, e - E)
    dg = float(np.abs(gpu.getGradient() - G).max())
    assert dg <= tg, (name, dg)


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_conformer_batch_512_against_oracle(precision):
    mols = workloads.conformer_batch(512, 1004)
    gpu = GFNFF(precision=precision)
    assert gpu.setMoleculeBatch(mols), gpu.getErrorMessage()
    e, st = gpu.calculateEnergyBatch()
    assert (st == 0).all(), np.nonzero(st)[0][:10]
    G = gpu.getGradient()
    te, tg = TOL[precision]
    off, de, dg = 0, 0.0, 0.0
    for m, (Z, X) in enumerate(mols):
        if "batch512" not in _cache:
            _cache["batch512"] = [None] * len(mols)
        if _cache["batch512"][m] is None:
            T, Go, q, cn = Oracle(Z, X).engrad(X)
            _cache["batch512"][m] = (T["total"], Go)
        Eo, Go = _cache["batch512"][m]
        n = len(Z)
        de = max(de, abs(e[m] - Eo))
        dg = max(dg, float(np.abs(G[off:off + n] - Go).max()))
        off += n
    assert de <= te and dg <= tg, (de, dg)
