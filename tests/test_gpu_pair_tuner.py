"""The set-up autotuner of the Coulomb + D4 pair kernel: every variant it chooses from gives
the same energy and gradient (each pair's arithmetic is the same; only the summation order
differs), and the pick is one of them.  Single molecule (1000 waters) and a conformer batch,
both precision forms."""
import numpy as np
import pytest

from curcuma_b200 import FP64, GFNFF, MIXED, workloads

pytestmark = pytest.mark.gpu

VARIANTS = ["sym32", "sym64", "sym64_occ10", "rows"]


def _run(mols, precision, monkeypatch, variant=None):
    if variant:
        monkeypatch.setenv("GFNFF_PAIRS_VARIANT", variant)
    else:
        monkeypatch.delenv("GFNFF_PAIRS_VARIANT", raising=False)
    g = GFNFF(precision=precision)
    if len(mols) == 1:
        assert g.setMolecule(*mols[0]), g.getErrorMessage()
        e = np.array([g.calculateEnergy(True)])
    else:
        assert g.setMoleculeBatch(mols), g.getErrorMessage()
        e, st = g.calculateEnergyBatch()
        assert (st == 0).all()
    assert not g.hasError(), g.getErrorMessage()
    return g.pairKernel(), e, g.getGradient()


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("system", ["water1000", "batch24"])
def test_variants_agree_and_tuner_picks_one(system, precision, monkeypatch):
    mols = ([workloads.water_cluster(1000, 1002)] if system == "water1000"
            else workloads.conformer_batch(24, 17, lo=20, hi=200))
    pick, e0, g0 = _run(mols, precision, monkeypatch)
    assert pick in VARIANTS
    for v in VARIANTS:
        name, e, g = _run(mols, precision, monkeypatch, v)
        assert name == v
        assert np.abs(e - e0).max() < 1e-9, (v, e - e0)
        assert np.abs(g - g0).max() < 1e-9, v
