"""The topology cache (`<geometry>.topo.json`, curcuma's format) through the GPU handle:
gfnff_set_geometry_file before gfnff_setup reads the cache on a fingerprint match and writes
it after the set-up (curcuma: ff_methods/gfnff_method.cpp:2941-2985, 8973-9040)."""
import json

import numpy as np
import pytest

from curcuma_b200 import GFNFF, MIXED, workloads
from tests.oracle_api import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, MIXED], ids=["fp64", "mixed"])
def test_handle_writes_then_hits(tmp_path, precision):
    Z, X = workloads.solvated_peptide(6, 40, 11)
    geom = tmp_path / "pep.xyz"
    topo = tmp_path / "pep.topo.json"
    g1 = GFNFF(precision=precision, geometry_file=geom)
    assert g1.setMolecule(Z, X), g1.getErrorMessage()
    assert topo.exists() and not g1.topologyCacheHit()
    e1 = g1.calculateEnergy(True)
    G1 = g1.getGradient()
    g2 = GFNFF(precision=precision, geometry_file=geom)
    assert g2.setMolecule(Z, X)
    assert g2.topologyCacheHit()
    e2 = g2.calculateEnergy(True)
    assert abs(e2 - e1) < 1e-10
    assert np.abs(g2.getGradient() - G1).max() < 1e-10
    T, G, q, cn = Oracle(Z, X).engrad(X)
    tol = 1e-8 if precision == 0 else 1e-6
    assert abs(e2 - T["total"]) < tol


def test_planted_cache_matches_the_oracle(tmp_path):
    Z, X = workloads.solvated_peptide(4, 20, 12)
    geom = tmp_path / "p.xyz"
    topo = tmp_path / "p.topo.json"
    g = GFNFF(geometry_file=geom)
    assert g.setMolecule(Z, X)
    d = json.loads(topo.read_text())
    d["dxi"] = [v + 0.01 * ((i % 3) - 1) for i, v in enumerate(d["dxi"])]
    d["dgam"][3] -= 0.02
    topo.write_text(json.dumps(d))
    g = GFNFF(geometry_file=geom)
    assert g.setMolecule(Z, X) and g.topologyCacheHit()
    e = g.calculateEnergy(True)
    o = Oracle(Z, X, topo_cache=topo)
    assert o.cache_hit
    T, G, q, cn = o.engrad(X)
    assert abs(e - T["total"]) < 1e-8
    assert np.abs(g.getGradient() - G).max() < 1e-7
    assert np.abs(g.getCharges() - q).max() < 1e-9
    T0 = Oracle(Z, X).engrad(X)[0]
    assert abs(T0["total"] - T["total"]) > 1e-6


def test_cache_off(tmp_path):
    Z, X = workloads.alkane(8, 5)
    g = GFNFF(geometry_file=tmp_path / "a.xyz", cache_topology=False)
    assert g.setMolecule(Z, X)
    assert not (tmp_path / "a.topo.json").exists()
    assert not g.topologyCacheHit()
