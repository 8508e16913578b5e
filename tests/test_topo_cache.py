"""The topology cache in curcuma's `<geometry>.topo.json` format (curcuma_b200/csrc/setup/
topo_cache.cpp; curcuma: ff_methods/gfnff_method.cpp:2515-2656 fingerprint and export,
2941-2985 the write after the set-up with its charge check, 8973-9040 the read before
Phase 1).  Host side only: the set-up with the cache through the product library's
host entry (gfnff_write_topology_cache) and through the oracle's set-up, which shares the
set-up sources.

* the file: curcuma's keys and types, fragments numbered from 1, charges summing to the
  molecular charge, a decimal fingerprint;
* a second set-up hits and reproduces the fresh model exactly (energies bit for bit);
* the Phase-1 data really come from the file: a planted dxi / dgam / alpeeq / qfrag change
  changes the energy the way the same change of the model does, and survives the rewrite;
* misses: another bond list (fingerprint), a foreign fingerprint, a missing Phase-1 key,
  wrong lengths, unparsable text;
* the write check refuses unphysical Phase-1 charges."""
import json

import numpy as np
import pytest

from curcuma_b200 import workloads, write_topology_cache
from tests.oracle_api import Oracle

FIX = json.loads(__import__("pathlib").Path(__file__).with_name("golden").joinpath(
    "alpb", "gfnff_alpb_xtb.json").read_text())


def _mol(name):
    rec = FIX["molecules"][name]
    return np.array(rec["Z"]), np.array(rec["xyz_angstrom"])


def _geom(tmp_path, name="mol.xyz"):
    return tmp_path / name, tmp_path / (name.rsplit(".", 1)[0] + ".topo.json")


def _energy(o, X):
    T, G, q, cn = o.engrad(X)
    return T["total"], G, q


@pytest.mark.parametrize("name", ["caffeine", "acetic_acid_dimer"])
def test_written_file_layout(tmp_path, name):
    Z, X = _mol(name)
    geom, topo = _geom(tmp_path)
    assert write_topology_cache(Z, X, geom) is False
    d = json.loads(topo.read_text())
    n = len(Z)
    for k in ("version", "nfrag", "fraglist", "qfrag", "topology_charges", "coordination_numbers",
              "hybridization", "ring_sizes", "pi_fragments", "is_aromatic", "is_metal", "rings",
              "is_amide_h", "dxi", "alpeeq", "dgam", "timestamp", "fingerprint"):
        assert k in d, k
    assert d["version"] == 1
    assert isinstance(d["fingerprint"], str) and d["fingerprint"].isdigit()
    for k in ("fraglist", "topology_charges", "coordination_numbers", "hybridization", "ring_sizes",
              "pi_fragments", "is_aromatic", "is_metal", "is_amide_h", "dxi", "alpeeq", "dgam"):
        assert len(d[k]) == n, k
    assert min(d["fraglist"]) == 1 and max(d["fraglist"]) == d["nfrag"] == len(d["qfrag"])
    assert abs(sum(d["topology_charges"])) < 1e-8
    assert all(isinstance(r, list) for r in d["rings"])
    if name == "caffeine":
        assert sorted(len(r) for r in d["rings"]) == [5, 6]
    if name == "acetic_acid_dimer":
        assert d["nfrag"] == 2


def test_hit_reproduces_the_fresh_set_up(tmp_path):
    Z, X = _mol("caffeine")
    geom, topo = _geom(tmp_path)
    assert not write_topology_cache(Z, X, geom)
    first = json.loads(topo.read_text())
    assert write_topology_cache(Z, X, geom)          # the second set-up reads the file
    second = json.loads(topo.read_text())
    for k in ("topology_charges", "dxi", "dgam", "alpeeq", "qfrag", "is_amide_h", "fingerprint"):
        assert first[k] == second[k], k
    fresh = Oracle(Z, X)
    cached = Oracle(Z, X, topo_cache=topo)
    assert cached.cache_hit and not fresh.cache_hit
    X2 = X + np.random.default_rng(3).normal(scale=0.02, size=X.shape)
    for geo in (X, X2):
        e0, g0, q0 = _energy(fresh, geo)
        e1, g1, q1 = _energy(cached, geo)
        assert e0 == e1
        assert np.array_equal(g0, g1) and np.array_equal(q0, q1)


@pytest.mark.parametrize("key", ["dxi", "dgam", "alpeeq"])
def test_planted_phase1_data_are_used(tmp_path, key):
    Z, X = _mol("caffeine")
    geom, topo = _geom(tmp_path)
    write_topology_cache(Z, X, geom)
    d = json.loads(topo.read_text())
    d[key][0] += 0.05
    topo.write_text(json.dumps(d))
    fresh, cached = Oracle(Z, X), Oracle(Z, X, topo_cache=topo)
    assert cached.cache_hit
    e0 = _energy(fresh, X)[0]
    e1, _, q1 = _energy(cached, X)
    assert abs(e1 - e0) > 1e-7
    assert abs(q1.sum()) < 1e-10
    # the hit carries the planted value into the rewritten file
    assert write_topology_cache(Z, X, geom)
    assert json.loads(topo.read_text())[key][0] == d[key][0]


def test_planted_fragment_charges_of_a_charged_dimer(tmp_path):
    """Ammonium + water: the set-up places the charge on one fragment; a cache that places
    it on the other is followed (curcuma restores qfrag on a hit)."""
    t = 1.03 / np.sqrt(3.0)
    a = np.deg2rad(104.52 / 2)
    X = np.array([[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t], [3.5, 0, 0],
                  [3.5 + 0.9572 * np.cos(a), 0.9572 * np.sin(a), 0],
                  [3.5 + 0.9572 * np.cos(a), -0.9572 * np.sin(a), 0]])
    Z = np.array([7, 1, 1, 1, 1, 8, 1, 1])
    geom, topo = _geom(tmp_path)
    write_topology_cache(Z, X, geom, charge=1)
    d = json.loads(topo.read_text())
    assert d["nfrag"] == 2 and sorted(d["qfrag"]) == [0.0, 1.0]
    _, _, q_fresh = _energy(Oracle(Z, X, charge=1), X)
    cached = Oracle(Z, X, charge=1, topo_cache=topo)
    assert cached.cache_hit
    _, _, q_cached = _energy(cached, X)
    assert np.array_equal(q_fresh, q_cached)
    d["qfrag"] = d["qfrag"][::-1]
    topo.write_text(json.dumps(d))
    swapped = Oracle(Z, X, charge=1, topo_cache=topo)
    assert swapped.cache_hit
    _, _, q_sw = _energy(swapped, X)
    f = np.array(d["fraglist"]) - 1
    for k in range(2):
        assert abs(q_sw[f == k].sum() - d["qfrag"][k]) < 1e-9


def test_misses(tmp_path):
    Z, X = _mol("caffeine")
    geom, topo = _geom(tmp_path)
    write_topology_cache(Z, X, geom)
    good = topo.read_text()
    d = json.loads(good)
    # another bond list: an H atom pulled off changes the fingerprint
    Xf = X.copy()
    h = int(np.where(Z == 1)[0][0])
    Xf[h] += 4.0
    assert not Oracle(Z, Xf, topo_cache=topo).cache_hit
    cases = {
        "foreign fingerprint": dict(d, fingerprint="12345"),
        "no dgam": {k: v for k, v in d.items() if k != "dgam"},
        "short dxi": dict(d, dxi=d["dxi"][:-1]),
        "qfrag of another fragment count": dict(d, qfrag=[0.0, 0.0]),
        "non-numeric charges": dict(d, topology_charges=["x"] * len(Z)),
    }
    for why, bad in cases.items():
        topo.write_text(json.dumps(bad))
        assert not Oracle(Z, X, topo_cache=topo).cache_hit, why
    topo.write_text(good[: len(good) // 2])
    assert not Oracle(Z, X, topo_cache=topo).cache_hit
    topo.write_text(good)
    assert Oracle(Z, X, topo_cache=topo).cache_hit
    assert not Oracle(Z, X, topo_cache=tmp_path / "absent.topo.json").cache_hit


def test_write_check_refuses_unphysical_charges(tmp_path):
    Z, X = _mol("caffeine")
    geom, topo = _geom(tmp_path)
    write_topology_cache(Z, X, geom)
    d = json.loads(topo.read_text())
    d["topology_charges"] = [q + 0.1 for q in d["topology_charges"]]   # sums to 2.4 e
    planted = json.dumps(d)
    topo.write_text(planted)
    with pytest.raises(RuntimeError, match="write check"):
        write_topology_cache(Z, X, geom)
    assert topo.read_text() == planted


def test_cache_path_follows_the_geometry_file(tmp_path):
    Z, X = _mol("H2O")
    write_topology_cache(Z, X, tmp_path / "water.coord.xyz")
    assert (tmp_path / "water.coord.topo.json").exists()
    write_topology_cache(Z, X, tmp_path / "noext")
    assert (tmp_path / "noext.topo.json").exists()


def test_larger_system_round_trip(tmp_path):
    Z, X = workloads.solvated_peptide(6, 30, 7)
    geom, topo = _geom(tmp_path, "pep.xyz")
    assert not write_topology_cache(Z, X, geom)
    assert write_topology_cache(Z, X, geom)
    d = json.loads(topo.read_text())
    assert d["nfrag"] == 31
    e0 = _energy(Oracle(Z, X), X)[0]
    e1 = _energy(Oracle(Z, X, topo_cache=topo), X)[0]
    assert e0 == e1
