"""Set-up lists built on the device (k_hbdetect.cuh) against the host builders.  Hydrogen-bond
terms detected on the device against the host detection of
the shared set-up (setup/parameters.cpp detect_hb_terms, the restatement of
gfnff_method.cpp:7936-8495): the same terms in the same order, so the energies and gradients of
the two modes are the same numbers.  The systems cover every case type: case 1 (a free H
between two acceptors), case 2 (water), case 3 (carbonyl and carboxyl O: the acetic-acid dimer,
caffeine, the peptide backbone), case 4 (two-coordinate N: the complex fixture), a single
water (no terms) and a refresh at a displaced geometry.  GFNFF_HB_DEVICE=1/0 forces the device or the host detection."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, workloads
from tests.oracle_api import Oracle, golden

pytestmark = pytest.mark.gpu


def _pair(monkeypatch, Z, X):
    out = []
    for mode in ("1", "0"):
        monkeypatch.setenv("GFNFF_HB_DEVICE", mode)
        g = GFNFF()
        assert g.setMolecule(Z, X), g.getErrorMessage()
        out.append(g)
    monkeypatch.delenv("GFNFF_HB_DEVICE")
    return out


def _systems():
    sy = {name: (np.array(golden(name)["Z"]), np.array(golden(name)["xyz_angstrom"]))
          for name in ("acetic_acid_dimer", "caffeine", "complex", "triose", "water")}
    sy["water200"] = workloads.water_cluster(200, 11)
    sy["peptide"] = workloads.solvated_peptide(8, 60, 12)
    return sy


@pytest.mark.parametrize("name", ["acetic_acid_dimer", "caffeine", "complex", "triose", "water", "water200",
                                  "peptide"])
def test_device_hb_lists_equal_host(name, monkeypatch):
    Z, X = _systems()[name]
    dev, host = _pair(monkeypatch, Z, X)
    Td, Th = dev.topology(6, 4), host.topology(6, 4)
    assert Td.shape == Th.shape and (Td == Th).all(), (Td.shape, Th.shape)
    if name in ("acetic_acid_dimer", "caffeine", "peptide"):
        assert (Th[:, 3] == 3).any()
    ed, eh = dev.calculateEnergy(True), host.calculateEnergy(True)
    assert not dev.hasError() and not host.hasError()
    assert abs(ed - eh) < 1e-13 * max(1.0, abs(eh))
    assert np.abs(dev.getGradient() - host.getGradient()).max() < 1e-11
    # a refresh at a displaced geometry (sqrt(sum d^2)/N > 0.3 bohr; atoms moved beyond 0.5 bohr
    # along an axis, so the topology is recomputed first: new fragments for most systems)
    X2 = X + np.random.default_rng(5).normal(scale=0.4, size=X.shape)
    assert dev.updateGeometry(X2) and host.updateGeometry(X2)
    ed, eh = dev.calculateEnergy(True), host.calculateEnergy(True)
    assert not dev.hasError() and not host.hasError(), (dev.getErrorMessage(), host.getErrorMessage())
    Td, Th = dev.topology(6, 4), host.topology(6, 4)
    assert Td.shape == Th.shape and (Td == Th).all()
    # a strained geometry (28 Eh): the iterative EEQ solve amplifies the order of the FP64
    # atomic sums, which differs from run to run
    assert abs(ed - eh) < 1e-10


def test_device_hb_case4_present(monkeypatch):
    """The complex fixture has two-coordinate N acceptors (case 4)."""
    Z, X = _systems()["complex"]
    dev, host = _pair(monkeypatch, Z, X)
    assert (host.topology(6, 4)[:, 3] == 4).any()
    assert (dev.topology(6, 4) == host.topology(6, 4)).all()


def test_device_hb_water1000(monkeypatch):
    """1000 waters: 1.19 million terms, detected on the device by default (N >= 512)."""
    Z, X = workloads.water_cluster(1000, 1002)
    g = GFNFF()
    assert g.setMolecule(Z, X)
    monkeypatch.setenv("GFNFF_HB_DEVICE", "0")
    h = GFNFF()
    assert h.setMolecule(Z, X)
    Td, Th = g.topology(6, 4), h.topology(6, 4)
    assert len(Th) > 1_000_000
    assert (Td == Th).all()
    assert abs(g.calculateEnergy(True) - h.calculateEnergy(True)) < 1e-10


def test_parameter_file_from_a_device_handle(tmp_path, monkeypatch):
    """A parameter file written from a device-detection handle holds the full host lists."""
    Z, X = _systems()["peptide"]
    monkeypatch.setenv("GFNFF_HB_DEVICE", "1")
    g = GFNFF()
    assert g.setMolecule(Z, X)
    e = g.calculateEnergy(True)
    path = tmp_path / "p.bin"
    assert g.saveParameters(path), g.getErrorMessage()
    monkeypatch.delenv("GFNFF_HB_DEVICE")
    r = GFNFF()
    assert r.setMoleculeFromParameters(path, Z, X), r.getErrorMessage()
    assert (r.topology(6, 4) == g.topology(6, 4)).all()
    assert abs(r.calculateEnergy(True) - e) < 1e-12


def test_cn_list_device_equals_host(monkeypatch):
    """The CN neighbour list built on the device (k_cnl_build) has the host builder's rows,
    so the CN sums are the same numbers, at set-up and after the refreshes that geometries
    moving atoms beyond half the skin trigger."""
    Z, X = workloads.water_cluster(300, 9)
    rng = np.random.default_rng(3)
    geoms = [X + rng.normal(scale=s, size=X.shape) for s in (0.02, 0.15, 0.15, 0.02)]
    hs = []
    for mode in ("host", None):
        if mode:
            monkeypatch.setenv("GFNFF_CN_LIST", mode)
        else:
            monkeypatch.delenv("GFNFF_CN_LIST")
        g = GFNFF()
        assert g.setMolecule(Z, X)
        hs.append(g)
    for Xk in geoms:
        cn = []
        for g in hs:
            g.updateGeometry(Xk)
            g.calculateEnergy(True)
            assert not g.hasError(), g.getErrorMessage()
            cn.append(g.getCoordinationNumbers())
        assert (cn[0] == cn[1]).all()


def test_topology_refresh_matches_oracle():
    """curcuma recomputes the topology when an atom has moved more than 0.5 bohr along an
    axis since the last one.  CH4 with one H pulled 1.5 A out: the C-H bond is gone from the
    new topology (two fragments, each neutral), the EEQ follows it, the force-field terms stay
    those of the set-up.  A small step afterwards (< 0.5 bohr) keeps the new topology."""
    Z = np.array([6, 1, 1, 1, 1])
    t = 1.09 / np.sqrt(3.0)
    X0 = np.array([[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t]])
    X1 = X0.copy()
    X1[1] *= (1.09 + 1.5) / 1.09
    X2 = X1 + np.random.default_rng(2).normal(scale=0.02, size=X1.shape)
    g = GFNFF()
    assert g.setMolecule(Z, X0)
    o = Oracle(Z, X0)
    e0 = g.calculateEnergy(True)
    assert abs(e0 - o.engrad(X0)[0]["total"]) < 1e-9
    for X, changes in ((X1, True), (X2, False)):
        assert o.refresh_topology(X) == changes
        o.redetect_hbxb(X)
        g.updateGeometry(X)
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        T, G, q, cn = o.engrad(X)
        assert abs(e - T["total"]) < 1e-9, (e, T["total"])
        assert np.abs(g.getGradient() - G).max() < 1e-8
        assert np.abs(g.getCharges() - q).max() < 1e-10
    assert abs(g.getCharges()[1]) < 1e-10   # the H alone is a neutral fragment
