"""Analytic gradient against central finite differences (h = 1e-4 bohr) and the device
velocity-Verlet loop against the same integrator driven from the host.

The default gradient reproduces curcuma's analytic gradient, which is not the exact
derivative of its energy (the D4 dC6/dCN term and the charges of Coulomb pairs cut at
100 bohr); the exact-gradient mode is, and it is what the finite differences check."""
import numpy as np
import pytest

from curcuma_b200 import GFNFF, atomic_masses, maxwell_boltzmann, workloads

pytestmark = pytest.mark.gpu

BOHR = 0.529177210903


@pytest.mark.parametrize("system", ["peptide", "water", "alkane", "alkane64"])
def test_exact_gradient_matches_central_differences(system):
    """The exact-gradient mode is the derivative of the energy; C64H130 spans more than
    100 bohr, so it exercises the EEQ charge response of the cut Coulomb pairs."""
    Z, X = {"peptide": lambda: workloads.solvated_peptide(6, 30, 21),
            "water": lambda: workloads.water_cluster(50, 8),
            "alkane": lambda: workloads.alkane(20, 5),
            "alkane64": lambda: workloads.alkane(64, 1001)}[system]()
    g = GFNFF(exact_gradient=True)
    assert g.setMolecule(Z, X)
    g.calculateEnergy(True)
    G = g.getGradient()
    rng = np.random.default_rng(64)
    atoms = rng.choice(len(Z), size=min(16, len(Z)), replace=False)
    h = 1e-4 * BOHR   # 1e-4 bohr in Angstrom
    worst = 0.0
    for a in atoms:
        for d in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[a, d] += h
            Xm[a, d] -= h
            g.updateGeometry(Xp)
            ep = g.calculateEnergy(True)
            g.updateGeometry(Xm)
            em = g.calculateEnergy(True)
            fd = (ep - em) / (2e-4)
            worst = max(worst, abs(fd - G[a, d]))
    assert worst < 1e-6, worst


def test_device_md_matches_host_driven_verlet():
    Z, X = workloads.water_cluster(20, 12)
    m = atomic_masses(Z)
    v0 = maxwell_boltzmann(m, 300.0, 5)
    dev = GFNFF()
    assert dev.setMolecule(Z, X)
    ep, ek = dev.runMD(10, 0.5, v0)
    assert not dev.hasError(), dev.getErrorMessage()
    # the same velocity Verlet from the host: bohr, atomic time units, electron masses
    host = GFNFF()
    assert host.setMolecule(Z, X)
    dt = 0.5 * 41.341373335
    me = m * 1822.888486209
    x = X / BOHR
    v = v0 / (BOHR * 41.341373335)
    host.updateGeometry(x * BOHR)
    e = host.calculateEnergy(True)
    g = host.getGradient()
    assert abs(e - ep[0]) < 1e-10
    for t in range(1, 11):
        v -= 0.5 * dt * g / me[:, None]
        x += dt * v
        host.updateGeometry(x * BOHR)
        e = host.calculateEnergy(True)
        g = host.getGradient()
        v -= 0.5 * dt * g / me[:, None]
        assert abs(e - ep[t]) < 1e-9, (t, e, ep[t])
        assert abs(0.5 * (me[:, None] * v * v).sum() - ek[t]) < 1e-9
    assert np.abs(dev.velocities() - v * BOHR * 41.341373335).max() < 1e-8


def _approaching_waters():
    """Two waters 8.6 A apart (O-O), out of each other's hydrogen-bond candidate range
    (about 8.4 A), the second moving at 0.02 A/fs towards the first: the HB list gains the
    dimer's four terms at the first refresh after the pair comes into range (step 64 at
    the default threshold, 43 at 0.1 bohr in the oracle's run of the same loop)."""
    w = workloads.water_geometry()
    X = np.vstack([w, w * np.array([-1.0, 1.0, 1.0]) + np.array([8.6, 0.0, 0.0])])
    Z = np.array([8, 1, 1, 8, 1, 1])
    V = np.zeros((6, 3))
    V[3:, 0] = -0.02
    V += np.random.default_rng(3).normal(scale=2e-3, size=V.shape)
    return Z, X, V


@pytest.mark.parametrize("thr,detect", [(0.3, "0"), (0.1, "0"), (0.1, "1")])
def test_hb_lists_refresh_at_the_same_steps_as_the_host_loop(thr, detect, monkeypatch):
    """The device loop re-detects the HB/XB lists at the first step whose
    sqrt(sum d^2)/N exceeds the threshold (rolling back to that step), which is where the
    single-point path, called once per step from the host, re-detects them too; the MD
    handle detects the HB terms on the host or on the device."""
    Z, X, V0 = _approaching_waters()
    m = atomic_masses(Z)
    nsteps = 240
    host = GFNFF(hb_rmsd_bohr=thr)
    assert host.setMolecule(Z, X)
    dt = 0.5 * 41.341373335
    me = m * 1822.888486209
    x = X / BOHR
    v = V0 / (BOHR * 41.341373335)
    ep_h = np.zeros(nsteps + 1)
    counts = []
    host.updateGeometry(x * BOHR)
    ep_h[0] = host.calculateEnergy(True)
    g = host.getGradient()
    counts.append(host.getHBCount())
    for t in range(1, nsteps + 1):
        v -= 0.5 * dt * g / me[:, None]
        x += dt * v
        host.updateGeometry(x * BOHR)
        ep_h[t] = host.calculateEnergy(True)
        g = host.getGradient()
        v -= 0.5 * dt * g / me[:, None]
        counts.append(host.getHBCount())
    changes = [t for t in range(1, len(counts)) if counts[t] != counts[t - 1]]
    assert changes and changes[0] % 100 != 0, counts   # the list changes inside a chunk
    monkeypatch.setenv("GFNFF_HB_DEVICE", detect)   # the MD handle's HB terms: host or device
    dev = GFNFF(hb_rmsd_bohr=thr)
    assert dev.setMolecule(Z, X)
    ep, ek = dev.runMD(nsteps, 0.5, V0)
    assert not dev.hasError(), dev.getErrorMessage()
    assert dev.getHBCount() == counts[-1]
    assert np.abs(ep - ep_h).max() < 1e-8, np.abs(ep - ep_h).argmax()
    assert np.abs(dev.velocities() - v * BOHR * 41.341373335).max() < 1e-8


def test_reference_and_exact_energies_agree():
    Z, X = workloads.alkane(64, 1001)
    a, b = GFNFF(), GFNFF(exact_gradient=True)
    assert a.setMolecule(Z, X) and b.setMolecule(Z, X)
    assert abs(a.calculateEnergy(True) - b.calculateEnergy(True)) < 1e-10
    # the gradients differ by the two terms the reference adds or leaves out
    assert np.abs(a.getGradient() - b.getGradient()).max() > 1e-7


def test_nve_energy_conservation():
    Z, X = workloads.water_cluster(64, 3)
    g = GFNFF(exact_gradient=True)
    assert g.setMolecule(Z, X)
    ep, ek = g.runMD(400, 0.5, maxwell_boltzmann(atomic_masses(Z), 300.0, 7))
    assert not g.hasError(), g.getErrorMessage()
    et = ep + ek
    assert np.abs(et - et[0]).max() < 1e-3
    slope = np.polyfit(np.arange(len(et)) * 0.5e-3, et, 1)[0]   # Eh per ps
    assert abs(slope) < 1e-3, slope
