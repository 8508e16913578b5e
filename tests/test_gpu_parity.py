"""GPU (FP64 form) against the CPU oracle on the same inputs, through the C ABI.

Bar (north-star plain form): energy within 1e-8 Eh, gradient within 1e-7 Eh/bohr
(max-abs), topology lists bit-exact."""
import ctypes

import numpy as np
import pytest

from curcuma_b200 import GFNFF, workloads
from tests.oracle_api import Oracle, OracleSequence, golden, golden_names

E_TOL = 1e-8
G_TOL = 1e-7

pytestmark = pytest.mark.gpu


def _compare(Z, X, charge=0, e_tol=E_TOL, g_tol=G_TOL):
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X, charge), gpu.getErrorMessage()
    e = gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    o = Oracle(Z, X, charge)
    T, G, q, cn = o.engrad(X)
    terms = gpu.getEnergyDecomposition()
    for k, v in T.items():
        assert abs(terms[k] - v) < e_tol, f"{k}: gpu {terms[k]!r} oracle {v!r}"
    assert abs(e - T["total"]) < e_tol
    g = gpu.getGradient()
    assert np.abs(g - G).max() < g_tol, np.abs(g - G).max()
    assert np.abs(gpu.getCharges() - q).max() < 1e-9
    assert np.abs(gpu.getCoordinationNumbers() - cn).max() < 1e-12
    return gpu, o


@pytest.mark.parametrize("name", golden_names())
def test_golden_molecules(name):
    g = golden(name)
    _compare(np.array(g["Z"]), np.array(g["xyz_angstrom"]))


@pytest.mark.parametrize("name", ["cli_complex", "cli_caffeine"])
def test_cli_molecules(name):
    g = golden(name)
    gpu, _ = _compare(np.array(g["Z"]), np.array(g["xyz_angstrom"]))
    assert abs(gpu.getEnergyDecomposition()["total"] - g["total_energy"]) < g["tolerance"]


def test_alkane_c64():
    Z, X = workloads.alkane(64, 1001)
    _compare(Z, X)


def test_water_cluster_small():
    Z, X = workloads.water_cluster(60, 77)
    gpu, o = _compare(Z, X)
    assert gpu.sizes() == (180, 60)


def test_conformers():
    for Z, X in workloads.conformer_batch(6, 1004):
        _compare(Z, X)


def test_peptide_small():
    Z, X = workloads.solvated_peptide(6, 40, 55)
    _compare(Z, X)


def test_topology_bit_exact():
    Z, X = workloads.water_cluster(40, 5)
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X)
    o = Oracle(Z, X)
    # dispersion pairs are enumerated on the device from the setup geometry
    assert np.array_equal(gpu.topology(4, 2), o.topology(4, 2))
    for kind, width in [(0, 2), (1, 3), (2, 4), (3, 4), (5, 2), (6, 4), (8, 1), (9, 1), (11, 2), (12, 3), (13, 3)]:
        assert np.array_equal(gpu.topology(kind, width), o.topology(kind, width)), kind


def test_hb_refresh_matches_oracle():
    Z, X = workloads.water_cluster(30, 9)
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X)
    X2 = X.copy()
    # translate 20 of the 30 waters by 3 bohr per axis: sqrt(sum d^2)/N = 0.45 > 0.3 bohr; the
    # atoms moved more than 0.5 bohr along an axis, so the topology is recomputed first (as in
    # curcuma's evaluation), then the HB/XB lists
    X2[: 3 * 20] += 3.0 * 0.529177210903
    gpu.updateGeometry(X2)
    e = gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    o = Oracle(Z, X)
    o.refresh_topology(X2)
    o.redetect_hbxb(X2)
    T, G, q, cn = o.engrad(X2)
    assert abs(e - T["total"]) < E_TOL
    assert np.abs(gpu.getGradient() - G).max() < G_TOL


def test_device_entry_point_matches_host():
    import torch
    Z, X = workloads.alkane(12, 3)
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X)
    e_host = gpu.calculateEnergy(True)
    g_host = gpu.getGradient()
    lib = gpu._lib
    xb = torch.tensor(X / 0.529177210903, dtype=torch.float64, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros(len(Z) * 3, dtype=torch.float64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.gfnff_energy_and_gradient_device(gpu.handle, ctypes.c_void_p(xb.data_ptr()), ctypes.c_void_p(e.data_ptr()),
                                             ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(st.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert abs(e.item() - e_host) < 1e-12
    assert np.abs(g.cpu().numpy().reshape(-1, 3) - g_host).max() < 1e-12


def test_error_paths():
    gpu = GFNFF()
    Z = np.array([8, 1, 1])
    X = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 0.9, 0.0]])
    assert not gpu.setMolecule(Z, X)           # coincident atoms -> setup failure
    assert gpu.hasError()
    X = np.array([[0.0, 0.0, 0.0], [0.96, 0.0, 0.0], [-0.24, 0.93, 0.0]])
    assert gpu.setMolecule(Z, X)
    Xn = X.copy()
    Xn[1, 0] = np.nan
    gpu.updateGeometry(Xn)
    assert gpu.calculateEnergy(True) == 0.0 and gpu.hasError()
    gpu.updateGeometry(X)
    assert gpu.calculateEnergy(True) != 0.0 and not gpu.hasError()


@pytest.mark.parametrize("solver", ["tiled", "library", "pcg", "pcg-lower", "pcg-classic", "pcg-resident",
                                    "batched"])
@pytest.mark.parametrize("system", ["water64", "water200", "alkane", "peptide"])
def test_eeq_solvers(solver, system, monkeypatch):
    """Every EEQ solver of the reduced system against the oracle; the 64-water cluster
    has 128 reduced unknowns, so the tiled Cholesky's right-hand-side row forms a tile of
    its own, and the alkane (one fragment) exercises the PCG with 64-row blocks.
    pcg-lower forces the PCG form of large systems (lower triangle only, M p by tiles),
    pcg-classic the two-barrier CG iteration instead of the pipelined one, pcg-resident the
    pipelined iteration over shared-memory resident tiles built from the atoms;
    batched is the per-molecule shared-memory solver, offered for molecules of at most
    320 atoms."""
    monkeypatch.setenv("GFNFF_PCG_SYM", "1" if solver == "pcg-lower" else "0")
    monkeypatch.setenv("GFNFF_PCG", "classic" if solver == "pcg-classic" else "pipelined")
    monkeypatch.setenv("GFNFF_PCG_RES", "1" if solver == "pcg-resident" else "0")
    solver = "pcg" if solver in ("pcg-lower", "pcg-classic", "pcg-resident") else solver
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", solver)
    Z, X = {"water64": lambda: workloads.water_cluster(64, 9),
            "water200": lambda: workloads.water_cluster(200, 10),
            "alkane": lambda: workloads.alkane(64, 1001),
            "peptide": lambda: workloads.solvated_peptide(8, 60, 12)}[system]()
    if solver == "batched" and len(Z) > 320:
        pytest.skip("the batched solver stages at most 320 atoms")
    gpu, _ = _compare(Z, X)
    assert gpu.eeqSolver() == solver


@pytest.mark.parametrize("system", ["water200", "alkane"])
def test_graph_replay_matches_direct_launches(system, monkeypatch):
    """The step replayed as a captured CUDA graph gives the same results as direct
    launches (GFNFF_GRAPHS=0), over several geometries."""
    Z, X = {"water200": lambda: workloads.water_cluster(200, 10),
            "alkane": lambda: workloads.alkane(64, 1001)}[system]()
    res = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("GFNFF_GRAPHS", flag)
        g = GFNFF()
        assert g.setMolecule(Z, X)
        out = []
        for k in range(3):
            g.updateGeometry(X + 0.002 * k)
            e = g.calculateEnergy(True)
            assert not g.hasError(), g.getErrorMessage()
            out.append((e, g.getGradient()))
        res[flag] = out
    for (e1, g1), (e0, g0) in zip(res["1"], res["0"]):
        assert abs(e1 - e0) < 1e-10
        assert np.abs(g1 - g0).max() < 1e-10


@pytest.mark.parametrize("system", ["water200", "alkane"])
def test_pcg_warm_start(system, monkeypatch):
    """PCG started from the previous geometry's solution reaches the same charges and
    energies as the oracle on every geometry of a short sequence, in fewer iterations than
    a start from zero."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", "pcg")
    monkeypatch.setenv("GFNFF_PCG_SYM", "1" if system == "water200" else "0")
    Z, X = {"water200": lambda: workloads.water_cluster(200, 10),
            "alkane": lambda: workloads.alkane(64, 1001)}[system]()
    rng = np.random.default_rng(5)
    geoms = [X + rng.normal(scale=0.01, size=X.shape) for _ in range(4)]
    iters = {}
    o = Oracle(Z, X)
    for flag in ("1", "0"):
        monkeypatch.setenv("GFNFF_PCG_WARM", flag)
        g = GFNFF()
        assert g.setMolecule(Z, X)
        iters[flag] = []
        for Xk in geoms:
            g.updateGeometry(Xk)
            e = g.calculateEnergy(True)
            assert not g.hasError(), g.getErrorMessage()
            iters[flag].append(g.eeqIterations())
            if flag == "1":
                T, G, q, _ = o.engrad(Xk)
                assert abs(e - T["total"]) < E_TOL
                assert np.abs(g.getGradient() - G).max() < G_TOL
                assert np.abs(g.getCharges() - q).max() < 1e-9
    assert sum(iters["1"][1:]) < sum(iters["0"][1:]), iters


def test_cn_neighbour_list_refresh():
    """CN and its chain rule run over a neighbour list with a 1-bohr skin.  Geometries that
    move atoms more than half the skin make the list stale: that evaluation falls back to the
    all-pairs kernels and the host rebuilds the list around it.  Every geometry of the
    sequence matches the oracle either way."""
    Z, X = workloads.water_cluster(64, 9)
    rng = np.random.default_rng(3)
    geoms = [X + rng.normal(scale=s, size=X.shape) for s in (0.02, 0.15, 0.15, 0.02)]
    o = OracleSequence(Z, X)   # the larger steps also refresh the topology and the HB lists
    g = GFNFF()
    assert g.setMolecule(Z, X)
    for Xk in geoms:
        g.updateGeometry(Xk)
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        T, G, q, cn = o.engrad(Xk)
        assert abs(e - T["total"]) < E_TOL
        assert np.abs(g.getGradient() - G).max() < G_TOL
        assert np.abs(g.getCoordinationNumbers() - cn).max() < 1e-12


@pytest.mark.parametrize("pcg_form", ["classic", "pipelined"])
def test_side_stream_gradients_repeat(pcg_form, monkeypatch):
    """The charge-independent terms run on a second stream beside the pair kernels, and both
    add into the same gradient entries.  Every one of many evaluations at one geometry must
    reproduce the oracle's gradient: an update lost between the streams shows up as a few
    atoms off by 1e-5..1e-2 Eh/bohr in some evaluations.  The classic PCG fills every SM, so
    the side kernels run after it, at the same time as the pair kernels."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", "pcg")
    monkeypatch.setenv("GFNFF_PCG", pcg_form)
    Z, X = workloads.water_cluster(200, 10)
    T, G, _, _ = Oracle(Z, X).engrad(X)
    g = GFNFF()
    assert g.setMolecule(Z, X)
    worst = 0.0
    for _ in range(25):
        e = g.calculateEnergy(True)
        assert not g.hasError(), g.getErrorMessage()
        assert abs(e - T["total"]) < E_TOL
        worst = max(worst, np.abs(g.getGradient() - G).max())
    assert worst < G_TOL, worst


def test_kernels_per_evaluation(monkeypatch):
    """The library counts its own kernels in the captured step graph (cuSOLVER's are not
    counted); direct launches report -1."""
    Z, X = workloads.water_cluster(64, 9)
    counts = {}
    for solver in ("pcg", "library"):
        monkeypatch.setenv("GFNFF_EEQ_SOLVER", solver)
        g = GFNFF()
        assert g.setMolecule(Z, X)
        g.calculateEnergy(True)
        k1 = g.kernelsPerEvaluation()
        g.calculateEnergy(True)
        assert g.kernelsPerEvaluation() == k1
        counts[solver] = k1
    assert 12 <= counts["library"] < counts["pcg"] <= 40, counts
    monkeypatch.setenv("GFNFF_GRAPHS", "0")
    g = GFNFF()
    assert g.setMolecule(Z, X)
    g.calculateEnergy(True)
    assert g.kernelsPerEvaluation() == -1


def test_setup_from_parameter_file(tmp_path, monkeypatch):
    """A handle set up from a parameter file evaluates like one set up from the structure (the
    same model; only the order of the FP64 atomic sums differs between any two runs), and
    refuses a file made for another structure."""
    monkeypatch.setenv("GFNFF_EEQ_SOLVER", "library")   # no timing-dependent solver choice
    Z, X = workloads.water_cluster(64, 9)
    a = GFNFF()
    assert a.setMolecule(Z, X)
    path = tmp_path / "water64.param.bin"
    assert a.saveParameters(path), a.getErrorMessage()
    b = GFNFF()
    assert b.setMoleculeFromParameters(path, Z, X), b.getErrorMessage()
    Xk = X + np.random.default_rng(2).normal(scale=0.01, size=X.shape)
    for g in (a, b):
        g.updateGeometry(Xk)
    ea, eb = a.calculateEnergy(True), b.calculateEnergy(True)
    assert abs(ea - eb) < 1e-11 and np.abs(a.getGradient() - b.getGradient()).max() < 1e-12
    c = GFNFF()
    Zo = Z.copy()
    Zo[0] = 7
    assert not c.setMoleculeFromParameters(path, Zo, X)
    assert "another structure" in c.getErrorMessage()


def test_computational_method_interface():
    """The rest of curcuma's ComputationalMethod interface on the Python mirror."""
    g = golden("H2O")
    Z, X = np.array(g["Z"]), np.array(g["xyz_angstrom"], dtype=float)
    m = GFNFF(exact_gradient=True)
    assert m.setMolecule(Z, X)
    e = m.calculateEnergy(True)
    assert m.getMethodName() == "gfnff" and m.hasGradient() and not m.isThreadSafe()
    buf = np.empty((len(Z), 3))
    m.copyGradientTo(buf)
    assert np.array_equal(buf, m.getGradient())
    assert np.array_equal(m.getCN(), m.getCoordinationNumbers())
    assert m.getBondOrders().shape == (3,) and not m.getBondOrders().any()
    assert not m.getDipole().any()
    assert m.getHBCount() >= 0 and m.getXBCount() == 0
    # exact mode: the analytic gradient is the derivative of the energy
    G = m.getGradient()
    assert np.abs(m.NumGrad(1e-4) - G).max() < 1e-6
    assert np.abs(m.getGradient() - G).max() < 1e-12     # results of the restored geometry
    assert m.calculateEnergy(True) == pytest.approx(e, abs=1e-12)
    m.setThreadCount(4)
    assert m.getParameters()["threads"] == 4
    m.setParameters({"precision": "mixed", "exact_gradient": False})
    assert m.getParameters()["precision"] == "mixed"
    assert m.setMolecule(Z, X)
    assert abs(m.calculateEnergy(True) - e) < 1e-6
    assert not m.updateGeometry(X[:2]) and m.hasError()
    m.clearError()
    assert not m.hasError()
    with pytest.raises(KeyError):
        m.setParameters({"no_such_key": 1})
