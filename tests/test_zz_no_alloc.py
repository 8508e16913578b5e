"""The allocation-free EEQ entry point (gfnff_eeq_charges_noalloc) against the charges of
the regular energy + gradient entry point.

Callers that cannot allocate device memory (inside another framework's memory pool, or
loops that forbid allocations after start-up) use gfnff_eeq_charges_noalloc: they pass
their own input and output buffers and the solver keeps its intermediates in a fixed
file-scope device array.  This file is collected last on purpose so that a run stopping
at the first failure has already run every other test; it also passes alone in a fresh
process."""
import ctypes

import numpy as np
import pytest

from curcuma_b200 import GFNFF, workloads
from tests.oracle_api import Oracle, golden

pytestmark = pytest.mark.gpu

Q_TOL = 1e-9   # same charge tolerance as the GPU/oracle parity tests


def _inputs(Z, X, charge=0):
    """Per-atom EEQ inputs of the model (from the setup shared with the oracle) and the
    reference charges/CN of one gfnff_energy_and_gradient evaluation."""
    import torch
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X, charge), gpu.getErrorMessage()
    gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    q_ref = gpu.getCharges()
    cn = gpu.getCoordinationNumbers()
    o = Oracle(Z, X, charge)
    dev = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    frag = o.topology(9, 1)
    qf_atom = o.atom_data(6)
    qfrag = np.zeros(o.nfrag)
    qfrag[frag] = qf_atom
    d = {"n": len(Z), "nfrag": o.nfrag, "xyz": dev(np.asarray(X) / 0.529177210903),
         "alpha": dev(o.atom_data(2)), "gam": dev(o.atom_data(3)), "chi": dev(o.atom_data(4)),
         "cnf": dev(o.atom_data(5)), "cn": dev(cn), "frag": dev(frag, torch.int32),
         "qfrag": dev(qfrag), "frag_host": frag, "qfrag_host": qfrag, "q": torch.zeros(len(Z), dtype=torch.float64, device="cuda"),
         "status": torch.full((1,), -1, dtype=torch.int32, device="cuda")}
    return gpu, d, q_ref


def _call(lib, d, expect=0):
    import torch
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.gfnff_eeq_charges_noalloc(d["n"], d["nfrag"], P(d["xyz"]), P(d["alpha"]), P(d["gam"]), P(d["chi"]),
                                       P(d["cnf"]), P(d["cn"]), P(d["frag"]), P(d["qfrag"]), P(d["q"]),
                                       P(d["status"]), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(d["status"].item()) == expect
    return d["q"].cpu().numpy()


def test_noalloc_charges_match_regular_entry_point_twice():
    g = golden("caffeine")
    gpu_a, a, qa = _inputs(np.array(g["Z"]), np.array(g["xyz_angstrom"]))
    Zw, Xw = workloads.water_cluster(100, 21)
    gpu_b, b, qb = _inputs(Zw, Xw)
    lib = gpu_a._lib
    # two calls in a row on different systems: the shared scratch must not carry over
    q1 = _call(lib, b)
    q2 = _call(lib, a)
    assert np.abs(q1 - qb).max() < Q_TOL
    assert np.abs(q2 - qa).max() < Q_TOL
    # and once more on the first system
    q3 = _call(lib, b)
    assert np.abs(q3 - qb).max() < Q_TOL


def test_noalloc_rejects_oversized_system():
    from curcuma_b200 import _lib
    lib = _lib.load()
    rc = lib.gfnff_eeq_charges_noalloc(2000, 1, *([ctypes.c_void_p(1)] * 10), None)
    assert rc == 1   # GFNFF_INVALID_ARG


def _ammonium_water():
    """NH4+ (N-H 1.03 A, tetrahedral) and a water 3.5 A away: two fragments, charge +1."""
    t = 1.03 / np.sqrt(3.0)
    nh4 = [[0, 0, 0], [t, t, t], [t, -t, -t], [-t, t, -t], [-t, -t, t]]
    a = np.deg2rad(104.52 / 2)
    h2o = [[3.5, 0, 0], [3.5 + 0.9572 * np.cos(a), 0.9572 * np.sin(a), 0],
           [3.5 + 0.9572 * np.cos(a), -0.9572 * np.sin(a), 0]]
    return np.array([7, 1, 1, 1, 1, 8, 1, 1]), np.array(nh4 + h2o, dtype=float)


def test_noalloc_charged_systems():
    """Nonzero target charges: q0 = qfrag/n_f, the residual x - A q0 and the anchors'
    expansion, one charged fragment and a charged + a neutral fragment."""
    from curcuma_b200 import _lib
    lib = _lib.load()
    g = golden("caffeine")
    cases = [(np.array(g["Z"]), np.array(g["xyz_angstrom"]), 1), (*_ammonium_water(), 1)]
    for Z, X, charge in cases:
        gpu, d, q_ref = _inputs(Z, X, charge)
        assert abs(d["qfrag_host"].sum() - charge) < 1e-12
        q = _call(lib, d)
        assert np.abs(q - q_ref).max() < Q_TOL
        for f in range(d["nfrag"]):
            assert abs(q[d["frag_host"] == f].sum() - d["qfrag_host"][f]) < Q_TOL
    # the two-fragment case really has two fragments
    assert _inputs(*_ammonium_water(), 1)[1]["nfrag"] == 2


def _tiny(frag, nfrag, gam=None):
    """A three-atom water with caller-chosen fragment ids; d_qfrag is allocated nfrag + 1
    long and the scratch holds far more than three atoms, so no access leaves allocated
    memory even if the device-side check were missing."""
    import torch
    Zw, Xw = workloads.water_cluster(1, 5)
    o = Oracle(Zw, Xw)
    dev = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    return {"n": 3, "nfrag": nfrag, "xyz": dev(np.asarray(Xw) / 0.529177210903), "alpha": dev(o.atom_data(2)),
            "gam": dev(o.atom_data(3) if gam is None else gam), "chi": dev(o.atom_data(4)),
            "cnf": dev(o.atom_data(5)), "cn": dev(o.atom_data(1)), "frag": dev(frag, torch.int32),
            "qfrag": dev(np.zeros(nfrag + 1)), "q": torch.full((3,), 7.0, dtype=torch.float64, device="cuda"),
            "status": torch.full((1,), -1, dtype=torch.int32, device="cuda")}


def test_noalloc_rejects_bad_fragment_ids_on_device():
    """An id equal to nfrag, a negative id and an unused id: GFNFF_INVALID_ARG in the
    status and d_q left as it was; a good call afterwards still solves."""
    from curcuma_b200 import _lib
    lib = _lib.load()
    for frag, nfrag in (([0, 1, 0], 1), ([0, -1, 0], 1), ([0, 0, 0], 2)):
        q = _call(lib, _tiny(frag, nfrag), expect=1)
        assert np.all(q == 7.0)
    q = _call(lib, _tiny([0, 0, 0], 1))
    assert abs(q.sum()) < 1e-12 and np.all(q != 7.0)


def test_noalloc_not_spd_leaves_output_untouched():
    """A negative hardness makes the reduced matrix indefinite: GFNFF_NOT_SPD and d_q
    unchanged."""
    from curcuma_b200 import _lib
    lib = _lib.load()
    q = _call(lib, _tiny([0, 0, 0], 1, gam=np.full(3, -5.0)), expect=3)
    assert np.all(q == 7.0)
