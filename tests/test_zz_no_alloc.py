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


def _inputs(Z, X):
    """Per-atom EEQ inputs of the model (from the setup shared with the oracle) and the
    reference charges/CN of one gfnff_energy_and_gradient evaluation."""
    import torch
    gpu = GFNFF()
    assert gpu.setMolecule(Z, X), gpu.getErrorMessage()
    gpu.calculateEnergy(True)
    assert not gpu.hasError(), gpu.getErrorMessage()
    q_ref = gpu.getCharges()
    cn = gpu.getCoordinationNumbers()
    o = Oracle(Z, X)
    dev = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    frag = o.topology(9, 1)
    d = {"n": len(Z), "nfrag": o.nfrag, "xyz": dev(np.asarray(X) / 0.529177210903),
         "alpha": dev(o.atom_data(2)), "gam": dev(o.atom_data(3)), "chi": dev(o.atom_data(4)),
         "cnf": dev(o.atom_data(5)), "cn": dev(cn), "frag": dev(frag, torch.int32),
         "qfrag": dev(np.zeros(o.nfrag)), "q": torch.zeros(len(Z), dtype=torch.float64, device="cuda"),
         "status": torch.full((1,), -1, dtype=torch.int32, device="cuda")}
    return gpu, d, q_ref


def _call(lib, d):
    import torch
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.gfnff_eeq_charges_noalloc(d["n"], d["nfrag"], P(d["xyz"]), P(d["alpha"]), P(d["gam"]), P(d["chi"]),
                                       P(d["cnf"]), P(d["cn"]), P(d["frag"]), P(d["qfrag"]), P(d["q"]),
                                       P(d["status"]), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(d["status"].item()) == 0
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
