"""Parameter file (the set-up result cached on disk), on CPU: the library writes it without a
GPU, and the oracle evaluated over the model read back from it gives bit-identical energies
and gradients to the oracle over a fresh set-up."""
import ctypes

import numpy as np
import pytest

from curcuma_b200 import workloads, write_parameters
from tests.oracle_api import TERMS, Oracle, golden, golden_names


def _systems():
    out = {name: (np.array(golden(name)["Z"]), np.array(golden(name)["xyz_angstrom"], dtype=float))
           for name in golden_names()[:6]}
    out["water64"] = workloads.water_cluster(64, 9)
    out["alkane"] = workloads.alkane(32, 1001)
    return out


@pytest.mark.parametrize("name", list(_systems()))
def test_round_trip_bit_identical(name, tmp_path):
    Z, X = _systems()[name]
    path = tmp_path / "mol.param.bin"
    write_parameters(Z, X, path)
    # one thread: the oracle's OpenMP reductions sum in a schedule-dependent order
    a = Oracle(Z, X).engrad(X, nthreads=1)
    b = Oracle.from_parameters(path, Z).engrad(X, nthreads=1)
    for k in TERMS:
        assert a[0][k] == b[0][k], k
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_deterministic_and_refuses_bad_files(tmp_path):
    Z, X = workloads.water_cluster(16, 3)
    p1, p2 = tmp_path / "a.bin", tmp_path / "b.bin"
    write_parameters(Z, X, p1)
    write_parameters(Z, X, p2)
    assert p1.read_bytes() == p2.read_bytes()
    data = p1.read_bytes()
    (tmp_path / "short.bin").write_bytes(data[: len(data) // 2])
    (tmp_path / "bad.bin").write_bytes(b"NOTAPARAMFILE" + data[13:])
    for bad in ("short.bin", "bad.bin", "missing.bin"):
        with pytest.raises(RuntimeError):
            Oracle.from_parameters(tmp_path / bad, Z)


def test_write_rejects_invalid_input(tmp_path):
    with pytest.raises((RuntimeError, ValueError)):
        write_parameters(np.array([1, 1], dtype=np.int32), np.zeros((3, 3)), tmp_path / "x.bin")
    with pytest.raises(RuntimeError):
        write_parameters(np.array([1], dtype=np.int32), np.zeros((1, 3)), tmp_path / "no_dir" / "x.bin")
