"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) for the tests.

The oracle is test infrastructure: a CPU restatement of curcuma's per-geometry GFN-FF
energy + gradient that the GPU path is checked against.  It is built from oracle/ by
``make -C oracle`` (``__graft_entry__.build()`` does that too).
"""
import ctypes
import json
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
BOHR_A = 0.529177210903   # Angstrom per bohr (the library's kAngToBohr)
LIB = ROOT / "oracle" / "_build" / "liboracle.so"
GOLDEN = ROOT / "tests" / "golden"
TERMS = ["bond", "angle", "torsion", "inversion", "storsion", "dispersion", "bonded_rep",
         "nonbonded_rep", "coulomb", "hbond", "xbond", "atm", "batm", "solvation", "total"]
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)
        L = ctypes.CDLL(str(LIB))
        c_v, c_i = ctypes.c_void_p, ctypes.c_int
        L.oracle_create.restype = c_v
        L.oracle_create.argtypes = [c_i, c_v, c_v, c_i]
        L.oracle_create_cached.restype = c_v
        L.oracle_create_cached.argtypes = [c_i, c_v, c_v, c_i, ctypes.c_char_p]
        L.oracle_topo_cache_hit.argtypes = [c_v]
        L.oracle_topo_cache_hit.restype = c_i
        L.oracle_set_cell.argtypes = [c_v, c_v]
        L.oracle_set_cell.restype = c_i
        L.oracle_create_from_parameters.restype = c_v
        L.oracle_create_from_parameters.argtypes = [ctypes.c_char_p]
        L.oracle_destroy.argtypes = [c_v]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_engrad.argtypes = [c_v, c_v, c_v, c_v, c_v, c_v, c_i]
        L.oracle_engrad.restype = c_i
        L.oracle_redetect_hbxb.argtypes = [c_v, c_v]
        L.oracle_list.argtypes = [c_v, c_i, c_v, ctypes.c_long]
        L.oracle_list.restype = ctypes.c_long
        L.oracle_atom_data.argtypes = [c_v, c_i, c_v]
        L.oracle_nfrag.argtypes = [c_v]
        L.oracle_term_params.argtypes = [c_v, c_i, c_v, ctypes.c_long]
        L.oracle_term_params.restype = ctypes.c_long
        L.oracle_set_solvent.argtypes = [c_v, ctypes.c_char_p]
        L.oracle_refresh_topology.argtypes = [c_v, c_v]
        L.oracle_refresh_topology.restype = c_i
        L.oracle_set_solvent.restype = c_i
        _lib = L
    return _lib


class Oracle:
    def __init__(self, Z, xyz, charge=0, solvent=None, topo_cache=None, unit_cell=None):
        """topo_cache: a `<geometry>.topo.json` consulted before Phase 1 (cache_hit tells
        whether it was used); unit_cell: 3x3, rows the lattice vectors (Angstrom)."""
        self.Z = np.ascontiguousarray(Z, dtype=np.int32)
        X = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.n = len(self.Z)
        if topo_cache:
            self.h = lib().oracle_create_cached(self.n, self.Z.ctypes.data, X.ctypes.data, int(charge),
                                                str(topo_cache).encode())
        else:
            self.h = lib().oracle_create(self.n, self.Z.ctypes.data, X.ctypes.data, int(charge))
        if not self.h:
            raise RuntimeError(lib().oracle_last_error().decode())
        if solvent and lib().oracle_set_solvent(self.h, solvent.encode()) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        if unit_cell is not None:
            cell = np.ascontiguousarray(unit_cell, dtype=np.float64).reshape(9)
            if lib().oracle_set_cell(self.h, cell.ctypes.data) != 0:
                raise RuntimeError(lib().oracle_last_error().decode())

    @property
    def cache_hit(self):
        return lib().oracle_topo_cache_hit(self.h) == 1

    @classmethod
    def from_parameters(cls, path, Z):
        """The oracle over the model stored in a parameter file (for round-trip checks)."""
        self = cls.__new__(cls)
        self.Z = np.ascontiguousarray(Z, dtype=np.int32)
        self.n = len(self.Z)
        self.h = lib().oracle_create_from_parameters(str(path).encode())
        if not self.h:
            raise RuntimeError(lib().oracle_last_error().decode())
        return self

    def engrad(self, xyz, nthreads=0):
        X = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        T = np.zeros(len(TERMS))
        G = np.zeros((self.n, 3))
        q = np.zeros(self.n)
        cn = np.zeros(self.n)
        rc = lib().oracle_engrad(self.h, X.ctypes.data, T.ctypes.data, G.ctypes.data, q.ctypes.data,
                                 cn.ctypes.data, nthreads)
        if rc != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return dict(zip(TERMS, T)), G, q, cn

    def refresh_topology(self, xyz):
        X = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        return lib().oracle_refresh_topology(self.h, X.ctypes.data) == 1

    def redetect_hbxb(self, xyz):
        X = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        lib().oracle_redetect_hbxb(self.h, X.ctypes.data)

    def topology(self, kind, width):
        cnt = lib().oracle_list(self.h, kind, None, 0)
        out = np.zeros(max(1, cnt * width), dtype=np.int32)
        lib().oracle_list(self.h, kind, out.ctypes.data, out.size)
        return out[:cnt * width].reshape(cnt, width) if width > 1 else out[:cnt]

    def atom_data(self, which):
        out = np.zeros(self.n)
        lib().oracle_atom_data(self.h, which, out.ctypes.data)
        return out

    def term_params(self, kind):
        """Set-up parameters per term (see oracle_term_params): a (count, width) array."""
        width = {0: 7, 1: 5, 2: 8, 3: 7}[kind]
        cnt = lib().oracle_term_params(self.h, kind, None, 0)
        out = np.zeros(max(1, cnt * width))
        lib().oracle_term_params(self.h, kind, out.ctypes.data, out.size)
        return out[:cnt * width].reshape(cnt, width)

    @property
    def nfrag(self):
        return lib().oracle_nfrag(self.h)

    def __del__(self):
        try:
            if self.h:
                lib().oracle_destroy(self.h)
        except Exception:
            pass


class OracleSequence:
    """The oracle over a sequence of geometries with the refreshes of curcuma's evaluation, in
    the order the library's single-point path applies them: the topology when an atom has moved
    more than 0.5 bohr along an axis since the last topology (a topology with new fragments
    also re-detects the HB/XB lists at their reference geometry, as the library does), then
    the HB/XB lists when sqrt(sum d^2)/N exceeds hb_rmsd_bohr since their last detection."""

    def __init__(self, Z, X, charge=0, solvent=None, hb_rmsd_bohr=0.3, unit_cell=None):
        self.oracle = Oracle(Z, X, charge, solvent, unit_cell=unit_cell)
        self.topo = np.asarray(X, dtype=np.float64) / BOHR_A
        self.hb = self.topo.copy()
        self.thr = hb_rmsd_bohr

    def engrad(self, X, nthreads=0):
        xb = np.asarray(X, dtype=np.float64) / BOHR_A
        if np.abs(xb - self.topo).max() > 0.5:
            frag0 = self.oracle.topology(9, 1).copy()
            self.oracle.refresh_topology(X)
            self.topo = xb
            if not np.array_equal(frag0, self.oracle.topology(9, 1)):
                self.oracle.redetect_hbxb(self.hb * BOHR_A)
        if np.sqrt(((xb - self.hb) ** 2).sum()) / len(xb) > self.thr:
            self.oracle.redetect_hbxb(X)
            self.hb = xb
        return self.oracle.engrad(X, nthreads)


def golden(name):
    return json.loads((GOLDEN / f"{name}.json").read_text())


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.json") if not p.stem.startswith("cli_"))
