"""Host-side mirror of curcuma's GFN-FF method plugin.

``GFNFF`` follows ``ComputationalMethod`` as implemented by ``GFNFFGPUComputationalMethod``
(src/core/energy_calculators/computational_method.h:43-360,
qm_methods/gfnff_gpu_method.h:52-194): ``setMolecule`` runs the topology/parameter setup
once, ``updateGeometry`` + ``calculateEnergy(gradient)`` evaluate one geometry, and the
results are read back with ``getGradient`` / ``getCharges`` / ``getEnergyDecomposition``.
Errors follow curcuma's convention: a returned energy of 0.0 plus ``hasError()``.
"""
import ctypes

import numpy as np

from . import _lib

FP64 = 0
MIXED = 1


class GFNFF:
    def __init__(self, precision: int = FP64, device: int = 0, hbond: bool = True,
                 hb_rmsd_bohr: float = 0.3):
        self._lib = _lib.load()
        opts = _lib.Options()
        self._lib.gfnff_default_options(ctypes.byref(opts))
        opts.precision = precision
        opts.device = device
        opts.hbond = 1 if hbond else 0
        opts.hb_rmsd_bohr = hb_rmsd_bohr
        h = ctypes.c_void_p()
        st = self._lib.gfnff_create(ctypes.byref(opts), ctypes.byref(h))
        if st != _lib.GFNFF_OK:
            raise RuntimeError(f"gfnff_create: {_lib.STATUS_NAMES.get(st)}: "
                               f"{self._lib.gfnff_last_error(None).decode()}")
        self._h = h
        self._n = 0
        self._xyz = None
        self._grad = None
        self._terms = np.zeros(_lib.NTERMS)
        self._nmol = 0
        self._err = ""

    # -- ComputationalMethod interface ---------------------------------------------
    def setMolecule(self, Z, xyz_angstrom, charge: int = 0) -> bool:
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        X = np.ascontiguousarray(xyz_angstrom, dtype=np.float64).reshape(-1, 3)
        if len(Z) != len(X):
            raise ValueError("Z and geometry sizes differ")
        st = self._lib.gfnff_setup(self._h, len(Z), Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(charge))
        if st != _lib.GFNFF_OK:
            self._err = self._lib.gfnff_last_error(self._h).decode()
            return False
        self._n = len(Z)
        self._xyz = X.copy()
        self._grad = np.zeros((self._n, 3))
        self._err = ""
        return True

    def updateGeometry(self, xyz_angstrom) -> bool:
        X = np.ascontiguousarray(xyz_angstrom, dtype=np.float64).reshape(-1, 3)
        if X.shape[0] != self._n:
            self._err = "atom count mismatch"
            return False
        self._xyz = X
        return True

    def calculateEnergy(self, gradient: bool = True) -> float:
        e = ctypes.c_double(0.0)
        st = self._lib.gfnff_energy_and_gradient(
            self._h, self._xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(e),
            self._grad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            self._terms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if st != _lib.GFNFF_OK:
            self._err = f"{_lib.STATUS_NAMES.get(st)}: {self._lib.gfnff_last_error(self._h).decode()}"
            return 0.0
        self._err = ""
        return e.value

    # -- batches of independent molecules ----------------------------------------
    def setMoleculeBatch(self, molecules, charges=None) -> bool:
        """molecules: sequence of (Z, xyz_angstrom); charges: per molecule or None."""
        nat = np.array([len(z) for z, _ in molecules], dtype=np.int32)
        Z = np.ascontiguousarray(np.concatenate([np.asarray(z) for z, _ in molecules]), dtype=np.int32)
        X = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1, 3)
                                                 for _, x in molecules]))
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.int32)
        IP, DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        st = self._lib.gfnff_setup_batch(self._h, len(nat), nat.ctypes.data_as(IP), Z.ctypes.data_as(IP),
                                         X.ctypes.data_as(DP), None if ch is None else ch.ctypes.data_as(IP))
        if st != _lib.GFNFF_OK:
            self._err = self._lib.gfnff_last_error(self._h).decode()
            return False
        self._n = len(Z)
        self._nmol = len(nat)
        self._xyz = X.copy()
        self._grad = np.zeros((self._n, 3))
        self._err = ""
        return True

    def calculateEnergyBatch(self):
        """Energies of all molecules (0.0 where a molecule failed) and their status codes."""
        e = np.zeros(self._nmol)
        st = np.zeros(self._nmol, dtype=np.int32)
        DP = ctypes.POINTER(ctypes.c_double)
        rc = self._lib.gfnff_energy_and_gradient_batch(self._h, self._xyz.ctypes.data_as(DP), e.ctypes.data_as(DP),
                                                       self._grad.ctypes.data_as(DP),
                                                       st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        self._err = "" if rc == _lib.GFNFF_OK else \
            f"{_lib.STATUS_NAMES.get(rc)}: {self._lib.gfnff_last_error(self._h).decode()}"
        return e, st

    def getGradient(self) -> np.ndarray:
        return self._grad.copy()

    def getCharges(self) -> np.ndarray:
        q = np.zeros(self._n)
        self._check(self._lib.gfnff_charges(self._h, q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return q

    def getCoordinationNumbers(self) -> np.ndarray:
        cn = np.zeros(self._n)
        self._check(self._lib.gfnff_coordination_numbers(self._h, cn.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return cn

    def getEnergyDecomposition(self) -> dict:
        return {k: float(v) for k, v in zip(_lib.TERM_NAMES, self._terms)}

    def hasError(self) -> bool:
        return bool(self._err)

    def getErrorMessage(self) -> str:
        return self._err

    # -- extras ----------------------------------------------------------------------
    def topology(self, kind: int, width: int) -> np.ndarray:
        cnt = ctypes.c_long(0)
        self._check(self._lib.gfnff_get_topology(self._h, kind, None, 0, ctypes.byref(cnt)))
        out = np.zeros(max(1, cnt.value * width), dtype=np.int32)
        self._check(self._lib.gfnff_get_topology(self._h, kind, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 out.size, ctypes.byref(cnt)))
        return out[:cnt.value * width].reshape(cnt.value, width) if width > 1 else out[:cnt.value]

    def eeqSolver(self) -> str:
        """EEQ solver chosen at setup ("library", "tiled", "pcg", "lu", "batched")."""
        return self._lib.gfnff_eeq_solver(self._h).decode()

    def eeqIterations(self) -> int:
        """Iterations of the last iterative EEQ solve (0 for direct solvers)."""
        return int(self._lib.gfnff_eeq_iterations(self._h))

    def sizes(self):
        n, f = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.gfnff_sizes(self._h, ctypes.byref(n), ctypes.byref(f)))
        return n.value, f.value

    @property
    def handle(self):
        return self._h

    def _check(self, st):
        if st != _lib.GFNFF_OK:
            raise RuntimeError(f"{_lib.STATUS_NAMES.get(st)}: {self._lib.gfnff_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gfnff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
