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

# standard atomic weights (amu) of H..Ar, for MD when no masses are given
_MASS = [1.008, 4.0026, 6.94, 9.0122, 10.81, 12.011, 14.007, 15.999, 18.998, 20.180, 22.990, 24.305, 26.982,
         28.085, 30.974, 32.06, 35.45, 39.948]


def atomic_masses(Z):
    return np.array([_MASS[z - 1] if 1 <= z <= len(_MASS) else 2.0 * z for z in np.asarray(Z)], dtype=np.float64)


def maxwell_boltzmann(masses_amu, temperature_k, seed):
    """Seeded Maxwell-Boltzmann velocities (Angstrom/fs) without centre-of-mass motion."""
    rng = np.random.default_rng(seed)
    kt = 3.166811563e-6 * temperature_k                      # Hartree
    m = np.asarray(masses_amu, dtype=np.float64) * 1822.888486209  # electron masses
    v = rng.normal(size=(len(m), 3)) * np.sqrt(kt / m)[:, None]    # bohr / atomic time unit
    v -= (m[:, None] * v).sum(axis=0) / m.sum()
    return v * 0.529177210903 * 41.341373335                 # Angstrom / fs


FP64 = 0
MIXED = 1


class GFNFF:
    def __init__(self, precision: int = FP64, device: int = 0, hbond: bool = True,
                 hb_rmsd_bohr: float = 0.3, exact_gradient: bool = False, solvent: str = "none",
                 geometry_file=None, cache_topology: bool = True, unit_cell=None):
        self._lib = _lib.load()
        self._params = {"precision": "mixed" if precision == MIXED else "fp64", "gpu_device": device,
                        "hbond": bool(hbond), "hb_rmsd_bohr": hb_rmsd_bohr,
                        "exact_gradient": bool(exact_gradient), "solvent": solvent or "none", "threads": 1,
                        "geometry_file": str(geometry_file) if geometry_file else "",
                        "cache_topology": bool(cache_topology),
                        "unit_cell": None if unit_cell is None else np.asarray(unit_cell, float).reshape(3, 3).tolist()}
        self._h = None
        self._create()

    def _create(self):
        p = self._params
        opts = _lib.Options()
        self._lib.gfnff_default_options(ctypes.byref(opts))
        opts.precision = MIXED if p["precision"] == "mixed" else FP64
        opts.device = int(p["gpu_device"])
        opts.hbond = 1 if p["hbond"] else 0
        opts.hb_rmsd_bohr = float(p["hb_rmsd_bohr"])
        opts.gradient = 1 if p["exact_gradient"] else 0
        h = ctypes.c_void_p()
        st = self._lib.gfnff_create(ctypes.byref(opts), ctypes.byref(h))
        if st != _lib.GFNFF_OK:
            raise RuntimeError(f"gfnff_create: {_lib.STATUS_NAMES.get(st)}: "
                               f"{self._lib.gfnff_last_error(None).decode()}")
        self._h = h
        st = self._lib.gfnff_set_solvent(h, str(p["solvent"]).encode())
        if st != _lib.GFNFF_OK:
            msg = self._lib.gfnff_last_error(h).decode()
            self._lib.gfnff_destroy(h)
            self._h = None
            raise ValueError(f"gfnff_set_solvent: {msg}")
        self._lib.gfnff_set_geometry_file(h, p["geometry_file"].encode(), 1 if p["cache_topology"] else 0)
        if p["unit_cell"] is not None:
            # rows of unit_cell are the lattice vectors a, b, c (Angstrom): row-major data is
            # the C layout cell[3*k + d]
            cell = np.ascontiguousarray(p["unit_cell"], dtype=np.float64).reshape(9)
            st = self._lib.gfnff_set_unit_cell(h, cell.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            if st != _lib.GFNFF_OK:
                msg = self._lib.gfnff_last_error(h).decode()
                self._lib.gfnff_destroy(h)
                self._h = None
                raise ValueError(f"gfnff_set_unit_cell: {msg}")
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
        self._masses = atomic_masses(Z)
        self._err = ""
        return True

    def saveParameters(self, path) -> bool:
        """Writes the set-up result of this molecule to a parameter file."""
        st = self._lib.gfnff_save_parameters(self._h, str(path).encode())
        if st != _lib.GFNFF_OK:
            self._err = self._lib.gfnff_last_error(self._h).decode()
            return False
        return True

    def setMoleculeFromParameters(self, path, Z, xyz_angstrom) -> bool:
        """setMolecule with the set-up read from a parameter file made for this structure
        (saveParameters or write_parameters); xyz_angstrom is the geometry evaluated until
        updateGeometry is called."""
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        X = np.ascontiguousarray(xyz_angstrom, dtype=np.float64).reshape(-1, 3)
        if len(Z) != len(X):
            raise ValueError("Z and geometry sizes differ")
        st = self._lib.gfnff_setup_from_parameters(self._h, str(path).encode(), len(Z),
                                                   Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if st != _lib.GFNFF_OK:
            self._err = self._lib.gfnff_last_error(self._h).decode()
            return False
        self._n = len(Z)
        self._xyz = X.copy()
        self._grad = np.zeros((self._n, 3))
        self._masses = atomic_masses(Z)
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

    # -- molecular dynamics ------------------------------------------------------
    def runMD(self, nsteps: int, dt_fs: float, velocities_ang_fs, masses_amu=None):
        """NVE velocity Verlet from the current geometry; returns (epot, ekin) traces of
        nsteps + 1 values and updates the geometry and velocities (see velocities())."""
        X = np.ascontiguousarray(self._xyz, dtype=np.float64).copy()
        V = np.ascontiguousarray(velocities_ang_fs, dtype=np.float64).reshape(-1, 3).copy()
        m = np.ascontiguousarray(masses_amu if masses_amu is not None else self._masses, dtype=np.float64)
        ep = np.zeros(nsteps + 1)
        ek = np.zeros(nsteps + 1)
        DP = ctypes.POINTER(ctypes.c_double)
        st = self._lib.gfnff_md_nve(self._h, int(nsteps), float(dt_fs), X.ctypes.data_as(DP), V.ctypes.data_as(DP),
                                    m.ctypes.data_as(DP), ep.ctypes.data_as(DP), ek.ctypes.data_as(DP))
        self._err = "" if st == _lib.GFNFF_OK else \
            f"{_lib.STATUS_NAMES.get(st)}: {self._lib.gfnff_last_error(self._h).decode()}"
        self._xyz = X
        self._vel = V
        return ep, ek

    def velocities(self) -> np.ndarray:
        return self._vel.copy()

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

    def getCN(self) -> np.ndarray:
        """Coordination numbers of the last evaluation (GFNFFComputationalMethod::getCN)."""
        return self.getCoordinationNumbers()

    def copyGradientTo(self, target) -> None:
        """Gradient (Eh/bohr) into a preallocated N x 3 array (computational_method.h:121-123)."""
        target[...] = self._grad

    def hasGradient(self) -> bool:
        return True

    def NumGrad(self, dx: float = 1e-5) -> np.ndarray:
        """Central-difference gradient of calculateEnergy in Eh/bohr, dx in Angstrom; restores
        the current geometry and its results (one more evaluation) afterwards.
        ComputationalMethod::NumGrad has this signature; its GFN-FF implementation keeps the
        base version, which returns an empty matrix."""
        X0 = self._xyz.copy()
        G = np.zeros((self._n, 3))
        for a in range(self._n):
            for d in range(3):
                for sgn in (1.0, -1.0):
                    X = X0.copy()
                    X[a, d] += sgn * dx
                    self.updateGeometry(X)
                    G[a, d] += sgn * self.calculateEnergy(False)
        self.updateGeometry(X0)
        self.calculateEnergy(True)
        return G / (2.0 * dx) * 0.529177210903   # per Angstrom -> per bohr

    def getBondOrders(self) -> np.ndarray:
        """curcuma's GFN-FF keeps a zero vector of N(N-1)/2 bond orders
        (ff_methods/gfnff_method.cpp:783); the same here."""
        return np.zeros(self._n * (self._n - 1) // 2)

    def getDipole(self) -> np.ndarray:
        """(0, 0, 0), as GFNFFComputationalMethod::getDipole returns."""
        return np.zeros(3)

    def getMethodName(self) -> str:
        return "gfnff"

    def isThreadSafe(self) -> bool:
        return False

    def setThreadCount(self, threads: int) -> None:
        """Recorded in the parameters; the per-geometry work runs on the GPU, the host set-up
        uses OpenMP (OMP_NUM_THREADS)."""
        self._params["threads"] = threads if threads > 0 else 1

    def setParameters(self, params: dict) -> None:
        """precision ("fp64"/"mixed"), gpu_device, hbond, hb_rmsd_bohr, exact_gradient, solvent
        (ALPB implicit solvation: curcuma's solvent names, "none" for the gas phase), threads,
        geometry_file and cache_topology (the `<geometry>.topo.json` topology cache), unit_cell
        (3x3, rows the lattice vectors in Angstrom, or None: periodic boundary conditions).
        A new handle is made with them: call setMolecule again afterwards."""
        unknown = set(params) - set(self._params)
        if unknown:
            raise KeyError(f"unknown parameters: {sorted(unknown)}")
        if "geometry_file" in params:
            params = dict(params, geometry_file=str(params["geometry_file"] or ""))
        if "unit_cell" in params and params["unit_cell"] is not None:
            params = dict(params, unit_cell=np.asarray(params["unit_cell"], float).reshape(3, 3).tolist())
        new = dict(self._params, **params)
        if new["precision"] not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if {k: v for k, v in new.items() if k != "threads"} != \
                {k: v for k, v in self._params.items() if k != "threads"}:
            self.close()
            self._params = new
            self._create()
        self._params = new

    def getParameters(self) -> dict:
        return dict(self._params)

    def clearError(self) -> None:
        self._err = ""

    def getHBCount(self) -> int:
        return len(self.topology(6, 4)) if self._n else 0

    def getXBCount(self) -> int:
        return len(self.topology(7, 3)) if self._n else 0

    # -- extras ----------------------------------------------------------------------
    def topology(self, kind: int, width: int) -> np.ndarray:
        cnt = ctypes.c_long(0)
        self._check(self._lib.gfnff_get_topology(self._h, kind, None, 0, ctypes.byref(cnt)))
        out = np.zeros(max(1, cnt.value * width), dtype=np.int32)
        self._check(self._lib.gfnff_get_topology(self._h, kind, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                 out.size, ctypes.byref(cnt)))
        return out[:cnt.value * width].reshape(cnt.value, width) if width > 1 else out[:cnt.value]

    def pairKernel(self) -> str:
        """Pair kernel variant picked by the set-up autotuner (diagnostic)."""
        return self._lib.gfnff_pair_kernel(self._h).decode()

    def eeqSolver(self) -> str:
        """EEQ solver chosen at setup ("library", "tiled", "pcg", "lu", "batched")."""
        return self._lib.gfnff_eeq_solver(self._h).decode()

    def topologyCacheHit(self) -> bool:
        """True when the last setMolecule took its Phase-1 data from `<geometry>.topo.json`."""
        return self._lib.gfnff_topology_cache_hit(self._h) == 1

    def eeqIterations(self) -> int:
        """Iterations of the last iterative EEQ solve (0 for direct solvers)."""
        return int(self._lib.gfnff_eeq_iterations(self._h))

    def eeqFP64Products(self) -> int:
        """FP64 matrix products of the mixed form's refinement solver in the last solve
        (-1 for the other solvers)."""
        return int(self._lib.gfnff_eeq_fp64_products(self._h))

    def kernelsPerEvaluation(self):
        """Kernels of this library per evaluation of the replayed step graph (-1: none yet)."""
        return int(self._lib.gfnff_kernels_per_evaluation(self._h))

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


def write_parameters(Z, xyz_angstrom, path, charge: int = 0, hbond: bool = True) -> None:
    """Runs the GFN-FF set-up on the host and writes its parameter file (no GPU needed);
    GFNFF.setMoleculeFromParameters reads it."""
    lib = _lib.load()
    Z = np.ascontiguousarray(Z, dtype=np.int32)
    X = np.ascontiguousarray(xyz_angstrom, dtype=np.float64).reshape(-1, 3)
    if len(Z) != len(X):
        raise ValueError("Z and geometry sizes differ")
    st = lib.gfnff_write_parameters(len(Z), Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                    X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(charge),
                                    1 if hbond else 0, str(path).encode())
    if st != _lib.GFNFF_OK:
        raise RuntimeError(lib.gfnff_last_error(None).decode())


def write_topology_cache(Z, xyz_angstrom, geometry_file, charge: int = 0) -> bool:
    """Runs the GFN-FF set-up on the host with the topology cache of geometry_file
    (`<geometry_file without extension>.topo.json`, curcuma's format) and writes the cache;
    returns True when the existing file's Phase-1 data were used.  No GPU needed."""
    lib = _lib.load()
    Z = np.ascontiguousarray(Z, dtype=np.int32)
    X = np.ascontiguousarray(xyz_angstrom, dtype=np.float64).reshape(-1, 3)
    if len(Z) != len(X):
        raise ValueError("Z and geometry sizes differ")
    hit = ctypes.c_int(0)
    st = lib.gfnff_write_topology_cache(len(Z), Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(charge),
                                        str(geometry_file).encode(), ctypes.byref(hit))
    if st != _lib.GFNFF_OK:
        raise RuntimeError(lib.gfnff_last_error(None).decode())
    return hit.value == 1
