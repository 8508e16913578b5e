"""ctypes binding of libgfnff_b200.so (include/gfnff_b200.h).

The library is built in-tree by ``curcuma_b200/build.py``.  Loading fails loudly when it
is missing: there is no CPU fallback for the GPU energy path.
"""
import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgfnff_b200.so"

GFNFF_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "SETUP_FAILED", 3: "NOT_SPD", 4: "NONFINITE",
                5: "REFINE_NOT_CONVERGED", 6: "CUDA_ERROR", 7: "NOT_READY"}
TERM_NAMES = ["bond", "angle", "torsion", "inversion", "storsion", "dispersion", "bonded_rep",
              "nonbonded_rep", "coulomb", "hbond", "xbond", "atm", "batm", "solvation", "total"]
NTERMS = len(TERM_NAMES)

# exported symbols declared in include/gfnff_b200.h
EXPORTED = ["gfnff_default_options", "gfnff_create", "gfnff_setup", "gfnff_energy_and_gradient",
            "gfnff_energy_and_gradient_device", "gfnff_stream", "gfnff_charges",
            "gfnff_coordination_numbers", "gfnff_get_topology", "gfnff_sizes", "gfnff_last_error",
            "gfnff_destroy", "gfnff_set_phase_timing", "gfnff_phase_times", "gfnff_fma_peak_tflops",
            "gfnff_eeq_charges_noalloc", "gfnff_eeq_solver", "gfnff_eeq_iterations", "gfnff_setup_batch",
            "gfnff_energy_and_gradient_batch", "gfnff_md_nve", "gfnff_kernels_per_evaluation",
            "gfnff_save_parameters", "gfnff_setup_from_parameters", "gfnff_write_parameters",
            "gfnff_pair_kernel", "gfnff_eeq_fp64_products", "gfnff_set_solvent", "gfnff_set_geometry_file",
            "gfnff_topology_cache_hit", "gfnff_write_topology_cache", "gfnff_set_unit_cell"]
PHASES = ["positions", "cn", "d4_weights", "eeq_matrix", "eeq_rhs", "eeq_solve", "bonded",
          "hbonds", "repulsion", "pairs", "post_chain", "finish"]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("hbond", ctypes.c_int),
                ("hb_rmsd_bohr", ctypes.c_double), ("gradient", ctypes.c_int)]


_lib = None


def load():
    """Returns the loaded library; raises if the in-tree build is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python curcuma_b200/build.py` first "
                           "(the GFN-FF GPU path has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.POINTER
    c_d, c_i, c_v = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    lib.gfnff_default_options.argtypes = [P(Options)]
    lib.gfnff_create.argtypes = [P(Options), P(c_v)]
    lib.gfnff_setup.argtypes = [c_v, c_i, P(c_i), P(c_d), c_i]
    lib.gfnff_energy_and_gradient.argtypes = [c_v, P(c_d), P(c_d), P(c_d), P(c_d)]
    lib.gfnff_energy_and_gradient_device.argtypes = [c_v, c_v, c_v, c_v, c_v]
    lib.gfnff_stream.argtypes = [c_v]
    lib.gfnff_stream.restype = c_v
    lib.gfnff_charges.argtypes = [c_v, P(c_d)]
    lib.gfnff_coordination_numbers.argtypes = [c_v, P(c_d)]
    lib.gfnff_get_topology.argtypes = [c_v, c_i, P(c_i), ctypes.c_long, P(ctypes.c_long)]
    lib.gfnff_sizes.argtypes = [c_v, P(c_i), P(c_i)]
    lib.gfnff_last_error.argtypes = [c_v]
    lib.gfnff_last_error.restype = ctypes.c_char_p
    lib.gfnff_destroy.argtypes = [c_v]
    lib.gfnff_set_phase_timing.argtypes = [c_v, c_i]
    lib.gfnff_phase_times.argtypes = [c_v, P(c_d), c_i]
    lib.gfnff_fma_peak_tflops.argtypes = [c_i, c_i]
    lib.gfnff_fma_peak_tflops.restype = c_d
    lib.gfnff_eeq_charges_noalloc.argtypes = [c_i, c_i] + [c_v] * 11
    lib.gfnff_eeq_solver.argtypes = [c_v]
    lib.gfnff_eeq_solver.restype = ctypes.c_char_p
    lib.gfnff_pair_kernel.argtypes = [c_v]
    lib.gfnff_pair_kernel.restype = ctypes.c_char_p
    lib.gfnff_eeq_iterations.argtypes = [c_v]
    lib.gfnff_eeq_fp64_products.argtypes = [c_v]
    lib.gfnff_set_solvent.argtypes = [c_v, ctypes.c_char_p]
    lib.gfnff_set_geometry_file.argtypes = [c_v, ctypes.c_char_p, c_i]
    lib.gfnff_set_unit_cell.argtypes = [c_v, P(c_d)]
    lib.gfnff_topology_cache_hit.argtypes = [c_v]
    lib.gfnff_write_topology_cache.argtypes = [c_i, P(c_i), P(c_d), c_i, ctypes.c_char_p, P(c_i)]
    lib.gfnff_kernels_per_evaluation.argtypes = [c_v]
    lib.gfnff_save_parameters.argtypes = [c_v, ctypes.c_char_p]
    lib.gfnff_setup_from_parameters.argtypes = [c_v, ctypes.c_char_p, c_i, P(c_i)]
    lib.gfnff_write_parameters.argtypes = [c_i, P(c_i), P(c_d), c_i, c_i, ctypes.c_char_p]
    lib.gfnff_setup_batch.argtypes = [c_v, c_i, P(c_i), P(c_i), P(c_d), P(c_i)]
    lib.gfnff_energy_and_gradient_batch.argtypes = [c_v, P(c_d), P(c_d), P(c_d), P(c_i)]
    lib.gfnff_md_nve.argtypes = [c_v, c_i, c_d, P(c_d), P(c_d), P(c_d), P(c_d), P(c_d)]
    for name in EXPORTED:
        if name not in ("gfnff_default_options", "gfnff_stream", "gfnff_last_error", "gfnff_fma_peak_tflops",
                        "gfnff_eeq_solver", "gfnff_pair_kernel"):
            getattr(lib, name).restype = c_i
    _lib = lib
    return lib
