/*
 * gfnff_b200 - GFN-FF energy + analytic gradient on NVIDIA B200 (sm_100a).
 *
 * C ABI of the drop-in for curcuma's `-method gfnff -gpu cuda` path.  One handle owns
 * one molecule (or one batch of molecules), its topology and parameters cached on the
 * device, and one CUDA stream.  Handles are not thread-safe.
 *
 * Units: coordinates in Angstrom at the boundary (as curcuma's Mol geometry),
 * energies in Hartree, gradients in Hartree/bohr (row-major N x 3), like
 * ComputationalMethod::getGradient().
 */
#ifndef GFNFF_B200_H
#define GFNFF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GFNFF_OK = 0,
    GFNFF_INVALID_ARG = 1,        /* bad pointer, size or element */
    GFNFF_SETUP_FAILED = 2,       /* topology / parameter generation failed */
    GFNFF_NOT_SPD = 3,            /* EEQ matrix not positive definite */
    GFNFF_NONFINITE = 4,          /* non-finite energy or gradient */
    GFNFF_REFINE_NOT_CONVERGED = 5,/* mixed-precision refinement did not reach 1e-10 */
    GFNFF_CUDA_ERROR = 6,         /* CUDA / cuSOLVER failure */
    GFNFF_NOT_READY = 7           /* gfnff_setup has not been called */
} gfnff_status;

/* precision of the per-geometry evaluation */
enum { GFNFF_FP64 = 0, GFNFF_MIXED = 1 };

/* per-term energies reported through gfnff_terms (Hartree) */
enum {
    GFNFF_E_BOND = 0, GFNFF_E_ANGLE, GFNFF_E_TORSION, GFNFF_E_INVERSION, GFNFF_E_STORSION,
    GFNFF_E_DISPERSION, GFNFF_E_BONDED_REP, GFNFF_E_NONBONDED_REP, GFNFF_E_COULOMB,
    GFNFF_E_HBOND, GFNFF_E_XBOND, GFNFF_E_ATM, GFNFF_E_BATM, GFNFF_E_SOLVATION, GFNFF_E_TOTAL, GFNFF_NTERMS
};

typedef struct {
    int precision;          /* GFNFF_FP64 (default) or GFNFF_MIXED */
    int device;             /* CUDA device ordinal */
    int hbond;              /* 1: hydrogen/halogen bonds on (default) */
    double hb_rmsd_bohr;    /* HB/XB list refresh threshold, default 0.3 */
    int gradient;           /* GFNFF_GRADIENT_REFERENCE (default) or GFNFF_GRADIENT_EXACT */
} gfnff_options;

/* Gradient definition.  REFERENCE reproduces curcuma's analytic gradient: it adds the
 * D4 dC6/dCN chain term although the dispersion energy uses the C6 of the set-up
 * geometry (ff_workspace_gfnff.cpp:715-772, gfnff_method.cpp:1333-1345), and it treats
 * the EEQ charges as stationary although the Coulomb pair energy is cut at 100 bohr
 * while the EEQ matrix is not.  EXACT is the derivative of the same energy: no dC6/dCN
 * term, plus the charge response of the cut pairs (one extra solve with the EEQ matrix
 * and one extra pair pass, only when a pair exceeds the cut).  The energy is the same. */
enum { GFNFF_GRADIENT_REFERENCE = 0, GFNFF_GRADIENT_EXACT = 1 };

typedef struct gfnff_handle gfnff_handle;

/* Fills opts with the defaults (FP64, device 0, HB on, 0.3 bohr). */
void gfnff_default_options(gfnff_options* opts);

/* ALPB implicit solvation for the next gfnff_setup / gfnff_setup_from_parameters of this
 * handle (curcuma's -gfnff.solvent, gfnff_method.cpp:811-840: the solvent's reaction field
 * enters the EEQ solve, A += B, and the solvation free energy 1/2 q^T B q + G_sasa + G_shift
 * is reported as GFNFF_E_SOLVATION; curcuma's solvent names and aliases, case-insensitive;
 * NULL, "" or "none": gas phase, the default).  Single-molecule handles only.  Returns
 * GFNFF_INVALID_ARG for an unknown solvent. */
gfnff_status gfnff_set_solvent(gfnff_handle* h, const char* solvent);

/* Replaces GFNFFGPUComputationalMethod construction
 * (src/core/energy_calculators/qm_methods/gfnff_gpu_method.h:52-194). */
gfnff_status gfnff_create(const gfnff_options* opts, gfnff_handle** out);

/* Replaces ComputationalMethod::setMolecule -> GFNFF::InitialiseMolecule
 * (computational_method.h:43-360, ff_methods/gfnff_method.cpp:709-848): topology and
 * parameters are generated on the host and cached on the device. */
gfnff_status gfnff_setup(gfnff_handle* h, int natoms, const int* Z, const double* xyz_angstrom,
                         int total_charge);

/* Parameter file: the complete set-up result (topology, parameters, term lists) of the
 * handle's molecule, so that a later run on the same structure skips the set-up.  Plays the
 * role of curcuma's parameter caching (`<input>.param.json`, PARAMETER_CACHING.md) and
 * topology export/import (ff_methods/gfnff_method.cpp:2515-2811); the format is this
 * library's own binary image, read only by a build with the same record layouts.
 * gfnff_save_parameters writes the model of a single-molecule handle after gfnff_setup
 * (with the HB/XB lists of the last detection); gfnff_setup_from_parameters replaces
 * gfnff_setup with a file (the file's set-up options apply) and refuses a file made for
 * another structure (natoms and Z must match); gfnff_write_parameters runs the set-up on
 * the host and writes the file without a handle or a GPU. */
gfnff_status gfnff_save_parameters(gfnff_handle* h, const char* path);
gfnff_status gfnff_setup_from_parameters(gfnff_handle* h, const char* path, int natoms, const int* Z);
gfnff_status gfnff_write_parameters(int natoms, const int* Z, const double* xyz_angstrom, int total_charge,
                                    int hbond, const char* path);

/* Periodic boundary conditions (curcuma's Mol::setUnitCell, GFNFF::InitialiseMolecule
 * gfnff_method.cpp:724-727 and 794-797, QM/gfnff_gpu_method.cpp:403-408): the unit cell for
 * the next gfnff_setup / gfnff_setup_from_parameters of this handle, 9 doubles in Angstrom,
 * cell_angstrom[3*k + d] = component d of lattice vector k (the column-major data of
 * curcuma's 3x3 cell matrix with the lattice vectors as columns); NULL: isolated system (the
 * default).  As in curcuma's CUDA kernels (cuda/gfnff_kernels.cu:92-119 and its callers)
 * the displacement vectors of the coordination numbers and their chain rule, bonds (with
 * their HB coordination numbers), angles, the A-H, H-B and A-B vectors of hydrogen and
 * halogen bonds, repulsion and the Coulomb and D4 pairs take the minimum image; torsions,
 * inversions, ATM, BATM, the EEQ matrix and the set-up (topology, term lists, D4 pair
 * membership by set-up distance, HB/XB detection) use the plain coordinates.  Single-molecule
 * handles, reference gradient mode, no ALPB: GFNFF_INVALID_ARG otherwise (a singular or
 * non-finite cell too). */
gfnff_status gfnff_set_unit_cell(gfnff_handle* h, const double* cell_angstrom);

/* Topology cache in curcuma's `<geometry>.topo.json` format (its `geometry_file` and
 * `cache_topology` parameters; ff_methods/gfnff_method.cpp:2515-2656 fingerprint and export,
 * 2941-2985 write, 8973-9040 read).  gfnff_set_geometry_file names the geometry file of the
 * next gfnff_setup of this handle; with cache_topology != 0 that set-up reads
 * `<geometry_file without its extension>.topo.json` and, when the file's fingerprint (atom
 * count, elements, geometric bond list) is this structure's, takes the Phase-1 charges,
 * fragment charges, dxi, dgam, alpeeq and amide-H flags from it instead of computing them;
 * after the set-up it writes the file (skipped when the Phase-1 charges fail curcuma's
 * write check, or the file cannot be written).  The topology refresh after a 0.5 bohr
 * displacement consults the same file.  NULL or cache_topology == 0: no cache (the default).
 * gfnff_topology_cache_hit: 1 when the last set-up of h used the cache, 0 when it did not,
 * -1 before a set-up.  gfnff_write_topology_cache runs the host set-up with the cache and
 * writes the file without a handle or a GPU; cache_hit (may be NULL) receives whether the
 * existing file was used. */
gfnff_status gfnff_set_geometry_file(gfnff_handle* h, const char* geometry_file, int cache_topology);
int gfnff_topology_cache_hit(gfnff_handle* h);
gfnff_status gfnff_write_topology_cache(int natoms, const int* Z, const double* xyz_angstrom, int total_charge,
                                        const char* geometry_file, int* cache_hit);

/* Replaces updateGeometry + calculateEnergy(true) + copyGradientTo
 * (gfnff_method.cpp:1692-2226, computational_method.h:121-123).  energy and grad are
 * host pointers; grad may be NULL for energy only (the gradient is still computed);
 * terms may be NULL, else GFNFF_NTERMS doubles. */
gfnff_status gfnff_energy_and_gradient(gfnff_handle* h, const double* xyz_angstrom, double* energy,
                                       double* grad, double* terms);

/* Device-resident variant for MD/optimisation loops: d_xyz_bohr (N*3 doubles, bohr) and
 * the outputs are device pointers; the call only enqueues work on the handle's stream
 * (no host synchronisation, no HB/XB list refresh).  d_energy and d_status receive one
 * value per molecule (nmol of a batch handle, else 1). */
gfnff_status gfnff_energy_and_gradient_device(gfnff_handle* h, const double* d_xyz_bohr,
                                              double* d_energy, double* d_grad, int* d_status);

/* Batched set-up of nmol independent molecules (conformer batches, the uneven-size
 * batches curcuma evaluates one molecule at a time in its conformer tools):
 * natoms[m] atoms each, Z and xyz_angstrom concatenated in molecule order, charges[m]
 * (NULL = all neutral).  Each molecule gets the full single-molecule set-up
 * (gfnff_setup), run in parallel on the host; the molecules do not interact.  Replaces
 * nmol calls of ComputationalMethod::setMolecule. */
gfnff_status gfnff_setup_batch(gfnff_handle* h, int nmol, const int* natoms, const int* Z,
                               const double* xyz_angstrom, const int* charges);

/* Energy + gradient of every molecule of a batch handle in one pass (nmol calls of
 * calculateEnergy + copyGradientTo).  energies: nmol doubles; grad: N*3 (may be NULL);
 * status: nmol gfnff_status values (may be NULL).  Returns the first failing status (the
 * failing molecules' energies are 0.0), else GFNFF_OK.  HB/XB lists stay those of the
 * set-up geometry. */
gfnff_status gfnff_energy_and_gradient_batch(gfnff_handle* h, const double* xyz_angstrom, double* energies,
                                             double* grad, int* status);

/* NVE velocity-Verlet molecular dynamics on the device, the loop of curcuma's SimpleMD
 * (capabilities/simplemd.cpp:2580-2674) with the energy + gradient step replayed as a
 * CUDA graph: nsteps steps of dt_fs femtoseconds.  xyz_angstrom and vel (Angstrom/fs,
 * N*3) are updated in place; mass (N, amu); epot and ekin receive nsteps + 1 energies
 * (Hartree, entry 0 = start).  The HB/XB lists are re-detected every 100 steps when
 * sqrt(sum d^2)/N exceeds hb_rmsd_bohr, as in gfnff_energy_and_gradient.  Returns the
 * first failing evaluation status (the run stops there). */
gfnff_status gfnff_md_nve(gfnff_handle* h, int nsteps, double dt_fs, double* xyz_angstrom, double* vel,
                          const double* mass, double* epot, double* ekin);

/* The handle's CUDA stream (a cudaStream_t). */
void* gfnff_stream(gfnff_handle* h);

/* Phase-2 EEQ charges of the last evaluation (ComputationalMethod::getCharges). */
gfnff_status gfnff_charges(gfnff_handle* h, double* q);

/* Coordination numbers of the last evaluation. */
gfnff_status gfnff_coordination_numbers(gfnff_handle* h, double* cn);

/* Topology lists for bit-exact comparison (same kinds as the oracle's list export):
 * 0 bonds(i,j) 1 angles(i,j,k) 2 torsions(i,j,k,l) 3 inversions 4 dispersion pairs
 * (device-enumerated) 5 non-bonded repulsion pairs 6 hbonds(a,h,b,case) 7 xbonds
 * 8 hybridisation 9 fragment 10 pi fragment 11 bonded repulsion 12 ATM 13 BATM.
 * Writes the record count to *count and up to cap ints into out (may be NULL). */
gfnff_status gfnff_get_topology(gfnff_handle* h, int kind, int* out, long cap, long* count);

/* Atom count and fragment count of the set-up system. */
gfnff_status gfnff_sizes(gfnff_handle* h, int* natoms, int* nfrag);

/* Per-phase CUDA-event timing of every evaluation (off by default; costs two event
 * records per phase).  gfnff_phase_times copies the milliseconds of the last
 * evaluation, in the order positions, cn, d4_weights, eeq_matrix, eeq_rhs,
 * eeq_solve, bonded, hbonds, repulsion, pairs, post_chain, finish, and returns
 * the number of phases (or -1).  Diagnostics without a counterpart in the reference
 * (curcuma prints phase timings at verbosity >= 2 instead, gfnff.h:742). */
gfnff_status gfnff_set_phase_timing(gfnff_handle* h, int on);
int gfnff_phase_times(gfnff_handle* h, double* ms, int cap);

/* FMA throughput of the device in TFLOP/s (fp64 != 0: FP64, else FP32), measured by a
 * short microbenchmark; the roofline denominator of the SIMT pair kernels.  No
 * counterpart in the reference. */
double gfnff_fma_peak_tflops(int device, int fp64);

/* Allocation-free EEQ charges, for callers that cannot allocate device memory (code
 * running inside another framework's memory pool, loops that forbid allocations after
 * start-up).  No counterpart in the reference.  Every buffer is a device pointer owned
 * by the caller: d_xyz_bohr (N*3), per-atom d_alpha (alpha^2 as in the EEQ matrix),
 * d_gam (hardness incl. corrections), d_chi (-chi + corrections), d_cnf, d_cn, d_frag
 * (0-based fragment ids, each in [0, nfrag) and each id used by at least one atom),
 * d_qfrag (nfrag target charges); outputs d_q (N) and d_status (1 int, gfnff_status of
 * the device solve: GFNFF_INVALID_ARG when a fragment id is out of range or unused,
 * GFNFF_NOT_SPD when the reduced EEQ matrix has no Cholesky factor; on either failure
 * d_q is not written).  The fragment ids are checked on the device, in a pass that reads
 * them before anything is indexed by them.  Work is enqueued on `stream` (a
 * cudaStream_t, NULL = legacy default) without host synchronisation.  All intermediate
 * storage is one file-scope device array sized for GFNFF_NOALLOC_MAX_ATOMS atoms (about
 * 17 MB, held by every GPU that loads the library until exit); larger systems return
 * GFNFF_INVALID_ARG.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and should come before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race.  A CUDA error already pending when the call
 * starts is returned as GFNFF_CUDA_ERROR without launching anything and is left pending
 * for the caller; an error of this call's own launches is returned and cleared. */
#define GFNFF_NOALLOC_MAX_ATOMS 1024
gfnff_status gfnff_eeq_charges_noalloc(int natoms, int nfrag, const double* d_xyz_bohr, const double* d_alpha,
                                       const double* d_gam, const double* d_chi, const double* d_cnf,
                                       const double* d_cn, const int* d_frag, const double* d_qfrag,
                                       double* d_q, int* d_status, void* stream);

/* Name of the EEQ solver chosen for the handle's molecule at setup: "tiled" (the in-house
 * persistent tiled Cholesky), "pcg" (block-Jacobi conjugate gradients; FP64 true residual
 * <= 1e-12 max|b| in the FP64 form, <= 1e-10 in the mixed form), "batched" (per-molecule
 * shared-memory Cholesky; tensor-core factorisation with FP64 refinement in the mixed
 * form), "lu" (indefinite matrix, cuSOLVER's pivoted LU) or "library" (cuSOLVER's Cholesky,
 * only when GFNFF_EEQ_SOLVER=library asks for it); "" before setup.  The choice is made by
 * timing the in-house solvers at setup.  curcuma's EEQSolver also picks among several solvers
 * (eeq_solver.cpp:1448-2086); this query has no counterpart there. */
const char* gfnff_eeq_solver(gfnff_handle* h);

/* Variant of the Coulomb + D4 pair kernel that the set-up autotuner picked for the
 * handle's system by timing: "sym32" / "sym64" (each pair once over 32- or 64-atom tiles),
 * "sym64_occ10" (64-atom tiles at 10 blocks per SM) or "rows" (both directions by rows); ""
 * before setup.  The pick is cached per device, batch or single molecule and size bucket.
 * Diagnostic without a counterpart in the reference. */
const char* gfnff_pair_kernel(gfnff_handle* h);

/* Iterations of the last iterative EEQ solve (0 for the direct solvers, -1 before
 * setup); synchronises the handle's stream.  Diagnostic without a counterpart in the
 * reference. */
int gfnff_eeq_iterations(gfnff_handle* h);

/* FP64 products with the reduced EEQ matrix in the last solve of the mixed form's
 * refinement solver (the true-residual checks beside the FP32 inner iterations that
 * gfnff_eeq_iterations counts); -1 for every other solver or before setup.  Synchronises
 * the handle's stream.  Diagnostic without a counterpart in the reference. */
int gfnff_eeq_fp64_products(gfnff_handle* h);

/* Kernels of this library launched per evaluation while the step replays as a CUDA graph
 * (the kernel nodes of the captured graph whose code is in this library, plus the
 * positions kernel launched before it); -1 before the first evaluation or with direct
 * launches.  Diagnostic without a counterpart in the reference. */
int gfnff_kernels_per_evaluation(gfnff_handle* h);

/* Last error message of the handle (static storage when h is NULL). */
const char* gfnff_last_error(gfnff_handle* h);

/* Frees all host and device resources. */
gfnff_status gfnff_destroy(gfnff_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* GFNFF_B200_H */
