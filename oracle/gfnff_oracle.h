// TEST INFRASTRUCTURE ONLY.  CPU restatement of curcuma's native GFN-FF energy +
// gradient per geometry, used by the tests and by bench.py's CPU-baseline leg as the
// parity checker.  The product (libgfnff_b200.so) never links or calls this code.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

// term energies written by oracle_engrad (Hartree)
enum {
    ORC_BOND = 0, ORC_ANGLE, ORC_TORSION, ORC_INVERSION, ORC_STORSION, ORC_DISPERSION,
    ORC_BONDED_REP, ORC_NONBONDED_REP, ORC_COULOMB, ORC_HBOND, ORC_XBOND, ORC_ATM, ORC_BATM,
    ORC_SOLVATION, ORC_TOTAL, ORC_NTERMS
};

typedef struct oracle_handle oracle_handle;

// Runs the host setup (shared with the product) for n atoms, xyz in Angstrom.
// Returns NULL on failure; oracle_last_error() tells why.
oracle_handle* oracle_create(int n, const int* Z, const double* xyz_ang, int charge);
// The model of a parameter file written by the library (gfnff_write_parameters); NULL on failure.
oracle_handle* oracle_create_from_parameters(const char* path);
// set-up with a topology cache file (<geometry>.topo.json): Phase 1 from the file on a
// fingerprint match; oracle_topo_cache_hit reports whether it was used
oracle_handle* oracle_create_cached(int n, const int* Z, const double* xyz_ang, int charge, const char* topo_json);
int oracle_topo_cache_hit(oracle_handle* h);
// periodic cell (cell_ang[3*k + d]: component d of lattice vector k, Angstrom; NULL: none)
int oracle_set_cell(oracle_handle* h, const double* cell_ang);
void oracle_destroy(oracle_handle* h);
// ALPB implicit solvation for the following evaluations (curcuma's solvent names and
// aliases; "" or "none": gas phase).  Returns 0, or 1 for an unknown solvent.
int oracle_set_solvent(oracle_handle* h, const char* solvent);
const char* oracle_last_error(void);

// Energy + gradient at xyz (Angstrom).  terms[ORC_NTERMS]; grad N*3 Eh/bohr; q and cn
// (each N) may be NULL.  nthreads <= 0 uses all OpenMP threads.  Returns 0 on success.
int oracle_engrad(oracle_handle* h, const double* xyz_ang, double* terms, double* grad,
                  double* q, double* cn, int nthreads);

// Re-detect the HB/XB lists at xyz (Angstrom) with the setup charges, as curcuma does
// when the RMSD from the last detection exceeds 0.3 bohr.
int oracle_redetect_hbxb(oracle_handle* h, const double* xyz_ang);

// The topology refresh at xyz (Angstrom) that curcuma applies when an atom has moved more
// than 0.5 bohr along an axis since the last topology (the shared set-up's
// refresh_topology).  Returns 1 when the topology changed, 0 when not.
int oracle_refresh_topology(oracle_handle* h, const double* xyz_ang);

// Topology / list export for bit-exact comparisons.  kind selects the list:
//  0 bonds (i,j)  1 angles (i,j,k)  2 torsions (i,j,k,l)  3 inversions (i,j,k,l)
//  4 dispersion pairs (i,j)  5 nonbonded repulsion pairs (i,j)  6 hbonds (a,h,b,case)
//  7 xbonds (a,x,b)  8 hybridisation (per atom)  9 fragment ids  10 pi-fragment ids
//  11 bonded repulsion (i,j)  12 atm (i,j,k)  13 batm (i,j,k)
// Returns the record count; copies up to cap ints (count*width) into out when non-NULL.
long oracle_list(oracle_handle* h, int kind, int* out, long cap);
// Per-atom setup data: which = 0 qa (Phase-1 charges), 1 setup CN, 2 alpeeq, 3 gam,
// 4 chi_base, 5 cnf, 6 target charge of the atom's fragment.  Returns 0 on success.
int oracle_atom_data(oracle_handle* h, int which, double* out);
// Number of fragments
int oracle_nfrag(oracle_handle* h);
// Per-term set-up parameters as doubles (indices as doubles), for comparisons with the
// reference's fixture parameter lists: kind 0 bonds (i, j, fc, alpha, r0 at the set-up CN in
// bohr, shift, ff), 1 angles (i, j, k, fc, theta0 rad; j the centre), 2 torsions (i, j, k, l, V, n, phi0,
// primary flag), 3 inversions (i, j, k, l, fc, omega0, type).  Returns the record count;
// copies up to cap doubles into out when non-NULL.
long oracle_term_params(oracle_handle* h, int kind, double* out, long cap);

#ifdef __cplusplus
}
#endif
