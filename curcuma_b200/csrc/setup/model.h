// GFN-FF parameter model: everything the per-geometry energy + gradient needs, produced
// once by the host setup (topology, charges, term lists) and then cached on the device.
//
// The model mirrors curcuma's GFNFFParameterSet (ff_methods/gfnff_parameters.h:247-290)
// plus the per-atom EEQ / CN / D4 data that curcuma keeps in TopologyInfo and the
// D4ParameterGenerator.  All lengths are bohr, energies Hartree.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace gfnff {

constexpr int kMaxRef = 7;        // D4 reference states per element
constexpr int kNumFreq = 23;      // D4 imaginary-frequency grid points
constexpr double kAngToBohr = 1.0 / 0.529177210903;   // units.h:81-82 (CODATA 2018)
constexpr double kAngToBohrCN = 1.8897259886;         // cn_calculator.cpp:126
constexpr double kAatoau = 1.0 / 0.52917726;          // gfnff_par.h:276

// ---- term records (host layout; the device uses SoA copies) --------------------
struct BondTerm {           // ff_workspace_gfnff.cpp:104-182, forcefieldthread.h:111-134
    int i, j;
    double fc;              // prefactor k (negative), Eh
    double alpha;           // exponent
    double r0_base_i, r0_base_j, cnfak_i, cnfak_j, rabshift, ff;
    double r0_setup;        // r0 at the setup CN (reported, not used per step)
    int nr_hb = 0;          // number of HB acceptors modulating this X-H bond
    int hb_h = -1;          // the H atom of an X-H bond with nr_hb > 0
};
struct AngleTerm { int i, j, k; double fc, theta0; };                 // :187-280
struct TorsionTerm { int i, j, k, l; double V, n, phi0; int nci; };   // :282-487
struct InversionTerm { int i, j, k, l; double fc, omega0; int type; };// :489-609
struct STorsionTerm { int i, j, k, l; double erefhalf; };             // :611-653
struct RepPair { int i, j; double alpha, repab; };                    // :774-848
struct DispPair { int i, j; double c6, r4r2, r0sq, zetac6; };         // :715-772
struct HBTerm {                                                       // :938-1409
    int a, h, b, case_type;
    double bas_a, bas_b, aci_a, aci_b, q_h, q_a, q_b;
    int parent_c = -1;
    std::vector<int> nb_b, nb_c;
};
struct XBTerm { int a, x, b; double aci_x, q_x, q_b; };               // :1411-1524
struct ATMTriple { int i, j, k; double c6ij, c6ik, c6jk, scale; };    // :1526-1663
struct BATMTriple { int i, j, k; double zi, zj, zk; };                // :1665-1739
struct BondHB { int a, h; std::vector<int> b_atoms; };                // gfnff_method.cpp:3680-3712

struct SetupOptions {
    bool hbond = true, dispersion = true, repulsion = true, coulomb = true;
    int cell_list_min_atoms = 800;   // nb_cell_list_min_atoms (gfnff.h:240)
    double hb_accuracy = 0.1;        // gfnff.h:270
};

struct Model {
    int n = 0, nfrag = 0, charge = 0;
    std::vector<int> Z;
    std::vector<double> xyz_setup;    // bohr, row-major N x 3

    // ---- topology (setup) ----
    std::vector<std::vector<int>> adj;          // fat-scaled bond graph (getCachedBondList)
    std::vector<int> hyb, pi_frag, ring_size, frag;   // frag 0-based
    std::vector<double> cn_setup;               // CN with the 1600 bohr^2 threshold
    std::vector<double> qa;                     // Phase-1 topology charges
    std::vector<double> qfrag;                  // per-fragment target charge
    std::vector<int> bond_type;                 // per adjacency bond (i<j order)
    std::vector<std::pair<int, int>> topo_bonds;// getCachedBondList order

    // ---- per-atom EEQ / CN data (per-step inputs) ----
    std::vector<double> rcov_cn;    // 4/3 * Pyykko(A) * 1.8897259886
    std::vector<double> rcov_d3;    // covalent_rad_d3 (bohr, no 4/3)
    std::vector<double> rvdw;       // covalent_radii (A table used as HB r_vdw)
    std::vector<double> chi_base;   // -chi + dxi (-0.02 amide H)
    std::vector<double> cnf;        // cnf_eeq
    std::vector<double> gam;        // gam_eeq + dgam
    std::vector<double> alpeeq;     // (alpha + ff*qa)^2

    // ---- D4 data ----
    std::vector<int> present_Z;                 // distinct elements, first-seen order
    std::vector<int> slot;                      // per atom: index into present_Z
    std::vector<int> nref;                      // per atom
    std::vector<double> refcn;                  // per atom x kMaxRef
    std::vector<double> c6ref;                  // K x K x kMaxRef x kMaxRef
    std::vector<double> w_setup;                // per atom x kMaxRef (setup CN weights)
    std::vector<double> zeta;                   // per atom zeta(qa)
    std::vector<double> sqrt_zr4r2;             // per atom

    // ---- term lists ----
    std::vector<BondTerm> bonds;
    std::vector<AngleTerm> angles;
    std::vector<TorsionTerm> torsions;          // primary + extra (extra have nci=0,n=1)
    int n_primary_torsions = 0;
    std::vector<InversionTerm> inversions;
    std::vector<STorsionTerm> storsions;
    std::vector<RepPair> rep_bonded, rep_nonbonded;
    std::vector<DispPair> disp;
    std::vector<HBTerm> hbonds;
    std::vector<XBTerm> xbonds;
    std::vector<ATMTriple> atm;
    std::vector<BATMTriple> batm;
    std::vector<BondHB> bond_hb;
    double e0 = 0.0;
    bool nonbonded_rep_all_pairs = true;        // N < cell threshold: every non-bonded pair
    SetupOptions opt;
    // lists left to the device (a run-time choice of the set-up; not in the parameter file):
    // hbonds/bond_hb empty and the bonds' nr_hb/hb_h unset, or disp empty
    bool hb_on_device = false, disp_on_device = false;

    // Phase-1 by-products kept for the topology cache (<geometry>.topo.json); not in the
    // parameter file: electronegativity and hardness corrections, amide-H flags, the rings
    // (sorted atom sets), and whether the last topology came from a cache hit
    std::vector<double> dxi, dgam;
    std::vector<char> amide_h;
    std::vector<std::vector<int>> rings;
    bool topo_cache_hit = false;
};

// Per-atom inputs of the hydrogen-bond detection at one geometry (gfnff_method.cpp:7936-8100):
// basicity (geometry dependent for two-coordinate carbon) and acidity (amide-H scaling),
// the H-candidate flag (charge above the donor's threshold), the acceptor/donor flag (charge
// below 0.1, 0.3 beyond neon; no non-pi carbon) and the two squared-distance thresholds:
// A-B pairs within thr1, and the A-H-B triangle of a non-bonded H within thr2 (bohr^2).
struct HBAtoms {
    std::vector<double> bas, aci;
    std::vector<char> hcand, ok;
    double thr1 = 0.0, thr2 = 0.0;
};

// Which of the two largest set-up lists the host builds.  The D4 pair list is enumerated
// on the device by the engine; the HB terms of a single molecule can be too.
struct BuildLists {
    bool host_hb = true;
    bool host_disp = true;
};

// Runs the complete GFN-FF setup for one molecule (curcuma GFNFF::InitialiseMolecule,
// gfnff_method.cpp:733-848).  xyz_ang is row-major N x 3 in Angstrom.  topo_cache, when
// not null, names a <geometry>.topo.json whose Phase-1 data replace Phase 1 on a
// fingerprint match (Model::topo_cache_hit); the file is only read here.
// Throws std::runtime_error on invalid input.
Model build_model(int n, const int* Z, const double* xyz_ang, int charge,
                  const SetupOptions& opt = SetupOptions(), const BuildLists& lists = BuildLists(),
                  const char* topo_cache = nullptr);

// HB/XB lists re-detected at a new geometry with the setup (Phase-1) charges
// (gfnff_method.cpp:1597-1690); also rebuilds the bond <-> HB cross reference.
// With m.hb_on_device only the XB list is rebuilt (the engine detects the HB terms).
void redetect_hbxb(Model& m, const double* xyz_bohr);

// The topology refresh of curcuma's evaluation when an atom has moved more than 0.5 bohr
// along an axis since the last topology (gfnff_method.cpp:885-937, 1007-1032;
// QM/gfnff_gpu_method.cpp:408-425): the topology (bond graph, fragments, hybridisation,
// pi systems, Phase-1 charges) and the EEQ parameters derived from it are recomputed at
// xyz_bohr; the force-field term lists and their parameters stay those of the set-up, as in
// curcuma.  Returns true when anything the evaluation uses changed (the model is updated),
// false when the new topology is the old one (the model is left as it is).  topo_cache as
// in build_model: curcuma's refresh consults the same cache.
bool refresh_topology(Model& m, const double* xyz_bohr, const char* topo_cache = nullptr);

// HBAtoms of the model at xyz_bohr (N x 3, caller order)
HBAtoms hb_atom_data(Model& m, const double* xyz_bohr);

// Builds on the host the lists the set-up left to the device: the D4 pair list at the
// set-up geometry and the HB terms (with the bond cross reference) at hb_xyz_bohr.  Used
// before a parameter file is written.
void complete_host_lists(Model& m, const double* hb_xyz_bohr);

// Parameter file (the whole set-up result, binary, this library's own format): written by
// save_parameters, read back by load_parameters, which throws std::runtime_error on a
// missing, truncated or foreign file.
void save_parameters(const Model& m, const char* path);
Model load_parameters(const char* path);

// D4 helpers shared by setup, oracle and device upload.
void d4_weights(const Model& m, int atom, double cn, double* w, double* dw);

}  // namespace gfnff
