// Set-up of the ALPB implicit-solvation model for GFN-FF (analytical linearised
// Poisson-Boltzmann; Ehlert, Stahn, Spicher, Grimme, J. Chem. Theory Comput. 2021, 17, 4250):
// solvent parameters, per-atom radii and surface data, the model constants and the
// 230-point Lebedev-Laikov sphere grid.  Restates curcuma's ALPBSolvation::init,
// loadSolventParameters and setupRadii (ff_methods/alpb_solvation.cpp:196-396) and the
// constants of ff_methods/alpb_parameters.h:18-56.  The per-geometry part (Born radii,
// surface areas, Born matrix, energy and gradient) is evaluated by the device kernels and,
// independently, by the CPU oracle.
#pragma once

#include <string>
#include <vector>

namespace gfnff {

// model constants (alpb_parameters.h:21-56); lengths in bohr, energies in Hartree
namespace alpb {
constexpr double kAuToAng = 0.52917726;               // the model's own bohr (vdwrad, probe)
constexpr double kAngToAu = 1.0 / kAuToAng;
constexpr double kKcalToAu = 1.0 / 627.50947428;
constexpr double kPi = 3.1415926535897932384626433832795029;
constexpr double kMolCm3ToAu = 8.92388e-2;
constexpr double kWSmooth = 0.3 * kAngToAu;            // SASA switching half-width
constexpr double kAh0 = 0.5;
constexpr double kAh1 = 3.0 / (4.0 * kWSmooth);
constexpr double kAh3 = -1.0 / (4.0 * kWSmooth * kWSmooth * kWSmooth);
constexpr double kSurfaceTension = 1.0e-5;
constexpr double kLrCut = 35.0 * kAngToAu;             // Born-radius neighbour cut
constexpr double kObcAlpha = 1.0, kObcBeta = 0.8, kObcGamma = 4.85;
constexpr double kZetaP16 = 1.028, kZetaP16o16 = kZetaP16 / 16.0;
constexpr double kAlpbFactor = 0.571412;
constexpr double kTolSesp = 1.0e-6;                    // grid points below count as buried
constexpr double kROffset = 2.0 * kAngToAu;
constexpr int kNang = 230;
}  // namespace alpb

struct AlpbModel {
    bool on = false;
    std::string solvent;
    double epsv = 0.0, keps = 0.0, alpbet = 0.0, born_scale = 0.0, born_offset = 0.0, probe = 0.0;
    double gshift = 0.0;   // free-energy shift of the gsolv reference state
    double srcut = 0.0;    // SASA neighbour cut
    bool lhb = false;      // any atom with a hydrogen-bond strength
    // per atom
    std::vector<double> vdwr, rho, svdw, vdwsa, trj2_lo, trj2_hi, wrp, gamsasa, hbmag;
    // Lebedev grid: unit vectors (x, y, z per point) and weights
    std::vector<double> grid, weight;
};

// Fills m for the atoms Z and the solvent name (case-insensitive, curcuma's names and
// aliases).  An empty name or "none" switches the model off.  Returns false for an unknown
// solvent.
bool alpb_setup(AlpbModel& m, const std::vector<int>& Z, const std::string& solvent);

// the 230-point Lebedev-Laikov grid: 3 * 230 unit-vector components and 230 weights
void lebedev230(std::vector<double>& xyz, std::vector<double>& w);

}  // namespace gfnff
