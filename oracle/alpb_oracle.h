// TEST INFRASTRUCTURE ONLY.  CPU restatement of curcuma's ALPB implicit solvation per
// geometry (ff_methods/alpb_solvation.cpp), the oracle's checker of the device kernels.
#pragma once

#include <vector>

#include "../curcuma_b200/csrc/setup/alpb.h"

namespace gfnff {

// per-geometry state: Born radii and d brad / d psi, surface areas, HB weights, shape
struct AlpbGeom {
    std::vector<double> psi, brad, dpsi, sasa, hbw, dhbdw;
    double adet = 0.0, gsasa = 0.0;
};

// Born radii, surface areas, HB weights and shape at x (bohr, N x 3); when Aeeq is non-null
// adds the Born matrix B into the EEQ matrix (n x n, row-major, both triangles)
void alpb_prepare(const AlpbModel& A, const double* x, int n, AlpbGeom& g, double* Aeeq);

// solvation free energy 1/2 q^T B q + G_sasa + G_shift for the charges q, and its
// gradient at fixed charges added into grad (N x 3)
double alpb_energy_gradient(const AlpbModel& A, const double* x, int n, const AlpbGeom& g, const double* q,
                            double* grad);

}  // namespace gfnff
