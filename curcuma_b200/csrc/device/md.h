// Device-resident NVE velocity-Verlet loop around an Engine (see md.cu).
#pragma once

#include "engine.h"

namespace gfnff {

// nsteps of velocity Verlet with time step dt_fs (fs).  xyz_ang (N*3, Angstrom) and
// vel_ang_fs (N*3, Angstrom/fs) are host arrays, updated in place; mass_amu has N
// entries.  epot and ekin receive nsteps + 1 values (Hartree; entry 0 is the start).
// Returns the worst gfnff_status seen (the run stops at the first failing check, made
// every 100 steps).  Throws std::runtime_error on CUDA failure.
int md_nve(Engine& eng, int nsteps, double dt_fs, double* xyz_ang, double* vel_ang_fs, const double* mass_amu,
           double* epot, double* ekin, int* status);

}  // namespace gfnff
