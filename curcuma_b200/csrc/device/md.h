// Device-resident NVE velocity-Verlet loop around an Engine (see md.cu).
#pragma once

#include <functional>

#include "engine.h"

namespace gfnff {

// Per-step refreshes inside the device loop.  Before each evaluation curcuma re-detects the
// hydrogen- and halogen-bond lists when sqrt(sum (x - x_ref)^2) / N exceeds hb_rmsd_bohr
// (gfnff_method.cpp:1597-1613, 2228-2259), and recomputes the topology when an atom has moved
// more than topo_disp_bohr along an axis since the last topology (gfnff_method.cpp:1007-1032,
// QM/gfnff_gpu_method.cpp:408-425).  The device loop evaluates both measures at every step; at
// the first step t that exceeds one, the state before the step's evaluation is recorded, and
// at the end of the 100-step chunk the run is rolled back to it, refresh(x_t, reasons) is
// called (bohr, caller order; reasons: 1 the HB lists, 2 the topology; it must update the
// engine and its reference geometries) and step t is evaluated again.
struct MdRefresh {
    double hb_rmsd_bohr = 0.0;                              // <= 0: no HB refresh
    double topo_disp_bohr = 0.0;                            // <= 0: no topology refresh
    std::function<void(const double* xyz_bohr, int reasons)> refresh;
};

// nsteps of velocity Verlet with time step dt_fs (fs).  xyz_ang (N*3, Angstrom) and
// vel_ang_fs (N*3, Angstrom/fs) are host arrays, updated in place; mass_amu has N
// entries.  epot and ekin receive nsteps + 1 values (Hartree; entry 0 is the start).
// Every evaluation's status is kept on the device; the run stops at the end of the
// 100-step chunk in which the first evaluation failed, and returns that gfnff_status
// (the traces after the failing step are zero).  Between chunks a CN neighbour list
// that went stale is rebuilt.  Throws std::runtime_error on CUDA failure.
int md_nve(Engine& eng, int nsteps, double dt_fs, double* xyz_ang, double* vel_ang_fs, const double* mass_amu,
           double* epot, double* ekin, int* status, const MdRefresh* refresh = nullptr);

}  // namespace gfnff
