// Device engine: the GFN-FF model of one molecule or of a batch of independent molecules
// cached in HBM, and the per-geometry energy + gradient pipeline (host-side interface;
// kernels live in engine.cu and the k_*.cuh files it includes).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../setup/alpb.h"
#include "../setup/model.h"

namespace gfnff {

struct EngineOptions {
    int precision = 0;      // 0 = FP64, 1 = mixed
    int device = 0;
    bool exact_gradient = false;   // derivative of the energy instead of curcuma's gradient
};

class Engine {
public:
    explicit Engine(const EngineOptions& opt);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Uploads one model (upload) or a batch of independent molecules (upload_batch; the
    // molecules do not interact, their atoms are concatenated in the given order).
    // Throws std::runtime_error on CUDA failure.
    // solv: ALPB implicit solvation of a single molecule (null or off: gas phase)
    void upload(const Model& m, const AlpbModel* solv = nullptr);
    void upload_batch(const std::vector<const Model*>& mols, const AlpbModel* solv = nullptr);
    // re-uploads the HB/XB lists and the bond<->HB cross reference (single model)
    // HB/XB lists of a single-molecule engine: the model's host lists, or, with
    // m.hb_on_device, the HB terms detected on the device at hb_xyz_bohr (caller order;
    // nullptr: the set-up geometry) and the model's XB list
    void upload_hbxb(const Model& m, const double* hb_xyz_bohr = nullptr);
    // the device-detected HB terms (A, H, B, case; caller order, detection order) and the
    // number of HB terms evaluated
    std::vector<int> hb_terms() const;
    long long hb_count() const;

    // Enqueues one energy+gradient evaluation.  xyz is N*3 doubles (all atoms of the
    // batch in upload order), device pointer, in bohr when bohr=true else Angstrom.
    // Results stay on the device (below), in the caller's atom order.
    // d_energies (optional, device): total energy of every molecule (nmol doubles).
    void enqueue(const double* d_xyz, bool bohr, double* d_energies = nullptr);

    // device result buffers of the last enqueue
    const double* d_terms() const;     // 16 doubles per molecule (kNumTerms used)
    const double* d_grad() const;      // N*3
    const double* d_charges() const;   // N
    const double* d_cn() const;        // N
    const int* d_status() const;       // 1 int (gfnff_status) per molecule
    const double* d_hb_msd() const;    // [0] sum of squared displacements vs the HB reference,
                                       // [1] largest |coordinate change| vs the topology reference
    double* d_xyz_scratch();           // N*3 staging buffer for host coordinates

    void* stream() const;
    int natoms() const;
    int nmol() const;
    void sync();
    // copies the last results to the host (molecule 0's terms and status)
    void fetch(double* terms, double* grad, int* status, double* hb_msd);
    // every molecule's 16 term slots, status per molecule, the whole gradient
    void fetch_batch(double* terms16, double* grad, int* status);
    // device-enumerated dispersion pair list (i<j, caller indices) at the setup geometry
    std::vector<int> device_dispersion_pairs();
    // sets the HB reference geometry (bohr, host, caller order) for the refresh test
    void set_hb_reference(const double* xyz_bohr);
    // sets the geometry of the last topology (bohr, host, caller order): d_hb_msd()[1] of an
    // evaluation holds the largest coordinate change since it
    void set_topo_reference(const double* xyz_bohr);
    // periodic cell for the next upload (single molecules): the lattice vectors a, b, c as
    // the columns of a 3x3 matrix, cell_bohr[3*col + row] (bohr); nullptr: isolated system.
    // Throws std::runtime_error for a singular cell.
    void set_cell(const double* cell_bohr);
    // EEQ parameters (chi, cnf, gamma, alpha, Phase-1 charges) of a refreshed topology of the
    // same molecule with the same fragments, in place
    void update_eeq_parameters(const Model& m);
    // the CN neighbour list no longer covers the geometry of the last evaluation (its
    // evaluations fell back to the all-pairs CN kernels); refresh_cn_list rebuilds it
    // around that geometry
    // (read_now: read the device flag; otherwise the value fetched with the last results)
    bool cn_list_stale(bool read_now = false);
    void refresh_cn_list();
    // switches the EEQ solve to pivoted LU (after a NOT_SPD status); false if already
    bool switch_to_lu();
    // switches an iterative EEQ solve to the direct one (after REFINE_NOT_CONVERGED)
    bool switch_to_direct();
    // EEQ solver in use: "library", "tiled", "pcg", "lu" or "batched"
    const char* solver_name() const;
    // Coulomb + D4 pair kernel variant picked by the set-up autotuner: "sym32", "sym64",
    // "sym64_occ10" or "rows"
    const char* pair_kernel_name() const;
    // iterations of the last iterative EEQ solve (0 for direct solvers)
    int eeq_iterations();
    // k_pcg_ir: FP64 products with the reduced matrix in the last solve; -1 otherwise
    int eeq_fp64_products();
    // kernels of this library per evaluation while the step replays as a graph (-1 before
    // the first capture or with direct launches)
    int kernels_per_evaluation() const;
    // per-phase CUDA-event timing of enqueue(); phase_ms returns the milliseconds of the
    // last evaluation per phase (order of kPhaseNames) after the stream has finished
    void set_timing(bool on);
    std::vector<double> phase_ms();
    static const char* const kPhaseNames[];
    static constexpr int kNumPhases = 12;

    static constexpr int kNumTerms = 15;

private:
    void tune_pairs(const std::vector<const Model*>& mols);
    void launch_positions(const double* d_xyz, bool bohr);
    void launch_body();
    struct Impl;
    std::unique_ptr<Impl> p_;
};

}  // namespace gfnff
