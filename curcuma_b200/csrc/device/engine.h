// Device engine: the GFN-FF model cached in HBM and the per-geometry energy + gradient
// pipeline (host-side interface; kernels live in engine.cu).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../setup/model.h"

namespace gfnff {

struct EngineOptions {
    int precision = 0;      // 0 = FP64, 1 = mixed
    int device = 0;
};

class Engine {
public:
    explicit Engine(const EngineOptions& opt);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // uploads the model; throws std::runtime_error on CUDA failure
    void upload(const Model& m);
    // re-uploads the HB/XB lists and the bond<->HB cross reference of m
    void upload_hbxb(const Model& m);

    // Enqueues one energy+gradient evaluation.  xyz is N*3 doubles, device pointer,
    // in bohr when bohr=true else Angstrom.  Results stay on the device (see below).
    void enqueue(const double* d_xyz, bool bohr);

    // device result buffers of the last enqueue
    const double* d_terms() const;     // kNumTerms doubles
    const double* d_grad() const;      // N*3
    const double* d_charges() const;   // N
    const double* d_cn() const;        // N
    const int* d_status() const;       // 1 int (gfnff_status)
    const double* d_hb_msd() const;    // sum of squared displacements vs HB reference
    double* d_xyz_scratch();           // N*3 staging buffer for host coordinates

    void* stream() const;
    int natoms() const;
    void sync();
    // copies the last results to the host
    void fetch(double* terms, double* grad, int* status, double* hb_msd);
    // device-enumerated dispersion pair list (i<j) at the setup geometry
    std::vector<int> device_dispersion_pairs();
    // sets the HB reference geometry (bohr, host) for the refresh test
    void set_hb_reference(const double* xyz_bohr);
    // switches the EEQ solve to pivoted LU (after a NOT_SPD status); false if already
    bool switch_to_lu();
    // per-phase CUDA-event timing of enqueue(); phase_ms returns the milliseconds of the
    // last evaluation per phase (order of kPhaseNames) after the stream has finished
    void set_timing(bool on);
    std::vector<double> phase_ms();
    static const char* const kPhaseNames[];
    static constexpr int kNumPhases = 12;

    static constexpr int kNumTerms = 14;

private:
    struct Impl;
    std::unique_ptr<Impl> p_;
};

}  // namespace gfnff
