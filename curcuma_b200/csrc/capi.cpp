// C ABI of gfnff_b200 (include/gfnff_b200.h): host setup + device engine per handle.
#include "../../include/gfnff_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <algorithm>
#include <string>
#include <vector>

#include "device/engine.h"
#include "device/md.h"
#include "setup/model.h"
#include "setup/topo_cache.h"

using namespace gfnff;

struct gfnff_handle {
    gfnff_options opt{};
    std::unique_ptr<Engine> eng;
    Model model;
    std::vector<Model> batch;       // models of a batch handle (gfnff_setup_batch)
    int nmol = 0;                   // 0: single molecule
    int natoms = 0;                 // all atoms of the handle
    std::vector<double> pin_terms;  // 16 per molecule
    bool ready = false;
    std::string err;
    std::vector<double> hb_ref;    // bohr, geometry of the last HB/XB detection
    std::vector<double> topo_ref;  // bohr, geometry of the last topology
    std::vector<double> xb;        // bohr, the geometry of the current call (host scratch)
    std::string solvent;            // ALPB solvent ("" gas phase)
    AlpbModel solv;
    std::string topo_cache;         // <geometry>.topo.json ("" no topology cache)
    std::vector<double> cell_bohr;  // periodic cell, 9 doubles (empty: isolated system)
    double* pin_xyz = nullptr;      // pinned staging for host coordinates
    double* pin_grad = nullptr;
    double* pin_out = nullptr;      // terms + status + msd
    int* pin_status = nullptr;
    ~gfnff_handle()
    {
        if (pin_xyz) cudaFreeHost(pin_xyz);
        if (pin_grad) cudaFreeHost(pin_grad);
        if (pin_out) cudaFreeHost(pin_out);
        if (pin_status) cudaFreeHost(pin_status);
    }
};

static thread_local std::string g_static_err;

// host copies of at least this many doubles are split over the OpenMP threads (the
// single-molecule pass, which also reduces, from half of it)
static constexpr long kParallelCopy = 1l << 16;

static gfnff_status fail(gfnff_handle* h, gfnff_status s, const std::string& msg)
{
    if (h) h->err = msg;
    else g_static_err = msg;
    return s;
}

extern "C" {

void gfnff_default_options(gfnff_options* o)
{
    if (!o) return;
    o->precision = GFNFF_FP64;
    o->device = 0;
    o->hbond = 1;
    o->hb_rmsd_bohr = 0.3;
    o->gradient = GFNFF_GRADIENT_REFERENCE;
}

gfnff_status gfnff_create(const gfnff_options* opts, gfnff_handle** out)
{
    if (!out) return fail(nullptr, GFNFF_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto h = std::make_unique<gfnff_handle>();
    if (opts) h->opt = *opts;
    else gfnff_default_options(&h->opt);
    if (h->opt.precision != GFNFF_FP64 && h->opt.precision != GFNFF_MIXED)
        return fail(nullptr, GFNFF_INVALID_ARG, "unknown precision");
    if (h->opt.gradient != GFNFF_GRADIENT_REFERENCE && h->opt.gradient != GFNFF_GRADIENT_EXACT)
        return fail(nullptr, GFNFF_INVALID_ARG, "unknown gradient mode");
    try {
        EngineOptions eo;
        eo.precision = h->opt.precision;
        eo.device = h->opt.device;
        eo.exact_gradient = h->opt.gradient == GFNFF_GRADIENT_EXACT;
        h->eng = std::make_unique<Engine>(eo);
    } catch (const std::exception& e) {
        return fail(nullptr, GFNFF_CUDA_ERROR, e.what());
    }
    *out = h.release();
    return GFNFF_OK;
}

static gfnff_status finish_setup(gfnff_handle* h, int n);

gfnff_status gfnff_set_solvent(gfnff_handle* h, const char* solvent)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    const std::string s = solvent ? solvent : "";
    AlpbModel probe;
    if (!alpb_setup(probe, std::vector<int>{1}, s)) return fail(h, GFNFF_INVALID_ARG, "unknown solvent: " + s);
    h->solvent = (s == "none") ? "" : s;
    return GFNFF_OK;
}

gfnff_status gfnff_set_unit_cell(gfnff_handle* h, const double* cell_angstrom)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!cell_angstrom) {
        h->cell_bohr.clear();
        return GFNFF_OK;
    }
    if (h->opt.gradient == GFNFF_GRADIENT_EXACT)
        return fail(h, GFNFF_INVALID_ARG, "a periodic cell needs the reference gradient mode");
    std::vector<double> c(9);
    for (int k = 0; k < 9; ++k) {
        if (!std::isfinite(cell_angstrom[k])) return fail(h, GFNFF_INVALID_ARG, "non-finite cell");
        c[k] = cell_angstrom[k] * kAngToBohr;
    }
    const double det = c[0] * (c[4] * c[8] - c[7] * c[5]) - c[3] * (c[1] * c[8] - c[7] * c[2]) +
                       c[6] * (c[1] * c[5] - c[4] * c[2]);
    if (!(std::fabs(det) > 1e-6)) return fail(h, GFNFF_INVALID_ARG, "singular cell");
    h->cell_bohr = c;
    return GFNFF_OK;
}

gfnff_status gfnff_set_geometry_file(gfnff_handle* h, const char* geometry_file, int cache_topology)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    const std::string g = geometry_file ? geometry_file : "";
    h->topo_cache = (cache_topology && !g.empty()) ? topology_cache_path(g) : std::string();
    return GFNFF_OK;
}

int gfnff_topology_cache_hit(gfnff_handle* h)
{
    if (!h || !h->ready || h->nmol) return -1;
    return h->model.topo_cache_hit ? 1 : 0;
}

// curcuma writes the cache after every set-up and ignores a file it cannot open
// (gfnff_method.cpp:2941-2985)
static void write_cache_quietly(const std::string& path, const Model& m)
{
    if (path.empty()) return;
    try {
        write_topology_cache(path, m);
    } catch (const std::exception&) {
    }
}

gfnff_status gfnff_write_topology_cache(int n, const int* Z, const double* xyz, int charge, const char* geometry_file,
                                        int* cache_hit)
{
    if (n <= 0 || !Z || !xyz || !geometry_file || !*geometry_file)
        return fail(nullptr, GFNFF_INVALID_ARG, "invalid molecule or geometry file");
    try {
        const std::string path = topology_cache_path(geometry_file);
        Model m = build_model(n, Z, xyz, charge, SetupOptions(), BuildLists(), path.c_str());
        if (cache_hit) *cache_hit = m.topo_cache_hit ? 1 : 0;
        if (!write_topology_cache(path, m))
            return fail(nullptr, GFNFF_SETUP_FAILED, "Phase-1 charges failed the cache's write check");
    } catch (const std::exception& e) {
        return fail(nullptr, GFNFF_SETUP_FAILED, e.what());
    }
    return GFNFF_OK;
}

gfnff_status gfnff_setup(gfnff_handle* h, int n, const int* Z, const double* xyz, int charge)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (n <= 0 || !Z || !xyz) return fail(h, GFNFF_INVALID_ARG, "invalid molecule");
    h->ready = false;
    try {
        SetupOptions so;
        so.hbond = h->opt.hbond != 0;
        // the D4 pair list is enumerated by the engine; the HB terms of larger molecules are
        // detected on the device (GFNFF_HB_DEVICE=0|1 forces the host or the device)
        BuildLists L;
        L.host_disp = false;
        const char* hd = std::getenv("GFNFF_HB_DEVICE");
        L.host_hb = hd ? !std::strcmp(hd, "0") : n < 512;
        h->model = build_model(n, Z, xyz, charge, so, L, h->topo_cache.empty() ? nullptr : h->topo_cache.c_str());
        if (!alpb_setup(h->solv, h->model.Z, h->solvent)) return fail(h, GFNFF_INVALID_ARG, "unknown solvent");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_SETUP_FAILED, e.what());
    }
    const gfnff_status st = finish_setup(h, n);
    if (st == GFNFF_OK) write_cache_quietly(h->topo_cache, h->model);
    return st;
}

// upload of h->model and the per-handle host staging (gfnff_setup, gfnff_setup_from_parameters)
static gfnff_status finish_setup(gfnff_handle* h, int n)
{
    if (!h->cell_bohr.empty() && h->solv.on)
        return fail(h, GFNFF_INVALID_ARG, "ALPB solvation and a periodic cell exclude each other");
    try {
        h->eng->set_cell(h->cell_bohr.empty() ? nullptr : h->cell_bohr.data());
        h->eng->upload(h->model, h->solv.on ? &h->solv : nullptr);
        if (h->pin_xyz) cudaFreeHost(h->pin_xyz);
        if (h->pin_grad) cudaFreeHost(h->pin_grad);
        if (!h->pin_out && cudaMallocHost(&h->pin_out, 32 * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
        if (!h->pin_status && cudaMallocHost(&h->pin_status, sizeof(int)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
        if (cudaMallocHost(&h->pin_xyz, 3 * (size_t)n * sizeof(double)) != cudaSuccess ||
            cudaMallocHost(&h->pin_grad, 3 * (size_t)n * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    h->hb_ref = h->model.xyz_setup;
    h->topo_ref = h->model.xyz_setup;
    h->nmol = 0;
    h->natoms = n;
    h->batch.clear();
    h->ready = true;
    return GFNFF_OK;
}

gfnff_status gfnff_save_parameters(gfnff_handle* h, const char* path)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!path) return fail(h, GFNFF_INVALID_ARG, "NULL path");
    if (!h->ready || h->nmol) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    try {
        if (h->model.hb_on_device || h->model.disp_on_device) {   // the file holds every list
            Model full = h->model;
            complete_host_lists(full, h->hb_ref.data());
            save_parameters(full, path);
        } else {
            save_parameters(h->model, path);
        }
    } catch (const std::exception& e) {
        return fail(h, GFNFF_INVALID_ARG, e.what());
    }
    return GFNFF_OK;
}

gfnff_status gfnff_setup_from_parameters(gfnff_handle* h, const char* path, int natoms, const int* Z)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!path || natoms <= 0 || !Z) return fail(h, GFNFF_INVALID_ARG, "invalid path or molecule");
    h->ready = false;
    try {
        Model m = load_parameters(path);
        if (m.n != natoms || !std::equal(m.Z.begin(), m.Z.end(), Z))
            return fail(h, GFNFF_SETUP_FAILED, "parameter file is for another structure");
        h->model = std::move(m);
        if (!alpb_setup(h->solv, h->model.Z, h->solvent)) return fail(h, GFNFF_INVALID_ARG, "unknown solvent");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_SETUP_FAILED, e.what());
    }
    return finish_setup(h, h->model.n);
}

gfnff_status gfnff_write_parameters(int n, const int* Z, const double* xyz, int charge, int hbond, const char* path)
{
    if (n <= 0 || !Z || !xyz || !path) return fail(nullptr, GFNFF_INVALID_ARG, "invalid molecule or path");
    try {
        SetupOptions so;
        so.hbond = hbond != 0;
        save_parameters(build_model(n, Z, xyz, charge, so), path);
    } catch (const std::exception& e) {
        return fail(nullptr, GFNFF_SETUP_FAILED, e.what());
    }
    return GFNFF_OK;
}

gfnff_status gfnff_setup_batch(gfnff_handle* h, int nmol, const int* natoms, const int* Z, const double* xyz,
                               const int* charges)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (nmol <= 0 || !natoms || !Z || !xyz) return fail(h, GFNFF_INVALID_ARG, "invalid batch");
    if (!h->solvent.empty()) return fail(h, GFNFF_INVALID_ARG, "ALPB solvation: single-molecule handles only");
    if (!h->cell_bohr.empty()) return fail(h, GFNFF_INVALID_ARG, "a periodic cell: single-molecule handles only");
    std::vector<long> off(nmol + 1, 0);
    for (int m = 0; m < nmol; ++m) {
        if (natoms[m] <= 0) return fail(h, GFNFF_INVALID_ARG, "molecule without atoms");
        off[m + 1] = off[m] + natoms[m];
    }
    if (off[nmol] > (1l << 30)) return fail(h, GFNFF_INVALID_ARG, "batch too large");
    h->ready = false;
    std::vector<Model> models(nmol);
    std::vector<std::string> errs(nmol);
    SetupOptions so;
    so.hbond = h->opt.hbond != 0;
#pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < nmol; ++m) {
        try {
            BuildLists L;
            L.host_disp = false;   // enumerated by the engine
            models[m] = build_model(natoms[m], Z + off[m], xyz + 3 * off[m], charges ? charges[m] : 0, so, L);
        } catch (const std::exception& e) {
            errs[m] = e.what();
        }
    }
    for (int m = 0; m < nmol; ++m)
        if (!errs[m].empty()) return fail(h, GFNFF_SETUP_FAILED, "molecule " + std::to_string(m) + ": " + errs[m]);
    const int n = (int)off[nmol];
    try {
        std::vector<const Model*> ptr(nmol);
        for (int m = 0; m < nmol; ++m) ptr[m] = &models[m];
        h->eng->set_cell(nullptr);
        h->eng->upload_batch(ptr);
        if (h->pin_xyz) cudaFreeHost(h->pin_xyz);
        if (h->pin_grad) cudaFreeHost(h->pin_grad);
        h->pin_xyz = h->pin_grad = nullptr;
        if (!h->pin_out && cudaMallocHost(&h->pin_out, 32 * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
        if (!h->pin_status && cudaMallocHost(&h->pin_status, sizeof(int)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
        if (cudaMallocHost(&h->pin_xyz, 3 * (size_t)n * sizeof(double)) != cudaSuccess ||
            cudaMallocHost(&h->pin_grad, 3 * (size_t)n * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("cudaMallocHost failed");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    h->batch = std::move(models);
    h->nmol = nmol;
    h->natoms = n;
    h->pin_terms.assign(16 * (size_t)nmol, 0.0);
    h->ready = true;
    return GFNFF_OK;
}

gfnff_status gfnff_energy_and_gradient_batch(gfnff_handle* h, const double* xyz, double* energies, double* grad,
                                             int* status)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup_batch has not been called");
    if (h->nmol == 0) return fail(h, GFNFF_INVALID_ARG, "not a batch handle (use gfnff_energy_and_gradient)");
    if (!xyz || !energies) return fail(h, GFNFF_INVALID_ARG, "NULL coordinates or energies");
    const int n = h->natoms, nm = h->nmol;
    const long n3 = 3l * n;
    // the finiteness check and the pinned copy in one pass, split over the host threads for
    // large batches (a single thread copies ~10 GB/s: 0.1 ms for 50k atoms)
    int bad = 0;
    double* pin = h->pin_xyz;
#pragma omp parallel for reduction(| : bad) if (n3 >= kParallelCopy)
    for (long k = 0; k < n3; ++k) {
        const double v = xyz[k];
        if (!std::isfinite(v)) bad = 1;
        pin[k] = v;
    }
    if (bad) return fail(h, GFNFF_NONFINITE, "non-finite coordinate");
    std::vector<int> st(nm, 0);
    try {
        cudaStream_t s = (cudaStream_t)h->eng->stream();
        if (cudaMemcpyAsync(h->eng->d_xyz_scratch(), h->pin_xyz, 3 * (size_t)n * sizeof(double),
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            throw std::runtime_error("H2D copy failed");
        h->eng->enqueue(h->eng->d_xyz_scratch(), false);
        h->eng->fetch_batch(h->pin_terms.data(), h->pin_grad, st.data());
        // the CN neighbour list no longer covers this geometry: rebuild it around it (this
        // evaluation used the all-pairs CN kernels)
        if (h->eng->cn_list_stale()) h->eng->refresh_cn_list();
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    gfnff_status first = GFNFF_OK;
    for (int m = 0; m < nm; ++m) {
        energies[m] = st[m] == GFNFF_OK ? h->pin_terms[16 * (size_t)m + GFNFF_E_TOTAL] : 0.0;
        if (status) status[m] = st[m];
        if (st[m] != GFNFF_OK && first == GFNFF_OK) first = (gfnff_status)st[m];
    }
    if (grad) {
        const double* pg = h->pin_grad;
#pragma omp parallel for if (n3 >= kParallelCopy)
        for (long k = 0; k < n3; ++k) grad[k] = pg[k];
    }
    if (first != GFNFF_OK) return fail(h, first, "at least one molecule failed (see status)");
    return GFNFF_OK;
}

// curcuma's topology refresh (gfnff_method.cpp:885-937, 1007-1032): when an atom has moved
// more than 0.5 bohr along an axis since the last topology, the topology and its EEQ
// parameters are recomputed at xb (bohr).  Same fragments: the EEQ parameters are updated in
// place (the HB/XB lists stay, as in curcuma, until their own refresh); new fragments: the
// HB/XB lists are detected again at their reference geometry with the new topology (their
// terms carry neighbour lists of the bond graph, which the upload checks against the new
// one) and the engine takes the whole model again.
static constexpr double kTopoDispBohr = 0.5;

static void topology_refresh(gfnff_handle* h, const double* xb)
{
    const int nfrag0 = h->model.nfrag;
    const std::vector<int> frag0 = h->model.frag;
    const std::vector<double> qfrag0 = h->model.qfrag;
    if (refresh_topology(h->model, xb, h->topo_cache.empty() ? nullptr : h->topo_cache.c_str())) {
        if (h->model.nfrag == nfrag0 && h->model.frag == frag0 && h->model.qfrag == qfrag0) {
            h->eng->update_eeq_parameters(h->model);
        } else {
            if (h->opt.hbond) redetect_hbxb(h->model, h->hb_ref.data());
            h->eng->upload(h->model, h->solv.on ? &h->solv : nullptr);
            if (h->model.hb_on_device) h->eng->upload_hbxb(h->model, h->hb_ref.data());
            h->eng->set_hb_reference(h->hb_ref.data());
        }
    }
    h->topo_ref.assign(xb, xb + 3 * (size_t)h->model.n);
    h->eng->set_topo_reference(xb);
}

gfnff_status gfnff_energy_and_gradient(gfnff_handle* h, const double* xyz, double* energy, double* grad,
                                       double* terms)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    if (!xyz || !energy) return fail(h, GFNFF_INVALID_ARG, "NULL coordinates or energy");
    if (h->nmol) return fail(h, GFNFF_INVALID_ARG, "batch handle (use gfnff_energy_and_gradient_batch)");
    const int n = h->model.n;
    // one pass over the coordinates: the finiteness check, the copy into the pinned staging
    // buffer, the geometry in bohr and both refresh measures (the largest coordinate change
    // since the last topology, the summed squared displacement since the HB/XB detection)
    h->xb.resize(3 * (size_t)n);
    double* xb = h->xb.data();
    double dmax = 0.0, ss = 0.0;
    {
        const double* tr = h->topo_ref.data();
        const double* hr = h->hb_ref.data();
        double* pin = h->pin_xyz;
        const long n3 = 3l * n;
        int bad = 0;
#pragma omp parallel for reduction(max : dmax) reduction(+ : ss) reduction(| : bad) if (n3 >= kParallelCopy / 2)
        for (long k = 0; k < n3; ++k) {
            const double v = xyz[k];
            if (!std::isfinite(v)) bad = 1;
            pin[k] = v;
            const double b = v * kAngToBohr;
            xb[k] = b;
            dmax = std::max(dmax, std::fabs(b - tr[k]));
            const double d = b - hr[k];
            ss += d * d;
        }
        if (bad) return fail(h, GFNFF_NONFINITE, "non-finite coordinate");
    }
    try {
        // topology refresh on a 0.5 bohr displacement, then the HB/XB refresh when the RMSD-like
        // measure sqrt(sum d^2)/N exceeds the threshold (gfnff_method.cpp:2228-2259), both
        // before this evaluation
        if (dmax > kTopoDispBohr) topology_refresh(h, xb);
        if (h->opt.hbond && std::sqrt(ss) / (double)n > h->opt.hb_rmsd_bohr) {
            redetect_hbxb(h->model, xb);
            h->eng->upload_hbxb(h->model, xb);
            h->hb_ref.assign(xb, xb + 3 * (size_t)n);
        }
        cudaStream_t s = (cudaStream_t)h->eng->stream();
        if (cudaMemcpyAsync(h->eng->d_xyz_scratch(), h->pin_xyz, 3 * (size_t)n * sizeof(double),
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            throw std::runtime_error("H2D copy failed");
        h->eng->enqueue(h->eng->d_xyz_scratch(), false);
        h->eng->fetch(h->pin_out, h->pin_grad, h->pin_status, nullptr);
        // an indefinite reduced matrix moves to LU, a stalled iterative solve to the
        // direct one; either way this geometry is evaluated again
        const bool retry = (*h->pin_status == GFNFF_NOT_SPD && h->eng->switch_to_lu()) ||
                           (*h->pin_status == GFNFF_REFINE_NOT_CONVERGED && h->eng->switch_to_direct());
        if (retry) {
            h->eng->enqueue(h->eng->d_xyz_scratch(), false);
            h->eng->fetch(h->pin_out, h->pin_grad, h->pin_status, nullptr);
        }
        // the CN neighbour list no longer covers this geometry: rebuild it around it (this
        // evaluation used the all-pairs CN kernels)
        if (h->eng->cn_list_stale()) h->eng->refresh_cn_list();
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    const int st = *h->pin_status;
    *energy = h->pin_out[GFNFF_E_TOTAL];
    if (terms) std::memcpy(terms, h->pin_out, GFNFF_NTERMS * sizeof(double));
    if (grad) {
        const double* pg = h->pin_grad;
        const long n3 = 3l * n;
#pragma omp parallel for if (n3 >= kParallelCopy / 2)
        for (long k = 0; k < n3; ++k) grad[k] = pg[k];
    }
    if (st != GFNFF_OK) {
        *energy = 0.0;   // curcuma's convention: an energy of 0.0 signals an error
        const char* why = st == GFNFF_NOT_SPD                ? "EEQ matrix not positive definite"
                          : st == GFNFF_REFINE_NOT_CONVERGED ? "EEQ iterative solve did not converge"
                          : st == GFNFF_CUDA_ERROR           ? "device wait gave up in the EEQ solve"
                                                             : "non-finite energy or gradient";
        return fail(h, (gfnff_status)st, why);
    }
    return GFNFF_OK;
}

gfnff_status gfnff_energy_and_gradient_device(gfnff_handle* h, const double* d_xyz, double* d_energy,
                                              double* d_grad, int* d_status)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    if (!d_xyz) return fail(h, GFNFF_INVALID_ARG, "NULL coordinates");
    try {
        h->eng->enqueue(d_xyz, true, d_energy);
        cudaStream_t s = (cudaStream_t)h->eng->stream();
        const int n = h->natoms;
        if (d_grad &&
            cudaMemcpyAsync(d_grad, h->eng->d_grad(), 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            throw std::runtime_error("D2D copy failed");
        if (d_status && cudaMemcpyAsync(d_status, h->eng->d_status(), sizeof(int) * std::max(1, h->nmol),
                                        cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            throw std::runtime_error("D2D copy failed");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    return GFNFF_OK;
}

void* gfnff_stream(gfnff_handle* h) { return h && h->eng ? h->eng->stream() : nullptr; }

static gfnff_status copy_atoms(gfnff_handle* h, const double* dsrc, double* out)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    if (!out) return fail(h, GFNFF_INVALID_ARG, "NULL output");
    cudaStream_t s = (cudaStream_t)h->eng->stream();
    if (cudaMemcpyAsync(out, dsrc, (size_t)h->natoms * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail(h, GFNFF_CUDA_ERROR, "D2H copy failed");
    return GFNFF_OK;
}

gfnff_status gfnff_charges(gfnff_handle* h, double* q) { return copy_atoms(h, h ? h->eng->d_charges() : nullptr, q); }
gfnff_status gfnff_coordination_numbers(gfnff_handle* h, double* cn) { return copy_atoms(h, h ? h->eng->d_cn() : nullptr, cn); }

gfnff_status gfnff_get_topology(gfnff_handle* h, int kind, int* out, long cap, long* count)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    if (h->nmol && kind != 4) return fail(h, GFNFF_INVALID_ARG, "topology lists of batch handles: kind 4 only");
    const Model& m = h->model;
    std::vector<int> v;
    long cnt = 0;
    try {
        switch (kind) {
            case 0: for (auto& b : m.bonds) { v.push_back(b.i); v.push_back(b.j); } cnt = (long)m.bonds.size(); break;
            case 1: for (auto& a : m.angles) v.insert(v.end(), {a.i, a.j, a.k}); cnt = (long)m.angles.size(); break;
            case 2: for (auto& t : m.torsions) v.insert(v.end(), {t.i, t.j, t.k, t.l}); cnt = (long)m.torsions.size(); break;
            case 3: for (auto& t : m.inversions) v.insert(v.end(), {t.i, t.j, t.k, t.l}); cnt = (long)m.inversions.size(); break;
            case 4: v = h->eng->device_dispersion_pairs(); cnt = (long)v.size() / 2; break;
            case 5: for (auto& r : m.rep_nonbonded) { v.push_back(r.i); v.push_back(r.j); } cnt = (long)m.rep_nonbonded.size(); break;
            case 6:
                if (m.hb_on_device) {
                    v = h->eng->hb_terms();
                    cnt = (long)v.size() / 4;
                } else {
                    for (auto& t : m.hbonds) v.insert(v.end(), {t.a, t.h, t.b, t.case_type});
                    cnt = (long)m.hbonds.size();
                }
                break;
            case 7: for (auto& t : m.xbonds) v.insert(v.end(), {t.a, t.x, t.b}); cnt = (long)m.xbonds.size(); break;
            case 8: v = m.hyb; cnt = m.n; break;
            case 9: v = m.frag; cnt = m.n; break;
            case 10: v = m.pi_frag; cnt = m.n; break;
            case 11: for (auto& r : m.rep_bonded) { v.push_back(r.i); v.push_back(r.j); } cnt = (long)m.rep_bonded.size(); break;
            case 12: for (auto& t : m.atm) v.insert(v.end(), {t.i, t.j, t.k}); cnt = (long)m.atm.size(); break;
            case 13: for (auto& t : m.batm) v.insert(v.end(), {t.i, t.j, t.k}); cnt = (long)m.batm.size(); break;
            default: return fail(h, GFNFF_INVALID_ARG, "unknown topology kind");
        }
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    if (count) *count = cnt;
    if (out) std::memcpy(out, v.data(), std::min<long>((long)v.size(), cap) * sizeof(int));
    return GFNFF_OK;
}

gfnff_status gfnff_sizes(gfnff_handle* h, int* natoms, int* nfrag)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    int nf = h->model.nfrag;
    if (h->nmol) {
        nf = 0;
        for (const auto& m : h->batch) nf += m.nfrag;
    }
    if (natoms) *natoms = h->natoms;
    if (nfrag) *nfrag = nf;
    return GFNFF_OK;
}

gfnff_status gfnff_set_phase_timing(gfnff_handle* h, int on)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    try {
        h->eng->set_timing(on != 0);
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    return GFNFF_OK;
}

int gfnff_phase_times(gfnff_handle* h, double* ms, int cap)
{
    if (!h || !ms) return -1;
    try {
        auto v = h->eng->phase_ms();
        const int n = std::min<int>(cap, (int)v.size());
        for (int k = 0; k < n; ++k) ms[k] = v[k];
        return (int)v.size();
    } catch (const std::exception& e) {
        fail(h, GFNFF_CUDA_ERROR, e.what());
        return -1;
    }
}

gfnff_status gfnff_md_nve(gfnff_handle* h, int nsteps, double dt_fs, double* xyz, double* vel, const double* mass,
                          double* epot, double* ekin)
{
    if (!h) return fail(nullptr, GFNFF_INVALID_ARG, "handle is NULL");
    if (!h->ready) return fail(h, GFNFF_NOT_READY, "gfnff_setup has not been called");
    if (nsteps < 0 || !(dt_fs > 0.0) || !xyz || !vel || !mass || !epot || !ekin)
        return fail(h, GFNFF_INVALID_ARG, "invalid MD arguments");
    if (h->nmol) return fail(h, GFNFF_INVALID_ARG, "batch handle (MD runs on single-molecule handles)");
    const int n = h->natoms;
    for (int i = 0; i < n; ++i)
        if (!(mass[i] > 0.0)) return fail(h, GFNFF_INVALID_ARG, "non-positive mass");
    try {
        // the HB/XB lists follow the trajectory step by step, as curcuma's evaluation does
        // before every energy (gfnff_method.cpp:1597-1613): the device loop finds the
        // first step over the threshold and rolls back to it for the re-detection
        MdRefresh R;
        R.topo_disp_bohr = kTopoDispBohr;
        h->eng->set_topo_reference(h->topo_ref.data());
        if (h->opt.hbond) {
            R.hb_rmsd_bohr = h->opt.hb_rmsd_bohr;
            h->eng->set_hb_reference(h->hb_ref.data());
        }
        R.refresh = [h](const double* xb, int reasons) {
            if (reasons & 2) topology_refresh(h, xb);
            if ((reasons & 1) && h->opt.hbond) {
                redetect_hbxb(h->model, xb);
                h->eng->upload_hbxb(h->model, xb);
                h->eng->set_hb_reference(xb);
                h->hb_ref.assign(xb, xb + 3 * (size_t)h->model.n);
            }
        };
        int worst = 0;
        md_nve(*h->eng, nsteps, dt_fs, xyz, vel, mass, epot, ekin, &worst, &R);
        if (worst != 0) return fail(h, (gfnff_status)worst, "MD stopped: evaluation failed");
    } catch (const std::exception& e) {
        return fail(h, GFNFF_CUDA_ERROR, e.what());
    }
    return GFNFF_OK;
}

const char* gfnff_eeq_solver(gfnff_handle* h)
{
    if (!h || !h->ready) return "";
    return h->eng->solver_name();
}

const char* gfnff_pair_kernel(gfnff_handle* h)
{
    if (!h || !h->ready) return "";
    return h->eng->pair_kernel_name();
}

int gfnff_kernels_per_evaluation(gfnff_handle* h)
{
    if (!h || !h->ready) return -1;
    return h->eng->kernels_per_evaluation();
}

int gfnff_eeq_iterations(gfnff_handle* h)
{
    if (!h || !h->ready) return -1;
    try {
        return h->eng->eeq_iterations();
    } catch (const std::exception& e) {
        fail(h, GFNFF_CUDA_ERROR, e.what());
        return -1;
    }
}

int gfnff_eeq_fp64_products(gfnff_handle* h)
{
    if (!h || !h->ready) return -1;
    try {
        return h->eng->eeq_fp64_products();
    } catch (const std::exception& e) {
        fail(h, GFNFF_CUDA_ERROR, e.what());
        return -1;
    }
}

const char* gfnff_last_error(gfnff_handle* h) { return h ? h->err.c_str() : g_static_err.c_str(); }

gfnff_status gfnff_destroy(gfnff_handle* h)
{
    delete h;
    return GFNFF_OK;
}

}  // extern "C"
