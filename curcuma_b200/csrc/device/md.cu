// NVE molecular dynamics on the device: velocity Verlet around the engine's energy +
// gradient step (curcuma SimpleMD, capabilities/simplemd.cpp:2580-2674, restated for a
// device-resident loop).  Positions, velocities, gradient and the energy traces stay in
// HBM for the whole run; every step is a kick/drift kernel, the engine's evaluation (the
// coordinate gather plus the replayed step graph) and a kick kernel that also sums the
// kinetic energy.  Units inside: bohr, atomic time units, electron masses, Hartree.
#include "md.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

namespace gfnff {
namespace {

constexpr double kFsToAtu = 41.341373335;         // 1 fs in atomic time units
constexpr double kAmuToMe = 1822.888486209;       // 1 amu in electron masses
constexpr double kAngToBohrMd = 1.0 / 0.529177210903;

#define MDCK(x)                                                                                       \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA (md): ") + cudaGetErrorString(e_)); \
    } while (0)

// Per-run device record: [0] first step whose evaluation should have followed a refresh
// (-1: none), [1] first step whose evaluation failed (-1: none), [2] its status, [3] the
// refreshes due at step [0] (1 HB/XB lists, 2 topology).
struct MdFlags {
    int* rec;
    const double* msd;      // the engine's [0] squared displacement sum vs the HB reference,
                            // [1] largest coordinate change vs the topology reference
    const int* eval_st;     // the engine's status of the last evaluation
    double thr;             // HB/XB refresh threshold (bohr); <= 0 disables it
    double tthr;            // topology refresh threshold (bohr); <= 0 disables it
    int natoms;
    double *xs, *vs;        // state before the recorded step's evaluation
    __device__ int refresh_due() const
    {
        if (rec[0] >= 0) return 0;
        int r = 0;
        if (thr > 0.0 && sqrt(msd[0]) / (double)natoms > thr) r |= 1;
        if (tthr > 0.0 && msd[1] > tthr) r |= 2;
        return r;
    }
    __device__ void mark(int t) const
    {
        const int r = refresh_due();
        if (r) {
            rec[0] = t;
            rec[3] = r;
        }
    }
};

// v += -dt/2 g / m ; x += dt v.  Thread 0 first closes the record of the previous step
// tprev (whose measure is still in msd; the next evaluation resets it).
__global__ void k_kick_drift(int n3, double dt, const double* __restrict__ invm, const double* __restrict__ g,
                             double* v, double* x, MdFlags F, int tprev)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k == 0) F.mark(tprev);
    if (k >= n3) return;
    const double vk = v[k] - 0.5 * dt * g[k] * invm[k / 3];
    v[k] = vk;
    x[k] += dt * vk;
}

// after step t's evaluation: keep (x, v) if the step is due for a refresh, note a failed
// evaluation, then v += -dt/2 g / m and ekin += sum m v^2 / 2
__global__ void k_kick_ekin(int n3, double dt, const double* __restrict__ invm, const double* __restrict__ g,
                            double* v, const double* __restrict__ x, double* ekin, MdFlags F, int t)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool snap = F.refresh_due() != 0;   // rec[0] is written only by later kernels
    if (k == 0 && *F.eval_st != 0 && F.rec[1] < 0) {
        F.rec[1] = t;
        F.rec[2] = *F.eval_st;
    }
    double e = 0.0;
    if (k < n3) {
        const double v0 = v[k];
        if (snap) {
            F.xs[k] = x[k];
            F.vs[k] = v0;
        }
        const double vk = v0 - 0.5 * dt * g[k] * invm[k / 3];
        v[k] = vk;
        e = 0.5 * vk * vk / invm[k / 3];
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = e;
    __syncthreads();
    if (w == 0) {
        e = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
        if (lane == 0 && e != 0.0) atomicAdd(ekin, e);
    }
}

// the record of the chunk's last step t
__global__ void k_md_close(MdFlags F, int t) { F.mark(t); }

__global__ void k_md_reset(int* rec)
{
    rec[0] = -1;
    rec[1] = -1;
    rec[2] = 0;
    rec[3] = 0;
}

template <class T>
struct Dev {
    T* p = nullptr;
    explicit Dev(size_t n)
    {
        MDCK(cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)));
    }
    ~Dev() { cudaFree(p); }
    Dev(const Dev&) = delete;
    Dev& operator=(const Dev&) = delete;
};

}  // namespace

int md_nve(Engine& eng, int nsteps, double dt_fs, double* xyz_ang, double* vel_ang_fs, const double* mass_amu,
           double* epot, double* ekin, int* status, const MdRefresh* refresh)
{
    const int n = eng.natoms(), n3 = 3 * n;
    cudaStream_t s = (cudaStream_t)eng.stream();
    const double dt = dt_fs * kFsToAtu;
    const double vconv = kAngToBohrMd / kFsToAtu;   // A/fs -> bohr/atu
    const bool hb = refresh && refresh->refresh && (refresh->hb_rmsd_bohr > 0.0 || refresh->topo_disp_bohr > 0.0);
    std::vector<double> hx(n3), hv(n3), him(n);
    for (int k = 0; k < n3; ++k) {
        hx[k] = xyz_ang[k] * kAngToBohrMd;
        hv[k] = vel_ang_fs[k] * vconv;
    }
    for (int i = 0; i < n; ++i) him[i] = 1.0 / (mass_amu[i] * kAmuToMe);
    Dev<double> x(n3), v(n3), invm(n), ep(nsteps + 1), ek(nsteps + 1), xs(hb ? n3 : 1), vs(hb ? n3 : 1);
    Dev<int> rec(4);
    MDCK(cudaMemcpyAsync(x.p, hx.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemcpyAsync(v.p, hv.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemcpyAsync(invm.p, him.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemsetAsync(ep.p, 0, (nsteps + 1) * sizeof(double), s));
    MDCK(cudaMemsetAsync(ek.p, 0, (nsteps + 1) * sizeof(double), s));
    // the engine's buffers may be reallocated by a refresh (a new topology): re-read them after one
    auto flags = [&]() {
        return MdFlags{rec.p, eng.d_hb_msd(), eng.d_status(), hb ? refresh->hb_rmsd_bohr : 0.0,
                       hb ? refresh->topo_disp_bohr : 0.0, n, xs.p, vs.p};
    };
    MdFlags F = flags();
    const int B = 256, G = (n3 + B - 1) / B;
    int h_rec[4];
    int worst = 0, last_good = nsteps, resumed_at = -1;
    int t = 0;
    bool fresh = true;   // step t starts from a recorded state: no drift before its evaluation
    k_md_reset<<<1, 1, 0, s>>>(rec.p);
    while (t <= nsteps) {
        // chunks of up to 100 evaluations; the host reads the record once per chunk
        const int end = std::min(t + 99, nsteps);
        for (int u = t; u <= end; ++u) {
            if (!(u == t && fresh)) k_kick_drift<<<G, B, 0, s>>>(n3, dt, invm.p, eng.d_grad(), v.p, x.p, F, u - 1);
            eng.enqueue(x.p, true, ep.p + u);
            k_kick_ekin<<<G, B, 0, s>>>(n3, u == 0 ? 0.0 : dt, invm.p, eng.d_grad(), v.p, x.p, ek.p + u, F, u);
        }
        k_md_close<<<1, 1, 0, s>>>(F, end);
        MDCK(cudaGetLastError());
        MDCK(cudaMemcpyAsync(h_rec, rec.p, sizeof(h_rec), cudaMemcpyDeviceToHost, s));
        MDCK(cudaStreamSynchronize(s));
        const int due = h_rec[0], failed = h_rec[1];
        if (failed >= 0 && (due < 0 || failed < due)) {
            worst = h_rec[2];
            last_good = failed;
            break;
        }
        if (due >= 0) {
            // roll back to the state before step `due`, refresh the lists there, redo it
            if (due == resumed_at) throw std::runtime_error("md: HB/XB refresh did not reset the reference geometry");
            MDCK(cudaMemcpyAsync(x.p, xs.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
            MDCK(cudaMemcpyAsync(v.p, vs.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
            MDCK(cudaMemcpyAsync(hx.data(), xs.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
            MDCK(cudaMemsetAsync(ek.p + due, 0, (nsteps + 1 - due) * sizeof(double), s));
            k_md_reset<<<1, 1, 0, s>>>(rec.p);
            MDCK(cudaStreamSynchronize(s));
            refresh->refresh(hx.data(), h_rec[3]);
            F = flags();
            t = due;
            fresh = true;
            resumed_at = due;
            continue;
        }
        if (end < nsteps && eng.cn_list_stale(true)) eng.refresh_cn_list();
        t = end + 1;
        fresh = false;
    }
    MDCK(cudaMemcpyAsync(hx.data(), x.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(hv.data(), v.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(epot, ep.p, (nsteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(ekin, ek.p, (nsteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaStreamSynchronize(s));
    for (int u = last_good + 1; u <= nsteps; ++u) epot[u] = ekin[u] = 0.0;
    for (int k = 0; k < n3; ++k) {
        xyz_ang[k] = hx[k] / kAngToBohrMd;
        vel_ang_fs[k] = hv[k] / vconv;
    }
    if (status) *status = worst;
    return worst;
}

}  // namespace gfnff
