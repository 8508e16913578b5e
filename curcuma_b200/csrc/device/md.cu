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

// v += -dt/2 g / m ; x += dt v
__global__ void k_kick_drift(int n3, double dt, const double* __restrict__ invm, const double* __restrict__ g,
                             double* v, double* x)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    const double vk = v[k] - 0.5 * dt * g[k] * invm[k / 3];
    v[k] = vk;
    x[k] += dt * vk;
}

// v += -dt/2 g / m and ekin += sum m v^2 / 2
__global__ void k_kick_ekin(int n3, double dt, const double* __restrict__ invm, const double* __restrict__ g,
                            double* v, double* ekin)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (k < n3) {
        const double vk = v[k] - 0.5 * dt * g[k] * invm[k / 3];
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
           double* epot, double* ekin, int* status)
{
    const int n = eng.natoms(), n3 = 3 * n;
    cudaStream_t s = (cudaStream_t)eng.stream();
    const double dt = dt_fs * kFsToAtu;
    const double vconv = kAngToBohrMd / kFsToAtu;   // A/fs -> bohr/atu
    std::vector<double> hx(n3), hv(n3), him(n);
    for (int k = 0; k < n3; ++k) {
        hx[k] = xyz_ang[k] * kAngToBohrMd;
        hv[k] = vel_ang_fs[k] * vconv;
    }
    for (int i = 0; i < n; ++i) him[i] = 1.0 / (mass_amu[i] * kAmuToMe);
    Dev<double> x(n3), v(n3), invm(n), ep(nsteps + 1), ek(nsteps + 1);
    MDCK(cudaMemcpyAsync(x.p, hx.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemcpyAsync(v.p, hv.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemcpyAsync(invm.p, him.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    MDCK(cudaMemsetAsync(ek.p, 0, (nsteps + 1) * sizeof(double), s));
    const int B = 256, G = (n3 + B - 1) / B;
    // step 0: forces at the start geometry and the initial kinetic energy
    eng.enqueue(x.p, true, ep.p);
    k_kick_ekin<<<G, B, 0, s>>>(n3, 0.0, invm.p, eng.d_grad(), v.p, ek.p);
    int worst = 0;
    for (int t = 1; t <= nsteps; ++t) {
        k_kick_drift<<<G, B, 0, s>>>(n3, dt, invm.p, eng.d_grad(), v.p, x.p);
        eng.enqueue(x.p, true, ep.p + t);
        k_kick_ekin<<<G, B, 0, s>>>(n3, dt, invm.p, eng.d_grad(), v.p, ek.p + t);
        if (t % 100 == 0 || t == nsteps) {   // status check without stalling every step
            int h = 0;
            MDCK(cudaMemcpyAsync(&h, eng.d_status(), sizeof(int), cudaMemcpyDeviceToHost, s));
            MDCK(cudaStreamSynchronize(s));
            worst = std::max(worst, h);
            if (h != 0) break;
        }
    }
    MDCK(cudaGetLastError());
    MDCK(cudaMemcpyAsync(hx.data(), x.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(hv.data(), v.p, n3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(epot, ep.p, (nsteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaMemcpyAsync(ekin, ek.p, (nsteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    MDCK(cudaStreamSynchronize(s));
    for (int k = 0; k < n3; ++k) {
        xyz_ang[k] = hx[k] / kAngToBohrMd;
        vel_ang_fs[k] = hv[k] / vconv;
    }
    if (status) *status = worst;
    return worst;
}

}  // namespace gfnff
