// Allocation-free EEQ charge solve.
//
// Some callers cannot allocate device memory at all: code that runs inside another
// framework's memory pool or arena, embedded or real-time loops that forbid
// allocations after start-up, and drivers that must not grow the process footprint
// after initialisation.  gfnff_eeq_charges_noalloc serves them: the caller passes every
// input and output buffer, and all intermediate storage (the dense EEQ matrix, its
// reduced form and the solve vectors) lives in one file-scope device array of fixed
// size.  The function calls no cudaMalloc, cudaFree or allocating library routine.
//
// The arithmetic is the engine's EEQ step (eeq_solver.cpp:3201-3700 of the reference):
// A_ij = erf(r_ij/sqrt(a_i+a_j))/r_ij, A_ii = gam_i + sqrt(2/pi)/sqrt(a_i),
// x_i = chi_i + cnf_i*sqrt(CN_i), one total-charge constraint per fragment, eliminated in
// the null space (q = q0 + B y, B the per-fragment difference basis), and the reduced
// system solved by a Cholesky factorisation run by one thread block.
#include <cuda_runtime.h>

#include <mutex>

#include "../../../include/gfnff_b200.h"

namespace {

constexpr int kMaxAtoms = GFNFF_NOALLOC_MAX_ATOMS;
constexpr int kThreads = 1024;
// doubles: A (n*n) + M (n*n) + pos (4n) + r, b, q0 (3n); ints: anchor, a2r, r2a, count (4n)
constexpr size_t kDoubles = 2ull * kMaxAtoms * kMaxAtoms + 7ull * kMaxAtoms;
constexpr size_t kInts = 4ull * kMaxAtoms + 4;

// Shared by every call on a device and kept between calls (every call rewrites what
// it reads, so nothing carries over).  Calls that overlap on the GPU race on it.
static __device__ __align__(256) double g_noalloc_scratch[kDoubles + kInts / 2 + 1];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

struct Scratch {
    double *A, *M, *pos, *r, *b, *q0;
    int *anchor, *a2r, *r2a, *meta;   // meta[0] = nred, meta[1] = failure flag
};

Scratch carve(double* base, int n)
{
    Scratch s;
    s.A = base;
    s.M = s.A + (size_t)n * n;
    s.pos = s.M + (size_t)n * n;
    s.r = s.pos + 4 * (size_t)n;
    s.b = s.r + n;
    s.q0 = s.b + n;
    int* ip = reinterpret_cast<int*>(s.q0 + n);
    s.anchor = ip;
    s.a2r = ip + n;
    s.r2a = ip + 2 * n;
    s.meta = ip + 4 * n;
    return s;
}

// Failure codes in meta[1]: every kernel after k_na_check returns early when it is set,
// and k_na_expand turns it into the status (d_q is then left as the caller had it).
constexpr int kFailNotSpd = 1;
constexpr int kFailBadFragment = 2;

// Validation pass: reads only d_frag and writes only the fragment counts (indexed by
// ids already checked to lie in [0, nfrag)) and meta.  Flags an id outside [0, nfrag)
// and a fragment id that no atom carries (its target charge would be lost).  One block.
__global__ void k_na_check(int n, int nfrag, const int* frag, Scratch s)
{
    int* count = s.a2r;   // nfrag <= n ints, rewritten by k_na_prepare afterwards
    for (int f = threadIdx.x; f < nfrag; f += blockDim.x) count[f] = 0;
    if (threadIdx.x == 0) s.meta[1] = 0;
    __syncthreads();
    bool bad = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int f = frag[i];
        if (f < 0 || f >= nfrag) bad = true;
        else atomicAdd(&count[f], 1);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nfrag; f += blockDim.x)
        if (count[f] == 0) bad = true;
    if (bad) atomicOr(&s.meta[1], kFailBadFragment);
}

// fragment anchors (first atom), uniform q0 = qfrag/n_f, reduced index maps; one thread
// (n <= kMaxAtoms).  Everything it reads later is written here first.  Runs only after
// k_na_check accepted every fragment id (a bad id would index outside the scratch).
__global__ void k_na_prepare(int n, int nfrag, const double* xyz, const int* frag, const double* qfrag,
                             Scratch s)
{
    if (blockIdx.x != 0 || s.meta[1] != 0) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        s.pos[4 * i] = xyz[3 * i];
        s.pos[4 * i + 1] = xyz[3 * i + 1];
        s.pos[4 * i + 2] = xyz[3 * i + 2];
        s.pos[4 * i + 3] = 0.0;
    }
    if (threadIdx.x != 0) return;
    int* first = s.r2a + n;          // nfrag <= n ints of temporary space
    for (int f = 0; f < nfrag; ++f) first[f] = -1;
    for (int i = 0; i < n; ++i) if (first[frag[i]] < 0) first[frag[i]] = i;
    // a2r still holds the per-fragment atom counts of k_na_check (every count >= 1)
    for (int i = 0; i < n; ++i) s.q0[i] = qfrag[frag[i]] / (double)s.a2r[frag[i]];
    for (int i = 0; i < n; ++i) s.anchor[i] = first[frag[i]];
    int nred = 0;
    for (int i = 0; i < n; ++i) {
        if (i == s.anchor[i]) s.a2r[i] = -frag[i] - 1;
        else { s.a2r[i] = nred; s.r2a[nred++] = i; }
    }
    s.meta[0] = nred;
}

__global__ void k_na_matrix(int n, const double* alpha, const double* gam, Scratch s)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= n || s.meta[1] != 0) return;
    double v;
    if (i == j) {
        v = gam[i] + 0.797884560802866 / sqrt(alpha[i]);
    } else {
        const double dx = s.pos[4 * i] - s.pos[4 * j], dy = s.pos[4 * i + 1] - s.pos[4 * j + 1],
                     dz = s.pos[4 * i + 2] - s.pos[4 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double g = 1.0 / sqrt(alpha[i] + alpha[j]);
        v = erf(g * r) / r;
    }
    s.A[(size_t)i * n + j] = v;
}

// r = x - A q0, one warp per row
__global__ void k_na_residual(int n, const double* chi, const double* cnf, const double* cn, Scratch s)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n || s.meta[1] != 0) return;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += s.A[(size_t)i * n + j] * s.q0[j];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) s.r[i] = chi[i] + cnf[i] * sqrt(cn[i]) - acc;
}

__global__ void k_na_reduce(int n, Scratch s)
{
    if (s.meta[1] != 0) return;
    const int nred = s.meta[0];
    const int lc = blockIdx.x * blockDim.x + threadIdx.x;
    const int kc = blockIdx.y;
    if (kc >= nred || lc >= nred) return;
    const int k = s.r2a[kc], l = s.r2a[lc];
    const int ak = s.anchor[k], al = s.anchor[l];
    const size_t nn = n;
    s.M[(size_t)kc * nred + lc] = s.A[k * nn + l] - s.A[k * nn + al] - s.A[ak * nn + l] + s.A[ak * nn + al];
    if (lc == 0) s.b[kc] = s.r[k] - s.r[ak];
}

// Cholesky of M (row-major, lower triangle) and the two triangular solves, one block
__global__ void __launch_bounds__(kThreads) k_na_cholesky_solve(Scratch s)
{
    if (s.meta[1] != 0) return;   // uniform over the block
    const int m = s.meta[0];
    __shared__ double inv;
    __shared__ int bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    if (tid == 0) bad = 0;
    __syncthreads();
    double* M = s.M;
    for (int k = 0; k < m; ++k) {
        if (tid == 0) {
            const double d = M[(size_t)k * m + k];
            if (!(d > 0.0)) bad = 1;
            else {
                const double L = sqrt(d);
                M[(size_t)k * m + k] = L;
                inv = 1.0 / L;
            }
        }
        __syncthreads();
        if (bad) break;
        for (int i = k + 1 + tid; i < m; i += blockDim.x) M[(size_t)i * m + k] *= inv;
        __syncthreads();
        for (int i = k + 1 + warp; i < m; i += nw) {
            const double lik = M[(size_t)i * m + k];
            for (int j = k + 1 + lane; j <= i; j += 32) M[(size_t)i * m + j] -= lik * M[(size_t)j * m + k];
        }
        __syncthreads();
    }
    if (bad) {
        if (tid == 0) s.meta[1] = kFailNotSpd;
        return;
    }
    // L y = b (column sweep), then L^T x = y
    double* b = s.b;
    for (int k = 0; k < m; ++k) {
        if (tid == 0) b[k] = b[k] / M[(size_t)k * m + k];
        __syncthreads();
        const double yk = b[k];
        for (int i = k + 1 + tid; i < m; i += blockDim.x) b[i] -= M[(size_t)i * m + k] * yk;
        __syncthreads();
    }
    for (int k = m - 1; k >= 0; --k) {
        if (tid == 0) b[k] = b[k] / M[(size_t)k * m + k];
        __syncthreads();
        const double xk = b[k];
        for (int i = tid; i < k; i += blockDim.x) b[i] -= M[(size_t)k * m + i] * xk;
        __syncthreads();
    }
}

// q = q0 + B y; the status of the call.  On a failure (bad fragment id, no Cholesky
// factor) only the status is written and d_q keeps the caller's contents.
__global__ void k_na_expand(int n, const int* frag, Scratch s, double* q, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int fail = s.meta[1];
    if (i == 0)
        *status = (fail & kFailBadFragment) ? GFNFF_INVALID_ARG : (fail ? GFNFF_NOT_SPD : GFNFF_OK);
    if (i >= n || fail != 0) return;
    const int rr = s.a2r[i];
    if (rr >= 0) {
        q[i] = s.q0[i] + s.b[rr];
    } else {
        double acc = 0.0;
        for (int a = 0; a < n; ++a)
            if (frag[a] == frag[i] && s.a2r[a] >= 0) acc += s.b[s.a2r[a]];
        q[i] = s.q0[i] - acc;
    }
}

}  // namespace

extern "C" gfnff_status gfnff_eeq_charges_noalloc(int natoms, int nfrag, const double* d_xyz_bohr,
                                                  const double* d_alpha, const double* d_gam, const double* d_chi,
                                                  const double* d_cnf, const double* d_cn, const int* d_frag,
                                                  const double* d_qfrag, double* d_q, int* d_status, void* stream)
{
    if (natoms < 1 || natoms > kMaxAtoms || nfrag < 1 || nfrag > natoms) return GFNFF_INVALID_ARG;
    if (!d_xyz_bohr || !d_alpha || !d_gam || !d_chi || !d_cnf || !d_cn || !d_frag || !d_qfrag || !d_q || !d_status)
        return GFNFF_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GFNFF_CUDA_ERROR;
    double* base = nullptr;
    {
        // once per device, with that device current: the device address of the array
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GFNFF_CUDA_ERROR;
            g_addr[dev] = static_cast<double*>(p);
        }
        base = g_addr[dev];
    }
    // an error left pending by earlier, unrelated work stays the caller's to read: report
    // it without launching (and without clearing it)
    if (cudaPeekAtLastError() != cudaSuccess) return GFNFF_CUDA_ERROR;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = natoms;
    Scratch sc = carve(base, n);
    k_na_check<<<1, kThreads, 0, s>>>(n, nfrag, d_frag, sc);
    k_na_prepare<<<1, 256, 0, s>>>(n, nfrag, d_xyz_bohr, d_frag, d_qfrag, sc);
    k_na_matrix<<<dim3((n + 127) / 128, n), 128, 0, s>>>(n, d_alpha, d_gam, sc);
    k_na_residual<<<(n * 32 + 127) / 128, 128, 0, s>>>(n, d_chi, d_cnf, d_cn, sc);
    k_na_reduce<<<dim3((n + 127) / 128, n), 128, 0, s>>>(n, sc);
    k_na_cholesky_solve<<<1, kThreads, 0, s>>>(sc);
    k_na_expand<<<(n + 127) / 128, 128, 0, s>>>(n, d_frag, sc, d_q, d_status);
    // nothing was pending before the launches, so an error now is one of them
    return cudaGetLastError() == cudaSuccess ? GFNFF_OK : GFNFF_CUDA_ERROR;
}
