// GFN-FF per-geometry energy + analytic gradient on B200 (sm_100a), FP64 form.
//
// Pipeline of one evaluation (single stream, every buffer device-resident):
//   positions -> CN (erf counting, 6 bohr) -> D4 Gaussian weights + half contraction
//   -> EEQ: dense Coulomb matrix, fragment constraints eliminated in the null space,
//      Cholesky solve -> charges
//   -> bonded terms (bond/angle/torsion/inversion/sTors/BATM/ATM/HB/XB, one thread per
//      term, gradient scattered with FP64 atomics)
//   -> repulsion (per-atom CSR lists) and all-pairs Coulomb + D4 dispersion (one thread
//      per atom row, partners staged through shared memory, no atomics)
//   -> self energy, CN chain rule (dE/dCN - q*cnf/(2 sqrt CN)) * dCN/dr, checks.
//
// Every kernel restates the curcuma routine cited beside it (paths relative to
// src/core/energy_calculators/ff_methods/).
#include "engine.h"

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/gfnff_b200.h"
#include "../tables/gfnff_tables.inc"

namespace gfnff {

#define CK(x)                                                                                \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess)                                                               \
            throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " + \
                                     __FILE__ + ":" + std::to_string(__LINE__));             \
    } while (0)

#define CS(x)                                                                                \
    do {                                                                                     \
        cusolverStatus_t s_ = (x);                                                           \
        if (s_ != CUSOLVER_STATUS_SUCCESS)                                                   \
            throw std::runtime_error("cuSOLVER error " + std::to_string((int)s_) + " at " +   \
                                     std::to_string(__LINE__));                              \
    } while (0)

namespace {

enum {
    T_BOND = 0, T_ANGLE, T_TORSION, T_INVERSION, T_STORSION, T_DISP, T_BREP, T_NBREP, T_COUL,
    T_HB, T_XB, T_ATM, T_BATM, T_TOTAL
};

constexpr int kBlock = 128;
constexpr double kPi = 3.14159265358979323846;

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t cnt)
    {
        free();
        n = cnt;
        if (cnt) CK(cudaMalloc(&p, cnt * sizeof(T)));
    }
    void upload(const std::vector<T>& v)
    {
        alloc(v.size());
        if (!v.empty()) CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    void free()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { free(); }
};

// ------------------------------------------------------------------------------------
// small device helpers
// ------------------------------------------------------------------------------------
struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double nrm(D3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ D3 ld(const double4* p, int i)
{
    double4 v = p[i];
    return {v.x, v.y, v.z};
}
__device__ __forceinline__ void agrad(double* g, int i, D3 v)
{
    atomicAdd(g + 3 * i, v.x);
    atomicAdd(g + 3 * i + 1, v.y);
    atomicAdd(g + 3 * i + 2, v.z);
}

// block-wide sum of one value, one atomicAdd per block into *dst
__device__ __forceinline__ void block_add(double v, double* dst)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v != 0.0) atomicAdd(dst, v);
    }
}

// bond-angle cosine and d(theta)/dx (forcefieldfunctions.h:47-83)
__device__ double angle_cos(D3 i, D3 j, D3 k, D3 d[3])
{
    D3 rij = i - j, rkj = k - j;
    const double a = nrm(rij), b = nrm(rkj);
    d[0] = d[1] = d[2] = mk(0, 0, 0);
    if (a < 1e-10 || b < 1e-10) return 1.0;
    D3 nij = (1.0 / a) * rij, nkj = (1.0 / b) * rkj;
    double c = dot(rij, rkj) / (a * b);
    c = fmax(-1.0, fmin(1.0, c));
    const double s = sqrt(fmax(0.0, 1.0 - c * c));
    if (s < 1e-14) return c;
    const double f = 1.0 / s;
    d[0] = (-f / a) * (nkj - c * nij);
    d[2] = (-f / b) * (nij - c * nkj);
    d[1] = -1.0 * (d[0] + d[2]);
    return c;
}

// dihedral angle and d(phi)/dx (gfnff_geometry.h:66-160)
__device__ double dihedral(D3 ri, D3 rj, D3 rk, D3 rl, D3 g[4])
{
    for (int a = 0; a < 4; ++a) g[a] = mk(0, 0, 0);
    D3 v1 = rj - ri, v2 = rk - rj, v3 = rl - rk;
    D3 n1 = cross(v1, v2), n2 = cross(v2, v3);
    const double n1n = nrm(n1), n2n = nrm(n2), v2n = nrm(v2);
    if (n1n < 1e-10 || n2n < 1e-10 || v2n < 1e-10) return 0.0;
    D3 h1 = (1.0 / n1n) * n1, h2 = (1.0 / n2n) * n2;
    const double cphi = dot(h1, h2);
    double sphi = (v2n * dot(h1, v3)) / n2n;
    sphi = fmax(-1.0, fmin(1.0, sphi));
    const double phi = atan2(sphi, cphi);
    const double nen = n1n * n2n * sin(phi);
    if (fabs(nen) < 1e-14) return phi;
    const double o = 1.0 / nen;
    D3 rab = cross(n1, v2), rbb = cross(n2, v2), rac = cross(n1, v3), rbc = cross(n2, v3);
    D3 rba = cross(n2, v1), raa = cross(n1, v1);
    D3 rapb = v1 + v2, rbpc = v2 + v3;
    D3 rapba = cross(rapb, n1), rapbb = cross(rapb, n2), rbpca = cross(rbpc, n1), rbpcb = cross(rbpc, n2);
    g[0] = o * ((cphi * n2n / n1n) * rab - rbb);
    g[1] = o * (cphi * ((n2n / n1n) * rapba + (n1n / n2n) * rbc) - (rac + rapbb));
    g[2] = o * (cphi * ((n2n / n1n) * raa + (n1n / n2n) * rbpcb) - (rba + rbpca));
    g[3] = o * ((cphi * n1n / n2n) * rbb - rab);
    return phi;
}

// out-of-plane angle and its derivative (gfnff_geometry.h:207-265)
__device__ double oop(D3 ri, D3 rj, D3 rk, D3 rl, D3 g[4])
{
    for (int a = 0; a < 4; ++a) g[a] = mk(0, 0, 0);
    D3 re = ri - rj, rd = rk - rj, rv = rl - ri;
    D3 rn = cross(re, rd);
    const double rnn = nrm(rn), rvn = nrm(rv);
    if (rnn < 1e-10 || rvn < 1e-10) return 0.0;
    double so = dot((1.0 / rnn) * rn, (1.0 / rvn) * rv);
    so = fmax(-1.0, fmin(1.0, so));
    const double om = asin(so);
    const double nen = rnn * rvn * cos(om);
    if (fabs(nen) < 1e-14) return om;
    const double o = 1.0 / nen, s = sin(om);
    D3 rdme = rd - re, rve = cross(rv, re), rne = cross(rn, re), rdv = cross(rd, rv), rdn = cross(rd, rn);
    D3 rvdme = cross(rv, rdme), rndme = cross(rn, rdme);
    g[0] = o * (rdv - rn - s * ((rvn / rnn) * rdn - (rnn / rvn) * rv));
    g[1] = o * (rvdme - (s * rvn / rnn) * rndme);
    g[2] = o * (rve - (s * rvn / rnn) * rne);
    g[3] = o * (rn - (s * rnn / rvn) * rv);
    return om;
}

// squared distance evaluated without FMA contraction, bit-identical to the host list
// builders ((dx*dx + dy*dy) + dz*dz)
__device__ __forceinline__ double d2_exact(double4 a, double4 b)
{
    const double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y), dz = __dsub_rn(a.z, b.z);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// ------------------------------------------------------------------------------------
// device view of the model
// ------------------------------------------------------------------------------------
struct View {
    int n, nfrag, K, nred;
    const double4* pos;       // current geometry (bohr)
    const double4* pos0;      // setup geometry (bohr)
    const double* rcov_cn;
    const double* rcov43;     // 4/3 * covalent_rad_d3 (angle/torsion damping)
    const double* rcov_d3;
    const double* chi_base;
    const double* cnf;
    const double* gam;
    const double* alpeeq;
    const double* qa;
    const int* slot;
    const int* nref;
    const double* refcn;      // n*7
    const double* w0;         // n*7 setup weights
    const double* g0;         // n*K*7 setup half contraction
    const double* c6ref;      // K*K*49
    const double* zeta;
    const double* szr;        // sqrt(0.5 r4/r2 sqrt Z)
    // per step
    double* cnraw;
    double* cn;
    double* dlog;
    double* w;                // n*7
    double* dw;
    double* hg;               // n*K*7
    double* hdg;
    double* q;
    double* dEdcn;
    double* v;
    double* grad;
    double* E;
    int* status;
};

// ------------------------------------------------------------------------------------
// geometry in, HB refresh metric (gfnff_method.cpp:2228-2259)
// ------------------------------------------------------------------------------------
__global__ void k_positions(int n, const double* __restrict__ xyz, double scale, double4* pos,
                            const double4* __restrict__ ref, double* msd, double* E, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < 16) E[threadIdx.x] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *status = 0;
    double s = 0.0;
    if (i < n) {
        const double x = xyz[3 * i] * scale, y = xyz[3 * i + 1] * scale, z = xyz[3 * i + 2] * scale;
        pos[i] = make_double4(x, y, z, 0.0);
        const double4 r = ref[i];
        s = (x - r.x) * (x - r.x) + (y - r.y) * (y - r.y) + (z - r.z) * (z - r.z);
    }
    block_add(s, msd);
}

// ------------------------------------------------------------------------------------
// coordination numbers, 6 bohr neighbour list (cn_calculator.cpp:367-428) and
// dlogCN/dCN (gfnff_method.cpp:5837-5940).  One thread per atom, partners staged in
// shared memory tiles.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_cn(View V)
{
    // one warp per atom i, lanes stride over the partners j
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= V.n) return;
    const double4 pi = V.pos[i];
    const double ri = V.rcov_cn[i];
    const double kn = -7.5;
    double s = 0.0;
    for (int j = lane; j < V.n; j += 32) {
        if (j == i) continue;
        const double4 pj = V.pos[j];
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < 36.0)) continue;
        const double r = sqrt(d2);
        const double rc = ri + V.rcov_cn[j];
        s += 0.5 * (1.0 + erf(kn * ((r - rc) / rc)));
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double cnmax = 4.4;
        V.cnraw[i] = s;
        V.cn[i] = log(1.0 + exp(cnmax)) - log(1.0 + exp(cnmax - s));
        V.dlog[i] = exp(cnmax) / (exp(cnmax) + exp(s));
    }
}

// ------------------------------------------------------------------------------------
// D4 Gaussian weights (wf = 4) and the half contraction with the reference C6
// (d4param_generator.cpp:1079-1290, :1692-1740)
// ------------------------------------------------------------------------------------
__global__ void k_d4_weights(View V)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.n) return;
    const int nr = V.nref[i];
    const double cn = V.cn[i];
    double ex[7], dex[7], w[7], dw[7];
    double norm = 0.0, dnorm = 0.0;
    for (int r = 0; r < 7; ++r) {
        ex[r] = dex[r] = w[r] = dw[r] = 0.0;
        if (r < nr) {
            const double d = cn - V.refcn[i * 7 + r];
            ex[r] = exp(-4.0 * d * d);
            dex[r] = (-2.0 * 4.0) * d * ex[r];
            norm += ex[r];
            dnorm += dex[r];
        }
    }
    if (nr > 0) {
        if (norm > 1e-10) {
            const double inv = 1.0 / norm, inv2 = 1.0 / (norm * norm);
            for (int r = 0; r < nr; ++r) {
                w[r] = ex[r] * inv;
                dw[r] = (dex[r] * norm - ex[r] * dnorm) * inv2;
            }
        } else {
            w[0] = 1.0;
        }
    }
    for (int r = 0; r < 7; ++r) { V.w[i * 7 + r] = w[r]; V.dw[i * 7 + r] = dw[r]; }
    const int si = V.slot[i];
    for (int s = 0; s < V.K; ++s) {
        const double* C = V.c6ref + ((size_t)(si * V.K + s)) * 49;
        for (int b = 0; b < 7; ++b) {
            double g = 0.0, dg = 0.0;
            for (int a = 0; a < nr; ++a) {
                g += w[a] * C[a * 7 + b];
                dg += dw[a] * C[a * 7 + b];
            }
            V.hg[((size_t)i * V.K + s) * 7 + b] = g;
            V.hdg[((size_t)i * V.K + s) * 7 + b] = dg;
        }
    }
}

// ------------------------------------------------------------------------------------
// EEQ (eeq_solver.cpp:3201-3700).  A_ij = erf(r/sqrt(a_i+a_j))/r, A_ii = gam_i +
// sqrt(2/pi)/sqrt(a_i), x_i = chi_i + cnf_i sqrt(CN_i), one charge constraint per
// fragment.  The constraints are removed by the substitution q = q0 + B y with
// q0 = qfrag/n_f and B the per-fragment difference basis (e_k - e_anchor); the reduced
// matrix B^T A B is SPD and is Cholesky-factored once per geometry.  This gives the
// same charges as curcuma's Schur-complement solve (:2087-2256).
// ------------------------------------------------------------------------------------
__global__ void k_eeq_matrix(View V, double* A)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= V.n) return;
    double v;
    if (i == j) {
        v = V.gam[i] + 0.797884560802866 / sqrt(V.alpeeq[i]);
    } else {
        const double4 a = V.pos[i], b = V.pos[j];
        const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double g = 1.0 / sqrt(V.alpeeq[i] + V.alpeeq[j]);
        v = erf(g * r) / r;
    }
    A[(size_t)i * V.n + j] = v;
}

// r = x - A q0 (one warp per row)
__global__ void k_eeq_residual(View V, const double* A, const double* q0, double* r)
{
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= V.n) return;
    double s = 0.0;
    for (int j = lane; j < V.n; j += 32) s += A[(size_t)i * V.n + j] * q0[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) r[i] = V.chi_base[i] + V.cnf[i] * sqrt(V.cn[i]) - s;
}

// M = B^T A B in the reduced (non-anchor) index space, b = B^T r
__global__ void k_eeq_reduce(View V, const double* A, const int* red2atom, const int* anchor,
                             const double* r, double* M, double* b)
{
    const int lc = blockIdx.x * blockDim.x + threadIdx.x;
    const int kc = blockIdx.y;
    if (lc >= V.nred) return;
    const int k = red2atom[kc], l = red2atom[lc];
    const int ak = anchor[k], al = anchor[l];
    const size_t n = V.n;
    M[(size_t)kc * V.nred + lc] = A[k * n + l] - A[k * n + al] - A[ak * n + l] + A[ak * n + al];
    if (lc == 0) b[kc] = r[k] - r[ak];
}

// q = q0 + B y
__global__ void k_eeq_expand(View V, const double* q0, const int* atom2red, const int* frag_off,
                             const int* frag_atoms, const int* anchor, const double* y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.n) return;
    const int rr = atom2red[i];
    if (rr >= 0) {
        V.q[i] = q0[i] + y[rr];
    } else {
        // anchor: minus the sum of its fragment's reduced variables
        const int f = -rr - 1;
        double s = 0.0;
        for (int p = frag_off[f]; p < frag_off[f + 1]; ++p) {
            const int a = frag_atoms[p];
            const int ra = atom2red[a];
            if (ra >= 0) s += y[ra];
        }
        V.q[i] = q0[i] - s;
    }
}

// ------------------------------------------------------------------------------------
// bonded terms
// ------------------------------------------------------------------------------------
struct BondSoA {
    int n;
    const int *i, *j, *hbh, *hb_off, *hb_b;
    const double *fc, *alpha, *r0i, *r0j, *cki, *ckj, *shift, *ff;
};

// bonds with the HB-modulated exponent and the r0(CN) chain rule
// (ff_workspace_gfnff.cpp:46-182)
__global__ void k_bonds(View V, BondSoA B)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (t < B.n) {
        const int i = B.i[t], j = B.j[t];
        D3 pi = ld(V.pos, i), pj = ld(V.pos, j);
        D3 ij = pi - pj;
        const double r = nrm(ij);
        D3 d0 = (1.0 / r) * ij;
        const double r0 = (B.r0i[t] + B.cki[t] * V.cn[i] + B.r0j[t] + B.ckj[t] * V.cn[j] + B.shift[t]) * B.ff[t];
        const double dr = r - r0;
        double alpha = B.alpha[t];
        const int H = B.hbh[t];
        const double kn = 27.5, isp = 0.5641895835477563;
        if (H >= 0) {
            double hcn = 0.0;
            D3 ph = ld(V.pos, H);
            for (int p = B.hb_off[t]; p < B.hb_off[t + 1]; ++p) {
                const int b = B.hb_b[p];
                D3 d = ld(V.pos, b) - ph;
                const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                if (r2 > 900.0) continue;
                const double rr = sqrt(r2);
                const double rc = 1.78 * (4.0 / 3.0) * (V.rcov_d3[H] + V.rcov_d3[b]);
                const double arg = -kn * (rr - rc) / rc;
                hcn += 0.5 * (1.0 + erf(arg));
            }
            alpha = (-(1.0 - 0.9) * hcn + 1.0) * B.alpha[t];
        }
        e = B.fc[t] * exp(-alpha * dr * dr);
        const double dEdr = -2.0 * alpha * dr * e;
        agrad(V.grad, i, dEdr * d0);
        agrad(V.grad, j, (-dEdr) * d0);
        if (H >= 0) {
            const double zz = 0.1 * B.alpha[t] * dr * dr * e;
            D3 ph = ld(V.pos, H);
            for (int p = B.hb_off[t]; p < B.hb_off[t + 1]; ++p) {
                const int b = B.hb_b[p];
                D3 d = ld(V.pos, b) - ph;
                const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                if (r2 > 900.0) continue;
                const double rr = sqrt(r2);
                const double rc = 1.78 * (4.0 / 3.0) * (V.rcov_d3[H] + V.rcov_d3[b]);
                const double arg = -kn * (rr - rc) / rc;
                const double dcn = isp * (-kn / rc) * exp(-arg * arg) / rr;
                agrad(V.grad, H, (zz * -dcn) * d);
                agrad(V.grad, b, (zz * dcn) * d);
            }
        }
        const double yy = -dEdr;
        atomicAdd(V.dEdcn + i, yy * B.ff[t] * B.cki[t]);
        atomicAdd(V.dEdcn + j, yy * B.ff[t] * B.ckj[t]);
    }
    block_add(e, V.E + T_BOND);
}

struct AngleSoA {
    int n;
    const int *i, *j, *k;
    const double *fc, *th0;
};

// angles with distance damping (ff_workspace_gfnff.cpp:187-280)
__global__ void k_angles(View V, AngleSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int ia = A.i[t], ja = A.j[t], ka = A.k[t];
        D3 pi = ld(V.pos, ia), pj = ld(V.pos, ja), pk = ld(V.pos, ka), d[3];
        double c = angle_cos(pi, pj, pk, d);
        c = fmax(-1.0, fmin(1.0, c));
        const double th = acos(c), th0 = A.th0[t], fc = A.fc[t];
        double e, dedth;
        if (fabs(kPi - th0) < 1e-6) {
            const double dt = th - th0;
            e = fc * dt * dt;
            dedth = 2.0 * fc * dt;
        } else {
            const double c0 = cos(th0), dc = c - c0;
            e = fc * dc * dc;
            dedth = 2.0 * fc * sin(th) * (c0 - c);
        }
        const double rij2 = dot(pi - pj, pi - pj), rjk2 = dot(pk - pj, pk - pj);
        const double ri = V.rcov43[ia], rj = V.rcov43[ja], rk = V.rcov43[ka];
        const double cij = 0.595 * (ri + rj) * (ri + rj), cjk = 0.595 * (rj + rk) * (rj + rk);
        double a1 = rij2 / cij; a1 = a1 * a1;
        double a2 = rjk2 / cjk; a2 = a2 * a2;
        const double dij = 1.0 / (1.0 + a1), djk = 1.0 / (1.0 + a2), damp = dij * djk;
        const double e2ij = rij2 > 1e-8 ? -2.0 * 2.0 * a1 / (rij2 * (1.0 + a1) * (1.0 + a1)) : 0.0;
        const double e2jk = rjk2 > 1e-8 ? -2.0 * 2.0 * a2 / (rjk2 * (1.0 + a2) * (1.0 + a2)) : 0.0;
        et = e * damp;
        D3 t1 = (e * e2ij * djk) * (pi - pj), t2 = (e * e2jk * dij) * (pk - pj);
        agrad(V.grad, ia, (dedth * damp) * d[0] + t1);
        agrad(V.grad, ja, (dedth * damp) * d[1] - t1 - t2);
        agrad(V.grad, ka, (dedth * damp) * d[2] + t2);
    }
    block_add(et, V.E + T_ANGLE);
}

struct TorsSoA {
    int n;
    const int *i, *j, *k, *l;
    const double *V, *nn, *phi0;
};

// torsions + extra torsions (ff_workspace_gfnff.cpp:282-487), triple-bond torsions
// (:611-653) when storsion = true
__global__ void k_torsions(View V, TorsSoA T, int storsion)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < T.n) {
        const int a = T.i[t], b = T.j[t], c = T.k[t], d = T.l[t];
        D3 ri = ld(V.pos, a), rj = ld(V.pos, b), rk = ld(V.pos, c), rl = ld(V.pos, d), g[4];
        const double phi = dihedral(ri, rj, rk, rl, g);
        if (storsion) {
            const double eh = T.V[t];
            et = -eh * cos(2.0 * phi) + eh;
            const double dEdphi = 2.0 * eh * sin(2.0 * phi);
            agrad(V.grad, a, dEdphi * g[0]);
            agrad(V.grad, b, dEdphi * g[1]);
            agrad(V.grad, c, dEdphi * g[2]);
            agrad(V.grad, d, dEdphi * g[3]);
        } else {
            const double Vb = T.V[t], n = T.nn[t];
            const double c1 = n * (phi - T.phi0[t]) + kPi;
            const double e = Vb * (1.0 + cos(c1));
            const double rij2 = dot(ri - rj, ri - rj), rjk2 = dot(rj - rk, rj - rk), rkl2 = dot(rk - rl, rk - rl);
            const double qa = V.rcov43[a], qb = V.rcov43[b], qc = V.rcov43[c], qd = V.rcov43[d];
            const double cij = 0.505 * (qa + qb) * (qa + qb), cjk = 0.505 * (qb + qc) * (qb + qc),
                         ckl = 0.505 * (qc + qd) * (qc + qd);
            double a1 = rij2 / cij; a1 *= a1;
            double a2 = rjk2 / cjk; a2 *= a2;
            double a3 = rkl2 / ckl; a3 *= a3;
            const double dij = 1.0 / (1.0 + a1), djk = 1.0 / (1.0 + a2), dkl = 1.0 / (1.0 + a3);
            const double damp = dij * djk * dkl;
            et = e * damp;
            const double dEdphi = -Vb * n * sin(c1) * damp;
            const double e2ij = rij2 > 1e-8 ? -4.0 * a1 / (rij2 * (1.0 + a1) * (1.0 + a1)) : 0.0;
            const double e2jk = rjk2 > 1e-8 ? -4.0 * a2 / (rjk2 * (1.0 + a2) * (1.0 + a2)) : 0.0;
            const double e2kl = rkl2 > 1e-8 ? -4.0 * a3 / (rkl2 * (1.0 + a3) * (1.0 + a3)) : 0.0;
            D3 t1 = (e * e2ij * djk * dkl) * (ri - rj), t2 = (e * dij * e2jk * dkl) * (rj - rk),
               t3 = (e * dij * djk * e2kl) * (rk - rl);
            agrad(V.grad, a, dEdphi * g[0] + t1);
            agrad(V.grad, b, dEdphi * g[1] + t2 - t1);
            agrad(V.grad, c, dEdphi * g[2] + t3 - t2);
            agrad(V.grad, d, dEdphi * g[3] - t3);
        }
    }
    block_add(et, V.E + (storsion ? T_STORSION : T_TORSION));
}

struct InvSoA {
    int n;
    const int *i, *j, *k, *l, *type;
    const double *fc, *om0;
};

// inversions (ff_workspace_gfnff.cpp:489-609)
__global__ void k_inversions(View V, InvSoA I)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < I.n) {
        const int a = I.i[t], b = I.j[t], c = I.k[t], d = I.l[t];
        D3 rc = ld(V.pos, a), r1 = ld(V.pos, b), r2 = ld(V.pos, c), r3 = ld(V.pos, d), g[4];
        const double om = oop(rc, r1, r2, r3, g);
        const double ci = V.rcov43[a], c1 = V.rcov43[b], c2 = V.rcov43[c], c3 = V.rcov43[d];
        auto damp = [](double rsq, double x, double y) {
            const double cut = 0.505 * (x + y) * (x + y);
            const double rr = (rsq / cut) * (rsq / cut);
            return 1.0 / (1.0 + rr);
        };
        auto ddamp = [](double rsq, double x, double y) {
            if (rsq < 1e-8) return 0.0;
            const double cut = 0.505 * (x + y) * (x + y);
            const double rr = (rsq / cut) * (rsq / cut);
            return -4.0 * rr / (rsq * (1.0 + rr) * (1.0 + rr));
        };
        const double rij2 = dot(r1 - rc, r1 - rc), rjk2 = dot(r1 - r2, r1 - r2), rjl2 = dot(r1 - r3, r1 - r3);
        const double dij = damp(rij2, ci, c1), djk = damp(rjk2, c2, c1), djl = damp(rjl2, c1, c3);
        const double dmp = dij * djk * djl;
        double et, dEdom;
        const double fc = I.fc[t];
        if (I.type[t] == 0) {
            et = fc * (1.0 - cos(om));
            dEdom = fc * sin(om) * dmp;
        } else {
            const double df = cos(om) - cos(I.om0[t]);
            et = fc * df * df;
            dEdom = -2.0 * fc * sin(om) * df * dmp;
        }
        etot = et * dmp;
        const double e1 = ddamp(rij2, ci, c1), e2 = ddamp(rjk2, c2, c1), e3 = ddamp(rjl2, c1, c3);
        D3 t1 = (et * e1 * djk * djl) * (r1 - rc), t2 = (et * e2 * dij * djl) * (r1 - r2),
           t3 = (et * e3 * dij * djk) * (r1 - r3);
        agrad(V.grad, a, dEdom * g[0] - t1);
        agrad(V.grad, b, dEdom * g[1] + t1 + t2 + t3);
        agrad(V.grad, c, dEdom * g[2] - t2);
        agrad(V.grad, d, dEdom * g[3] - t3);
    }
    block_add(etot, V.E + T_INVERSION);
}

struct TripSoA {
    int n;
    const int *i, *j, *k;
    const double *c9, *r0ij, *r0ik, *r0jk, *scale;   // ATM; BATM uses c9 only
};

// D4 ATM over bonded triplets (ff_workspace_gfnff.cpp:1526-1663)
__global__ void k_atm(View V, TripSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int a = A.i[t], b = A.j[t], c = A.k[t];
        D3 pi = ld(V.pos, a), pj = ld(V.pos, b), pk = ld(V.pos, c);
        D3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double rij = nrm(vij), rik = nrm(vik), rjk = nrm(vjk);
        const double r2ij = rij * rij, r2ik = rik * rik, r2jk = rjk * rjk;
        const double c9 = A.c9[t];
        const double rijk = rij * rik * rjk, r2ijk = r2ij * r2ik * r2jk, r3ijk = rijk * r2ijk;
        const double tmp = pow(A.r0ij[t] * A.r0ik[t] * A.r0jk[t] / rijk, 14.0 / 3.0);
        const double fdmp = 1.0 / (1.0 + 6.0 * tmp);
        const double X = r2ij + r2jk - r2ik, Y = r2ij + r2ik - r2jk, Zc = r2ik + r2jk - r2ij;
        const double ang = (0.375 * X * Y * Zc / r2ijk + 1.0) / r3ijk;
        const double sc = A.scale[t];
        et = ang * fdmp * c9 / 3.0 * sc;
        const double r5ijk = r2ijk * r3ijk;
        const double dfdmp = -2.0 * 14.0 * tmp * fdmp * fdmp;
        const double dij = -0.375 * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik) +
                                     r2ij * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ik + 3.0 * r2ik * r2ik) -
                                     5.0 * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) / r5ijk;
        const double dik = -0.375 * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij) +
                                     r2ik * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) / r5ijk;
        const double djk = -0.375 * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij) +
                                     r2jk * (3.0 * r2ik * r2ik + 2.0 * r2ik * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) / r5ijk;
        const double pre = -c9 * sc / 3.0;
        D3 gij = (pre * (-dij * fdmp + ang * dfdmp) / r2ij) * vij;
        D3 gik = (pre * (-dik * fdmp + ang * dfdmp) / r2ik) * vik;
        D3 gjk = (pre * (-djk * fdmp + ang * dfdmp) / r2jk) * vjk;
        agrad(V.grad, a, -1.0 * (gij + gik));
        agrad(V.grad, b, gij - gjk);
        agrad(V.grad, c, gik + gjk);
    }
    block_add(et, V.E + T_ATM);
}

// bonded ATM with the Phase-1 charge factors folded into c9 (ff_workspace_gfnff.cpp:1665-1739)
__global__ void k_batm(View V, TripSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int a = A.i[t], b = A.j[t], c = A.k[t];
        D3 pi = ld(V.pos, a), pj = ld(V.pos, b), pk = ld(V.pos, c);
        D3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double r2ij = dot(vij, vij), r2jk = dot(vjk, vjk), r2ik = dot(vik, vik);
        const double rij = sqrt(r2ij), rjk = sqrt(r2jk), rik = sqrt(r2ik);
        const double rijk3 = r2ij * r2jk * r2ik;
        const double mijk = -r2ij + r2jk + r2ik, imjk = r2ij - r2jk + r2ik, ijmk = r2ij + r2jk - r2ik;
        const double ang = 0.375 * ijmk * imjk * mijk / rijk3;
        const double rav3 = pow(rijk3, 1.5);
        const double c9 = A.c9[t];
        et = c9 * ((ang + 1.0) / rav3);
        const double den = rijk3 * rav3;
        const double dij = -0.375 * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik) +
                                     r2ij * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ik + 3.0 * r2ik * r2ik) -
                                     5.0 * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) / (rij * den);
        const double djk = -0.375 * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij) +
                                     r2jk * (3.0 * r2ik * r2ik + 2.0 * r2ik * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) / (rjk * den);
        const double dik = -0.375 * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij) +
                                     r2ik * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) / (rik * den);
        D3 gij = (-dij * c9 / rij) * vij, gjk = (-djk * c9 / rjk) * vjk, gik = (-dik * c9 / rik) * vik;
        agrad(V.grad, b, gjk - gij);
        agrad(V.grad, c, -1.0 * gik - gjk);
        agrad(V.grad, a, gij + gik);
    }
    block_add(et, V.E + T_BATM);
}

struct HBSoA {
    int n;
    const int *a, *h, *b, *cas, *pc, *nbb_off, *nbb, *nbc_off, *nbc;
    const double *bas_a, *bas_b, *aci_a, *aci_b, *QH, *QA, *QB, *rv, *zlp;
    const int* nflag;   // acceptor is N with a single neighbour: neighbour cutoff 2.0
};

// hydrogen bonds, cases 1-4 (ff_workspace_gfnff.cpp:938-1409)
__global__ void __launch_bounds__(kBlock) k_hbonds(View V, HBSoA S)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < S.n) {
        const double HB_BACUT = 49.0, HB_SCUT = 22.0, HB_ALP = 6.0, HB_LONGCUT = 85.0, HB_NBCUT = 11.20;
        const double TORS_HB = 0.94, BEND_HB = 0.20, HBLPCUT = 56.0;
        const int A = S.a[t], H = S.h[t], Bq = S.b[t], cs = S.cas[t];
        D3 pA = ld(V.pos, A), pH = ld(V.pos, H), pB = ld(V.pos, Bq);
        const double rAH = nrm(pH - pA), rHB = nrm(pB - pH), rAB = nrm(pB - pA);
        if (rAB <= 50.0) {
            const double rAH4 = rAH * rAH * rAH * rAH, rHB4 = rHB * rHB * rHB * rHB;
            const double den = 1.0 / (rAH4 + rHB4);
            const double QH = S.QH[t], QA = S.QA[t], QB = S.QB[t];
            const double bas = (QA * S.bas_a[t] * rAH4 + QB * S.bas_b[t] * rHB4) * den;
            const double aci = (S.aci_b[t] * rAH4 + S.aci_a[t] * rHB4) * den;
            const double rv = S.rv[t];
            const double dsh = 1.0 / (1.0 + pow(HB_SCUT * rv / (rAB * rAB), HB_ALP));
            const double dlg = 1.0 / (1.0 + pow(rAB * rAB / HB_LONGCUT, HB_ALP));
            const double denv = dsh * dlg;
            double doutl;
            {
                const double ex = (HB_BACUT / rv) * ((rAH + rHB) / rAB - 1.0);
                doutl = ex > 15.0 ? 0.0 : 2.0 / (1.0 + exp(ex));
            }
            const int nb0 = S.nbb_off[t], nb1 = S.nbb_off[t + 1];
            const double nbcut = S.nflag[t] ? 2.0 : HB_NBCUT;
            double onb = 1.0;
            if (cs >= 2)
                for (int p = nb0; p < nb1; ++p) {
                    D3 pn = ld(V.pos, S.nbb[p]);
                    const double ra = nrm(pn - pA), rb = nrm(pn - pB);
                    const double ex = (nbcut / rv) * ((ra + rb) / rAB - 1.0);
                    onb *= (2.0 / (1.0 + exp(-ex)) - 1.0);
                }
            const double rdamp = cs >= 2 ? denv * (1.8 / (rHB * rHB * rHB) - 0.8 / (rAB * rAB * rAB))
                                         : denv / (rAB * rAB * rAB);
            double olp = 1.0, lpd = 0.0;
            int nlp = 0;
            D3 lpv = mk(0, 0, 0), lpp = pB;
            if (cs == 4) {
                lpd = 0.50 - 0.018 * S.zlp[t];
                nlp = nb1 - nb0;
                for (int p = nb0; p < nb1; ++p) lpv = lpv + (ld(V.pos, S.nbb[p]) - pB);
                const double vn = nrm(lpv);
                if (vn > 1e-10 && nlp > 0) {
                    lpp = pB + (-lpd) * ((1.0 / vn) * lpv);
                    const double ral = nrm(pA - lpp);
                    const double ex = (HBLPCUT / rv) * ((ral + lpd + 1e-12) / rAB - 1.0);
                    olp = 2.0 / (1.0 + exp(ex));
                } else {
                    nlp = 0;
                    olp = 1.0;
                }
            }
            const double qhoutl = QH * doutl * onb * olp;
            double eangl = 1.0, etors = 1.0;
            D3 ga3[3] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)};
            const int Ci = S.pc[t];
            const bool c3 = (cs == 3 && Ci != -1);
            if (c3) {
                const double c0 = 120.0 * kPi / 180.0;
                const double kijk = (1.0 - BEND_HB) / ((cos(0.0) - cos(c0)) * (cos(0.0) - cos(c0)));
                D3 va = ld(V.pos, Ci), vb = pB, vc = pH;
                D3 vab = va - vb, vcb = vc - vb;
                const double rab2 = dot(vab, vab), rcb2 = dot(vcb, vcb);
                D3 vp = cross(vcb, vab);
                const double rp = nrm(vp) + 1e-14;
                double ca = dot(vab, vcb) / (sqrt(rab2) * sqrt(rcb2) + 1e-14);
                ca = fmax(-1.0, fmin(1.0, ca));
                const double th = acos(ca);
                const double ea = kijk * (ca - cos(c0)) * (ca - cos(c0));
                const double deddt = 2.0 * kijk * sin(th) * (cos(c0) - ca);
                eangl = 1.0 - ea;
                D3 deda = (-deddt / (rab2 * rp)) * cross(vab, vp);
                D3 dedc = (deddt / (rcb2 * rp)) * cross(vcb, vp);
                ga3[0] = deda + dedc;
                ga3[1] = -1.0 * deda;
                ga3[2] = -1.0 * dedc;
                for (int p = S.nbc_off[t]; p < S.nbc_off[t + 1]; ++p) {
                    const int D = S.nbc[p];
                    if (D == Bq) continue;
                    D3 g[4];
                    const double phi = dihedral(ld(V.pos, D), pB, va, pH, g);
                    const double fct = (1.0 - TORS_HB) / 2.0;
                    const double c1 = 2 * (phi - kPi / 2.0) + kPi;
                    etors *= (1.0 + cos(c1)) * fct + TORS_HB;
                }
            }
            double gs = 1.0;
            if (cs == 2 || cs == 4) gs = 0.268;
            else if (cs == 3) gs = 0.350;
            const double cst = S.aci_a[t] * S.bas_b[t] * QA * QB * gs;
            const double E = cs >= 2 ? -rdamp * qhoutl * cst * eangl * etors : -bas * aci * rdamp * qhoutl;
            etot = E;

            D3 drab = pA - pB, drah = pA - pH, drbh = pB - pH;
            const double rab2 = rAB * rAB, rbh2 = rHB * rHB, rah2 = rAH * rAH;
            const double rahprbh = rAH + rHB + 1e-12;
            const double ratio1 = pow(rab2 / HB_LONGCUT, HB_ALP);
            const double ratio3 = pow(HB_SCUT * rv / rab2, HB_ALP);
            const double ddamp = (-2.0 * HB_ALP * ratio1 / (1.0 + ratio1)) + (2.0 * HB_ALP * ratio3 / (1.0 + ratio3));
            const double expo = (HB_BACUT / rv) * (rahprbh / rAB - 1.0);
            if (expo <= 15.0) {
                const double ratio2 = exp(expo);
                D3 ga = mk(0, 0, 0), gb = mk(0, 0, 0), gh = mk(0, 0, 0);
                if (cs >= 2) {
                    const double rbhdamp = denv * 1.8 / (rbh2 * rHB);
                    const double rabdamp = denv * (-0.8) / (rab2 * rAB);
                    const double dterm = -qhoutl * eangl * etors * cst;
                    const double aterm = -rdamp * QH * onb * olp * eangl * etors * cst;
                    const double nbterm = -rdamp * QH * doutl * olp * eangl * etors * cst;
                    double gi = ((rabdamp + rbhdamp) * ddamp - 3.0 * rabdamp) / rab2;
                    gi *= dterm;
                    D3 dg = gi * drab;
                    ga = dg;
                    gb = -1.0 * dg;
                    gi = -3.0 * rbhdamp / rbh2;
                    gi *= dterm;
                    dg = gi * drbh;
                    gb = gb + dg;
                    gh = -1.0 * dg;
                    const double tmp1 = -2.0 * aterm * ratio2 * expo / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB);
                    gi = -tmp1 * rahprbh / rab2;
                    dg = gi * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    D3 dgao = (tmp1 / rAH) * drah, dgbo = (tmp1 / rHB) * drbh;
                    ga = ga + dgao;
                    gb = gb + dgbo;
                    gh = gh - dgao - dgbo;
                    for (int p = nb0; p < nb1; ++p) {
                        const int nb = S.nbb[p];
                        D3 pn = ld(V.pos, nb);
                        D3 dranb = pA - pn, drbnb = pB - pn;
                        const double ranb = nrm(dranb), rbnb = nrm(drbnb);
                        const double sum = ranb + rbnb + 1e-12;
                        const double ex = (nbcut / rv) * (sum / rAB - 1.0);
                        const double r2n = exp(-ex);
                        const double oi = 2.0 / (1.0 + r2n) - 1.0;
                        const double others = fabs(oi) > 1e-12 ? onb / oi : 1.0;
                        const double tmp2 = 2.0 * nbterm * others * r2n * ex / ((1.0 + r2n) * (1.0 + r2n)) / (sum - rAB);
                        dg = (-tmp2 * sum / rab2) * drab;
                        ga = ga + dg;
                        gb = gb - dg;
                        D3 dgan = (tmp2 / ranb) * dranb, dgbn = (tmp2 / rbnb) * drbnb;
                        ga = ga + dgan;
                        gb = gb + dgbn;
                        agrad(V.grad, nb, -1.0 * dgan - dgbn);
                    }
                    if (cs == 4 && nlp > 0) {
                        const double lpterm = -rdamp * QH * doutl * onb * cst;
                        const double ral = nrm(pA - lpp);
                        const double sum = ral + lpd + 1e-12;
                        const double ex = (HBLPCUT / rv) * (sum / rAB - 1.0);
                        const double r2l = exp(ex);
                        const double tmp3 = -2.0 * lpterm * r2l * ex / ((1.0 + r2l) * (1.0 + r2l)) / (sum - rAB);
                        D3 dgl = (-tmp3 * sum / rab2) * drab;
                        ga = ga + dgl;
                        gb = gb - dgl;
                        D3 dral = pA - lpp;
                        D3 dgal = (tmp3 / (ral + 1e-12)) * dral;
                        ga = ga + dgal;
                        gb = gb - dgal;
                        D3 glp = -1.0 * dgal;
                        const double vn = nrm(lpv);
                        if (vn > 1e-10) {
                            const double lv[3] = {lpv.x, lpv.y, lpv.z}, gl3[3] = {glp.x, glp.y, glp.z};
                            double out[3] = {0, 0, 0};
                            const double vn3 = pow(vn, 3.0);
                            for (int col = 0; col < 3; ++col)
                                for (int row = 0; row < 3; ++row) {
                                    const double unit = (row == col) ? -1.0 : 0.0;
                                    out[row] += -lpd * (double)nlp * (unit / vn + lv[row] * lv[col] / vn3) * gl3[col];
                                }
                            D3 gnb = mk(out[0], out[1], out[2]);
                            gb = gb + gnb;
                            D3 share = (1.0 / (double)nlp) * gnb;
                            for (int p = nb0; p < nb1; ++p) agrad(V.grad, S.nbb[p], -1.0 * share);
                        }
                    }
                    if (c3) {
                        const double bterm = -rdamp * qhoutl * etors * cst;
                        const double tterm = -rdamp * qhoutl * eangl * cst;
                        agrad(V.grad, Bq, bterm * ga3[0]);
                        agrad(V.grad, Ci, bterm * ga3[1]);
                        agrad(V.grad, H, bterm * ga3[2]);
                        D3 va = ld(V.pos, Ci);
                        for (int p = S.nbc_off[t]; p < S.nbc_off[t + 1]; ++p) {
                            const int D = S.nbc[p];
                            if (D == Bq) continue;
                            D3 g[4];
                            const double phi = dihedral(ld(V.pos, D), pB, va, pH, g);
                            const double fct = (1.0 - TORS_HB) / 2.0;
                            const double c1 = 2 * (phi - kPi / 2.0) + kPi;
                            const double ek = (1.0 + cos(c1)) * fct + TORS_HB;
                            const double dij = -2 * sin(c1) * fct;
                            const double fk = fabs(ek) > 1e-12 ? etors / ek : 0.0;
                            const double tk = fk * tterm;
                            agrad(V.grad, D, (tk * dij) * g[0]);
                            agrad(V.grad, Bq, (tk * dij) * g[1]);
                            agrad(V.grad, Ci, (tk * dij) * g[2]);
                            agrad(V.grad, H, (tk * dij) * g[3]);
                        }
                    }
                } else {
                    const double caa = QA * S.bas_a[t], cbb = QB * S.bas_b[t];
                    const double rterm = -aci * rdamp * qhoutl, dterm = -aci * bas * qhoutl;
                    const double sterm = -rdamp * bas * qhoutl, aterm = -aci * bas * rdamp * QH;
                    const double dv = 1.0 / (rAH4 + rHB4);
                    const double tmp = dv * dv * 4.0;
                    const double dd24a = rah2 * rHB4 * tmp, dd24b = rbh2 * rAH4 * tmp;
                    double gi = (caa - cbb) * dd24a * rterm;
                    ga = gi * drah;
                    gi = (cbb - caa) * dd24b * rterm;
                    gb = gi * drbh;
                    gh = -1.0 * ga - gb;
                    gi = (S.aci_b[t] - S.aci_a[t]) * dd24a;
                    D3 dga = (gi * sterm) * drah;
                    ga = ga + dga;
                    gi = (S.aci_a[t] - S.aci_b[t]) * dd24b;
                    D3 dgb = (gi * sterm) * drbh;
                    gb = gb + dgb;
                    gh = gh - dga - dgb;
                    gi = rdamp * (ddamp - 3.0) / rab2;
                    D3 dg = (gi * dterm) * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    gi = aterm * 2.0 * ratio2 * expo * rahprbh / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB) / rab2;
                    dg = gi * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    const double to = -2.0 * aterm * ratio2 * expo / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB);
                    D3 dgao = (to / rAH) * drah, dgbo = (to / rHB) * drbh;
                    ga = ga + dgao;
                    gb = gb + dgbo;
                    gh = gh - dgao - dgbo;
                }
                agrad(V.grad, A, ga);
                agrad(V.grad, Bq, gb);
                agrad(V.grad, H, gh);
            }
        }
    }
    block_add(etot, V.E + T_HB);
}

struct XBSoA {
    int n;
    const int *a, *x, *b;
    const double *pre, *rv;
};

// halogen bonds (ff_workspace_gfnff.cpp:1411-1524); pre = -Q_B * acidity_X * Q_X
__global__ void k_xbonds(View V, XBSoA S)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < S.n) {
        const double XB_BACUT = 70.0, XB_SCUT = 5.0, ALP = 6.0, LC = 70.0;
        D3 pA = ld(V.pos, S.a[t]), pX = ld(V.pos, S.x[t]), pB = ld(V.pos, S.b[t]);
        D3 vAX = pX - pA, vXB = pB - pX, vAB = pB - pA;
        const double rAX = nrm(vAX), rXB = nrm(vXB), rAB = nrm(vAB);
        const double ex = XB_BACUT * ((rAX + rXB) / rAB - 1.0);
        if (rXB <= 20.0 && ex <= 15.0) {
            const double rv = S.rv[t];
            const double dsh = 1.0 / (1.0 + pow(XB_SCUT * rv / (rXB * rXB), ALP));
            const double dlg = 1.0 / (1.0 + pow(rXB * rXB / LC, ALP));
            const double dol = 2.0 / (1.0 + exp(ex));
            const double r3 = rXB * rXB * rXB;
            const double R = dsh * dlg * dol / r3;
            const double pre = S.pre[t];
            etot = R * pre;
            const double st = pow(XB_SCUT * rv / (rXB * rXB), ALP);
            const double dds = -2.0 * ALP * dsh * st / (rXB * (1.0 + st));
            const double lt = pow((rXB * rXB) / LC, ALP);
            const double ddl = -2.0 * ALP * rXB * dlg * lt / (LC * (1.0 + lt));
            const double et = exp(ex), de = 1.0 + et;
            const double do_ax = -2.0 * et * XB_BACUT / (rAB * de * de);
            const double do_ab = 2.0 * et * XB_BACUT * (rAX + rXB) / (rAB * rAB * de * de);
            const double dR_xb = (dds * dlg * dol + dsh * ddl * dol + dsh * dlg * do_ax) / r3 - 3.0 * R / rXB;
            const double eXB = pre * dR_xb, eAX = pre * dsh * dlg * do_ax / r3, eAB = pre * dsh * dlg * do_ab / r3;
            D3 uAX = (1.0 / (rAX + 1e-14)) * vAX, uXB = (1.0 / (rXB + 1e-14)) * vXB, uAB = (1.0 / (rAB + 1e-14)) * vAB;
            agrad(V.grad, S.a[t], -eAX * uAX - eAB * uAB);
            agrad(V.grad, S.x[t], eAX * uAX - eXB * uXB);
            agrad(V.grad, S.b[t], eXB * uXB + eAB * uAB);
        }
    }
    block_add(etot, V.E + T_XB);
}

// ------------------------------------------------------------------------------------
// repulsion over per-atom CSR lists holding both pair directions
// (ff_workspace_gfnff.cpp:774-848); kind 0 = bonded, 1 = non-bonded
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_repulsion(View V, const int* off, const int* nbj, const double* alpha,
                                                     const double* repab, const unsigned char* kind)
{
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    double eb = 0.0, enb = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    if (i < V.n) {
        const double4 pi = V.pos[i];
        for (int p = off[i] + lane; p < off[i + 1]; p += 32) {
            const double4 pj = V.pos[nbj[p]];
            const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r > 20.0 || r < 1e-8) continue;
            const double sr = sqrt(r);
            const double e = repab[p] * exp(-alpha[p] * (r * sr)) / r;
            if (kind[p]) enb += 0.5 * e; else eb += 0.5 * e;
            const double dEdr = -e / r - 1.5 * alpha[p] * sr * e;
            const double f = dEdr / r;
            gx += f * dx; gy += f * dy; gz += f * dz;
        }
        for (int o = 16; o > 0; o >>= 1) {
            gx += __shfl_down_sync(0xffffffffu, gx, o);
            gy += __shfl_down_sync(0xffffffffu, gy, o);
            gz += __shfl_down_sync(0xffffffffu, gz, o);
        }
        if (lane == 0) {
            V.grad[3 * i] += gx;
            V.grad[3 * i + 1] += gy;
            V.grad[3 * i + 2] += gz;
        }
    }
    block_add(eb, V.E + T_BREP);
    block_add(enb, V.E + T_NBREP);
}

// ------------------------------------------------------------------------------------
// all-pairs Coulomb (r <= 100 bohr; ff_workspace_gfnff.cpp:850-900) and D4 dispersion
// over the setup pair list (setup distance <= 60 bohr, evaluated for r <= 50;
// :715-772, d4param_generator.cpp:1959-2092) with the frozen setup C6 and the
// per-step dC6/dCN chain term.  One thread owns one row i; energies are halved.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_pairs(View V)
{
    // one warp per row i, lanes stride over the partners j (coalesced SoA loads)
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    double ec = 0.0, ed = 0.0, gx = 0.0, gy = 0.0, gz = 0.0, dcn = 0.0;
    if (i < V.n) {
        const double4 pi = V.pos[i], p0i = V.pos0[i];
        const double ai = V.alpeeq[i], qi = V.q[i], zi = V.zeta[i], szi = V.szr[i];
        const double* g0i = V.g0 + (size_t)i * V.K * 7;
        const double* dgi = V.hdg + (size_t)i * V.K * 7;
        const double a1 = 0.58, a2 = 4.80, tsp = 2.0 / 1.772453850905516;
        for (int j = lane; j < V.n; j += 32) {
            if (j == i) continue;
            const double4 pj = V.pos[j];
            const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            double dEdr = 0.0;
            if (r <= 100.0 && r >= 1e-10) {
                const double g = 1.0 / sqrt(ai + V.alpeeq[j]);
                const double gr = g * r;
                const double ef = erf(gr);
                const double qq = qi * V.q[j];
                ec += qq * ef / r;
                dEdr += qq * ((g * exp(-gr * gr) * tsp) / r - ef / (r * r));
            }
            if (r <= 50.0 && r >= 1e-10 && d2_exact(p0i, V.pos0[j]) <= 3600.0) {
                const int sj = V.slot[j], nr = V.nref[j];
                const double* g0 = g0i + sj * 7;
                const double* dg = dgi + sj * 7;
                const double* w0 = V.w0 + (size_t)j * 7;
                const double* w = V.w + (size_t)j * 7;
                double c6 = 0.0, dc6 = 0.0;
                for (int b = 0; b < nr; ++b) {
                    c6 += g0[b] * w0[b];
                    dc6 += dg[b] * w[b];
                }
                const double r4r2 = 3.0 * szi * V.szr[j];
                const double t = a1 * sqrt(r4r2) + a2;
                const double r0sq = t * t;
                const double zz = zi * V.zeta[j];
                const double r2 = r * r, r6 = r2 * r2 * r2, r06 = r0sq * r0sq * r0sq;
                const double t6 = 1.0 / (r6 + r06);
                const double t8 = 1.0 / (r6 * r2 + r06 * r0sq);
                const double sum = t6 + 2.0 * r4r2 * t8;
                ed += -c6 * sum * zz;
                const double d6 = -6.0 * r2 * r2 * t6 * t6, d8 = -8.0 * r2 * r2 * r2 * t8 * t8;
                dEdr += -c6 * zz * (d6 + 2.0 * r4r2 * d8) * r;
                dcn -= dc6 * sum * zz;
            }
            if (dEdr != 0.0) {
                const double f = dEdr / r;
                gx += f * dx; gy += f * dy; gz += f * dz;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            gx += __shfl_down_sync(0xffffffffu, gx, o);
            gy += __shfl_down_sync(0xffffffffu, gy, o);
            gz += __shfl_down_sync(0xffffffffu, gz, o);
            dcn += __shfl_down_sync(0xffffffffu, dcn, o);
        }
        if (lane == 0) {
            V.grad[3 * i] += gx;
            V.grad[3 * i + 1] += gy;
            V.grad[3 * i + 2] += gz;
            V.dEdcn[i] += dcn;
        }
    }
    block_add(0.5 * ec, V.E + T_COUL);
    block_add(0.5 * ed, V.E + T_DISP);
}

// ------------------------------------------------------------------------------------
// Coulomb self terms and the CN-chain weight v = dE/dCN - q cnf/(2 sqrt CN)
// (ff_workspace.cpp:415-536)
// ------------------------------------------------------------------------------------
__global__ void k_post(View V)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < V.n) {
        const double q = V.q[i], cn = fmax(V.cn[i], 0.0);
        if (V.n >= 2 && V.alpeeq[i] > 0.0) {
            const double chi = V.chi_base[i] + V.cnf[i] * sqrt(cn);
            e = -q * chi + 0.5 * q * q * (V.gam[i] + 0.797884560802865 / sqrt(V.alpeeq[i]));
        }
        V.v[i] = V.dEdcn[i] - q * V.cnf[i] / (2.0 * sqrt(cn) + 1e-16);
    }
    block_add(e, V.E + T_COUL);
}

// CN chain rule: grad_i += sum_j dS_ij/dr (dlog_i v_i + dlog_j v_j) (x_i - x_j)/r
// over the 6 bohr neighbours (gfnff_method.cpp:5837-6260, forcefieldthread.h:80-109)
__global__ void __launch_bounds__(kBlock) k_cn_chain(View V)
{
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= V.n) return;
    const double4 pi = V.pos[i];
    const double ri = V.rcov_cn[i];
    const double ui = V.dlog[i] * V.v[i];
    const double kn = -7.5, sqrtpi = 1.77245385091;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int j = lane; j < V.n; j += 32) {
        if (j == i) continue;
        const double4 pj = V.pos[j];
        const double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < 36.0)) continue;
        const double r = sqrt(d2);
        const double rs = ri + V.rcov_cn[j];
        const double dr = (r - rs) / rs;
        const double de = (kn / sqrtpi) * exp(-kn * kn * dr * dr) / rs;
        const double f = -(de / r) * (ui + V.dlog[j] * V.v[j]);
        gx += f * dx; gy += f * dy; gz += f * dz;
    }
    for (int o = 16; o > 0; o >>= 1) {
        gx += __shfl_down_sync(0xffffffffu, gx, o);
        gy += __shfl_down_sync(0xffffffffu, gy, o);
        gz += __shfl_down_sync(0xffffffffu, gz, o);
    }
    if (lane == 0) {
        V.grad[3 * i] += gx;
        V.grad[3 * i + 1] += gy;
        V.grad[3 * i + 2] += gz;
    }
}

// total energy, finiteness check, optional copies to caller buffers
__global__ void k_finish(View V, const int* potrf_info, double e0, double* out_e, double* out_grad)
{
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < 3 * V.n; k += blockDim.x) {
        const double g = V.grad[k];
        if (!isfinite(g)) bad = 1;
        if (out_grad) out_grad[k] = g;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = e0;
        for (int t = 0; t < T_TOTAL; ++t) tot += V.E[t];
        V.E[T_TOTAL] = tot;
        if (out_e) *out_e = tot;
        int st = 0;
        if (potrf_info && *potrf_info != 0) st = GFNFF_NOT_SPD;
        else if (!isfinite(tot) || bad) st = GFNFF_NONFINITE;
        *V.status = st;
    }
}

// device enumeration of the D4 pair list at the setup geometry (topology check)
__global__ void k_disp_count(int n, const double4* pos0, unsigned long long* cnt, int2* out, unsigned long long cap)
{
    const int i = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j <= i || j >= n) return;
    if (d2_exact(pos0[i], pos0[j]) <= 3600.0) {
        const unsigned long long s = atomicAdd(cnt, 1ull);
        if (out && s < cap) out[s] = make_int2(i, j);
    }
}

inline int nblk(long n, int b = kBlock) { return (int)((n + b - 1) / b); }

}  // namespace

// ====================================================================================
// Engine implementation
// ====================================================================================
struct Engine::Impl {
    EngineOptions opt;
    cudaStream_t stream = nullptr;
    cusolverDnHandle_t sol = nullptr;
    int n = 0, nfrag = 0, K = 0, nred = 0;
    double e0 = 0.0;
    // model
    DBuf<double4> pos, pos0, hbref;
    DBuf<double> rcov_cn, rcov43, rcov_d3, chi_base, cnf, gam, alpeeq, qa, refcn, w0, g0, c6ref, zeta, szr;
    DBuf<int> slot, nref;
    // EEQ structure
    DBuf<int> red2atom, atom2red, anchor, frag_off, frag_atoms;
    DBuf<double> q0;
    // bonded lists
    DBuf<int> b_i, b_j, b_h, b_off, b_hb;
    DBuf<double> b_fc, b_al, b_r0i, b_r0j, b_cki, b_ckj, b_sh, b_ff;
    DBuf<int> a_i, a_j, a_k;
    DBuf<double> a_fc, a_th;
    DBuf<int> t_i, t_j, t_k, t_l;
    DBuf<double> t_V, t_n, t_p;
    DBuf<int> s_i, s_j, s_k, s_l;
    DBuf<double> s_e;
    DBuf<int> v_i, v_j, v_k, v_l, v_t;
    DBuf<double> v_fc, v_om;
    DBuf<int> at_i, at_j, at_k;
    DBuf<double> at_c9, at_r0ij, at_r0ik, at_r0jk, at_sc;
    DBuf<int> ba_i, ba_j, ba_k;
    DBuf<double> ba_c9;
    DBuf<int> h_a, h_h, h_b, h_c, h_pc, h_nbo, h_nb, h_nco, h_nc, h_nfl;
    DBuf<double> h_ba, h_bb, h_aa, h_ab, h_QH, h_QA, h_QB, h_rv, h_zlp;
    DBuf<int> x_a, x_x, x_b;
    DBuf<double> x_pre, x_rv;
    DBuf<int> r_off, r_j;
    DBuf<double> r_al, r_ab;
    DBuf<unsigned char> r_kind;
    // per step
    DBuf<double> cnraw, cn, dlog, w, dw, hg, hdg, q, dEdcn, v, grad, E, A, M, rvec, bvec, xyz_stage, msd;
    DBuf<double> work;
    DBuf<int> info, info2, status, ipiv;
    int lwork = 0;
    bool use_lu = false;   // reduced EEQ matrix not positive definite: pivoted LU instead
    bool timing = false;
    cudaEvent_t ev[Engine::kNumPhases + 1] = {};
    void mark(int k)
    {
        if (timing) CK(cudaEventRecord(ev[k], stream));
    }
    int nb = 0, na = 0, nt = 0, ns = 0, ninv = 0, natm = 0, nbatm = 0, nhb = 0, nxb = 0;

    View view() const
    {
        View V;
        V.n = n; V.nfrag = nfrag; V.K = K; V.nred = nred;
        V.pos = pos.p; V.pos0 = pos0.p; V.rcov_cn = rcov_cn.p; V.rcov43 = rcov43.p; V.rcov_d3 = rcov_d3.p;
        V.chi_base = chi_base.p; V.cnf = cnf.p; V.gam = gam.p; V.alpeeq = alpeeq.p; V.qa = qa.p;
        V.slot = slot.p; V.nref = nref.p; V.refcn = refcn.p; V.w0 = w0.p; V.g0 = g0.p; V.c6ref = c6ref.p;
        V.zeta = zeta.p; V.szr = szr.p;
        V.cnraw = cnraw.p; V.cn = cn.p; V.dlog = dlog.p; V.w = w.p; V.dw = dw.p; V.hg = hg.p; V.hdg = hdg.p;
        V.q = q.p; V.dEdcn = dEdcn.p; V.v = v.p; V.grad = grad.p; V.E = E.p; V.status = status.p;
        return V;
    }
};

Engine::Engine(const EngineOptions& opt) : p_(new Impl)
{
    p_->opt = opt;
    CK(cudaSetDevice(opt.device));
    CK(cudaStreamCreateWithFlags(&p_->stream, cudaStreamNonBlocking));
    CS(cusolverDnCreate(&p_->sol));
    CS(cusolverDnSetStream(p_->sol, p_->stream));
}

const char* const Engine::kPhaseNames[] = {"positions", "cn", "d4_weights", "eeq_matrix", "eeq_reduce",
                                           "eeq_factor_solve", "bonded", "hbonds", "repulsion", "pairs",
                                           "post_chain", "finish"};

void Engine::set_timing(bool on)
{
    if (on && !p_->ev[0])
        for (int k = 0; k <= kNumPhases; ++k) CK(cudaEventCreate(&p_->ev[k]));
    p_->timing = on;
}

std::vector<double> Engine::phase_ms()
{
    std::vector<double> out(kNumPhases, 0.0);
    if (!p_->timing) return out;
    CK(cudaEventSynchronize(p_->ev[kNumPhases]));
    for (int k = 0; k < kNumPhases; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p_->ev[k], p_->ev[k + 1]));
        out[k] = ms;
    }
    return out;
}

Engine::~Engine()
{
    for (auto& e : p_->ev)
        if (e) cudaEventDestroy(e);
    if (p_->sol) cusolverDnDestroy(p_->sol);
    if (p_->stream) cudaStreamDestroy(p_->stream);
}

static std::vector<double4> to4(const std::vector<double>& x)
{
    std::vector<double4> o(x.size() / 3);
    for (size_t i = 0; i < o.size(); ++i) o[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0);
    return o;
}

void Engine::upload_hbxb(const Model& m)
{
    Impl& P = *p_;
    // bonds carry the HB modulation data
    {
        std::vector<int> bi, bj, bh, off{0}, hb;
        std::vector<double> fc, al, r0i, r0j, cki, ckj, sh, ff;
        std::map<int, std::vector<int>> byH;
        for (auto& e : m.bond_hb) byH[e.h].insert(byH[e.h].end(), e.b_atoms.begin(), e.b_atoms.end());
        for (auto& b : m.bonds) {
            bi.push_back(b.i); bj.push_back(b.j);
            fc.push_back(b.fc); al.push_back(b.alpha); r0i.push_back(b.r0_base_i); r0j.push_back(b.r0_base_j);
            cki.push_back(b.cnfak_i); ckj.push_back(b.cnfak_j); sh.push_back(b.rabshift); ff.push_back(b.ff);
            int H = b.nr_hb >= 1 ? b.hb_h : -1;
            bh.push_back(H);
            if (H >= 0) { auto& L = byH[H]; hb.insert(hb.end(), L.begin(), L.end()); }
            off.push_back((int)hb.size());
        }
        P.nb = (int)m.bonds.size();
        P.b_i.upload(bi); P.b_j.upload(bj); P.b_h.upload(bh); P.b_off.upload(off); P.b_hb.upload(hb);
        P.b_fc.upload(fc); P.b_al.upload(al); P.b_r0i.upload(r0i); P.b_r0j.upload(r0j);
        P.b_cki.upload(cki); P.b_ckj.upload(ckj); P.b_sh.upload(sh); P.b_ff.upload(ff);
    }
    {
        std::vector<int> a, h, b, c, pc, nbo{0}, nb, nco{0}, nc, nfl;
        std::vector<double> ba, bb, aa, ab, QH, QA, QB, rv, zlp;
        auto qs = [](double q, double st, double sf) { const double e = std::exp(st * q); return e / (e + sf); };
        for (auto& t : m.hbonds) {
            a.push_back(t.a); h.push_back(t.h); b.push_back(t.b); c.push_back(t.case_type); pc.push_back(t.parent_c);
            nb.insert(nb.end(), t.nb_b.begin(), t.nb_b.end()); nbo.push_back((int)nb.size());
            if (t.case_type == 3) nc.insert(nc.end(), t.nb_c.begin(), t.nb_c.end());
            nco.push_back((int)nc.size());
            ba.push_back(t.bas_a); bb.push_back(t.bas_b); aa.push_back(t.aci_a); ab.push_back(t.aci_b);
            QH.push_back(qs(t.q_h, 15.0, 1.0)); QA.push_back(qs(-t.q_a, 15.0, 1.0)); QB.push_back(qs(-t.q_b, 15.0, 1.0));
            rv.push_back(m.rvdw[t.a] + m.rvdw[t.b]);
            const int zb = m.Z[t.b];
            zlp.push_back((zb >= 1 && zb <= 86) ? gfnff_tables::repz[zb - 1] : 1.0);
            nfl.push_back((zb == 7 && t.nb_b.size() == 1) ? 1 : 0);
        }
        P.nhb = (int)m.hbonds.size();
        P.h_a.upload(a); P.h_h.upload(h); P.h_b.upload(b); P.h_c.upload(c); P.h_pc.upload(pc);
        P.h_nbo.upload(nbo); P.h_nb.upload(nb); P.h_nco.upload(nco); P.h_nc.upload(nc);
        P.h_ba.upload(ba); P.h_bb.upload(bb); P.h_aa.upload(aa); P.h_ab.upload(ab);
        P.h_QH.upload(QH); P.h_QA.upload(QA); P.h_QB.upload(QB); P.h_rv.upload(rv); P.h_zlp.upload(zlp);
        P.h_nfl.upload(nfl);
    }
    {
        std::vector<int> a, x, b;
        std::vector<double> pre, rv;
        auto qs = [](double q, double st, double sf) { const double e = std::exp(st * q); return e / (e + sf); };
        for (auto& t : m.xbonds) {
            a.push_back(t.a); x.push_back(t.x); b.push_back(t.b);
            pre.push_back(-qs(-t.q_b, 15.0, 0.03) * t.aci_x * qs(t.q_x, 15.0, 0.03));
            rv.push_back(m.rvdw[t.a] + m.rvdw[t.b]);
        }
        P.nxb = (int)m.xbonds.size();
        P.x_a.upload(a); P.x_x.upload(x); P.x_b.upload(b); P.x_pre.upload(pre); P.x_rv.upload(rv);
    }
}

void Engine::upload(const Model& m)
{
    Impl& P = *p_;
    CK(cudaSetDevice(P.opt.device));
    const int n = m.n;
    P.n = n;
    P.nfrag = m.nfrag;
    P.K = (int)m.present_Z.size();
    P.e0 = m.e0;
    P.pos0.upload(to4(m.xyz_setup));
    P.hbref.upload(to4(m.xyz_setup));
    P.pos.alloc(n);
    P.rcov_cn.upload(m.rcov_cn);
    std::vector<double> r43(n);
    for (int i = 0; i < n; ++i) r43[i] = m.rcov_d3[i] * (4.0 / 3.0);
    P.rcov43.upload(r43);
    P.rcov_d3.upload(m.rcov_d3);
    P.chi_base.upload(m.chi_base); P.cnf.upload(m.cnf); P.gam.upload(m.gam); P.alpeeq.upload(m.alpeeq);
    P.qa.upload(m.qa); P.slot.upload(m.slot); P.nref.upload(m.nref); P.refcn.upload(m.refcn);
    P.w0.upload(m.w_setup); P.c6ref.upload(m.c6ref); P.zeta.upload(m.zeta); P.szr.upload(m.sqrt_zr4r2);
    {   // frozen half contraction at the setup weights (d4param_generator.cpp:1235-1290)
        const int K = P.K;
        std::vector<double> g((size_t)n * K * 7, 0.0);
        for (int i = 0; i < n; ++i)
            for (int s = 0; s < K; ++s) {
                const double* C = &m.c6ref[(((size_t)m.slot[i] * K + s) * 7) * 7];
                for (int b = 0; b < 7; ++b) {
                    double v = 0.0;
                    for (int a = 0; a < m.nref[i]; ++a) v += m.w_setup[(size_t)i * 7 + a] * C[a * 7 + b];
                    g[((size_t)i * K + s) * 7 + b] = v;
                }
            }
        P.g0.upload(g);
    }
    // EEQ null-space structure
    {
        std::vector<int> anchor(n, -1), first(m.nfrag, -1), cntf(m.nfrag, 0);
        for (int i = 0; i < n; ++i) { const int f = m.frag[i]; if (first[f] < 0) first[f] = i; ++cntf[f]; }
        std::vector<int> a2r(n), r2a;
        std::vector<double> q0(n);
        for (int i = 0; i < n; ++i) {
            const int f = m.frag[i];
            anchor[i] = first[f];
            q0[i] = m.qfrag[f] / (double)cntf[f];
            if (i == first[f]) a2r[i] = -f - 1;
            else { a2r[i] = (int)r2a.size(); r2a.push_back(i); }
        }
        std::vector<int> off(m.nfrag + 1, 0), fa(n);
        for (int f = 0; f < m.nfrag; ++f) off[f + 1] = off[f] + cntf[f];
        std::vector<int> pos = off;
        for (int i = 0; i < n; ++i) fa[pos[m.frag[i]]++] = i;
        P.nred = (int)r2a.size();
        P.anchor.upload(anchor); P.atom2red.upload(a2r); P.red2atom.upload(r2a);
        P.frag_off.upload(off); P.frag_atoms.upload(fa); P.q0.upload(q0);
    }
    // term lists
    {
        std::vector<int> i, j, k;
        std::vector<double> fc, th;
        for (auto& a : m.angles) { i.push_back(a.i); j.push_back(a.j); k.push_back(a.k); fc.push_back(a.fc); th.push_back(a.theta0); }
        P.na = (int)m.angles.size();
        P.a_i.upload(i); P.a_j.upload(j); P.a_k.upload(k); P.a_fc.upload(fc); P.a_th.upload(th);
    }
    {
        std::vector<int> i, j, k, l;
        std::vector<double> V, nn, ph;
        for (auto& t : m.torsions) { i.push_back(t.i); j.push_back(t.j); k.push_back(t.k); l.push_back(t.l); V.push_back(t.V); nn.push_back(t.n); ph.push_back(t.phi0); }
        P.nt = (int)m.torsions.size();
        P.t_i.upload(i); P.t_j.upload(j); P.t_k.upload(k); P.t_l.upload(l); P.t_V.upload(V); P.t_n.upload(nn); P.t_p.upload(ph);
    }
    {
        std::vector<int> i, j, k, l;
        std::vector<double> e;
        for (auto& t : m.storsions) { i.push_back(t.i); j.push_back(t.j); k.push_back(t.k); l.push_back(t.l); e.push_back(t.erefhalf); }
        P.ns = (int)m.storsions.size();
        P.s_i.upload(i); P.s_j.upload(j); P.s_k.upload(k); P.s_l.upload(l); P.s_e.upload(e);
    }
    {
        std::vector<int> i, j, k, l, ty;
        std::vector<double> fc, om;
        for (auto& t : m.inversions) { i.push_back(t.i); j.push_back(t.j); k.push_back(t.k); l.push_back(t.l); ty.push_back(t.type); fc.push_back(t.fc); om.push_back(t.omega0); }
        P.ninv = (int)m.inversions.size();
        P.v_i.upload(i); P.v_j.upload(j); P.v_k.upload(k); P.v_l.upload(l); P.v_t.upload(ty); P.v_fc.upload(fc); P.v_om.upload(om);
    }
    {
        std::vector<int> i, j, k;
        std::vector<double> c9, r0ij, r0ik, r0jk, sc;
        for (auto& t : m.atm) {
            i.push_back(t.i); j.push_back(t.j); k.push_back(t.k);
            c9.push_back(std::sqrt(std::fabs(t.c6ij * t.c6ik * t.c6jk)));
            auto r0 = [&](int a, int b) { return 0.58 * std::sqrt(3.0 * m.rcov_d3[a] * m.rcov_d3[b]) + 4.80; };
            r0ij.push_back(r0(t.i, t.j)); r0ik.push_back(r0(t.i, t.k)); r0jk.push_back(r0(t.j, t.k));
            sc.push_back(t.scale);
        }
        P.natm = (int)m.atm.size();
        P.at_i.upload(i); P.at_j.upload(j); P.at_k.upload(k); P.at_c9.upload(c9);
        P.at_r0ij.upload(r0ij); P.at_r0ik.upload(r0ik); P.at_r0jk.upload(r0jk); P.at_sc.upload(sc);
    }
    {
        std::vector<int> i, j, k;
        std::vector<double> c9;
        auto fq = [&](int a) { return std::min(std::max(1.0 - 3.0 * m.qa[a], -4.0), 4.0); };
        for (auto& t : m.batm) {
            i.push_back(t.i); j.push_back(t.j); k.push_back(t.k);
            c9.push_back(fq(t.i) * fq(t.j) * fq(t.k) * t.zi * t.zj * t.zk);
        }
        P.nbatm = (int)m.batm.size();
        P.ba_i.upload(i); P.ba_j.upload(j); P.ba_k.upload(k); P.ba_c9.upload(c9);
    }
    {   // repulsion CSR, both directions
        std::vector<std::vector<std::tuple<int, double, double, unsigned char>>> rows(n);
        for (auto& r : m.rep_bonded) {
            rows[r.i].push_back({r.j, r.alpha, r.repab, 0});
            rows[r.j].push_back({r.i, r.alpha, r.repab, 0});
        }
        for (auto& r : m.rep_nonbonded) {
            rows[r.i].push_back({r.j, r.alpha, r.repab, 1});
            rows[r.j].push_back({r.i, r.alpha, r.repab, 1});
        }
        std::vector<int> off{0}, jj;
        std::vector<double> al, ab;
        std::vector<unsigned char> kd;
        for (int a = 0; a < n; ++a) {
            for (auto& e : rows[a]) { jj.push_back(std::get<0>(e)); al.push_back(std::get<1>(e)); ab.push_back(std::get<2>(e)); kd.push_back(std::get<3>(e)); }
            off.push_back((int)jj.size());
        }
        P.r_off.upload(off); P.r_j.upload(jj); P.r_al.upload(al); P.r_ab.upload(ab); P.r_kind.upload(kd);
    }
    upload_hbxb(m);
    // per-step buffers
    P.cnraw.alloc(n); P.cn.alloc(n); P.dlog.alloc(n); P.w.alloc((size_t)n * 7); P.dw.alloc((size_t)n * 7);
    P.hg.alloc((size_t)n * P.K * 7); P.hdg.alloc((size_t)n * P.K * 7);
    P.q.alloc(n); P.dEdcn.alloc(n); P.v.alloc(n); P.grad.alloc(3 * (size_t)n); P.E.alloc(16);
    P.A.alloc((size_t)n * n); P.M.alloc((size_t)std::max(1, P.nred) * std::max(1, P.nred));
    P.rvec.alloc(n); P.bvec.alloc(std::max(1, P.nred)); P.xyz_stage.alloc(3 * (size_t)n); P.msd.alloc(1);
    P.info.alloc(1); P.info2.alloc(1); P.status.alloc(1);
    P.use_lu = false;
    if (P.nred > 0) {
        int l1 = 0, l2 = 0;
        CS(cusolverDnDpotrf_bufferSize(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, P.M.p, P.nred, &l1));
        CS(cusolverDnDgetrf_bufferSize(P.sol, P.nred, P.nred, P.M.p, P.nred, &l2));
        P.lwork = std::max(l1, l2);
        P.work.alloc(std::max(1, P.lwork));
        P.ipiv.alloc(P.nred);
    }
    CK(cudaMemset(P.info.p, 0, sizeof(int)));
    CK(cudaDeviceSynchronize());
    // The reduced EEQ matrix is indefinite for some systems (hydrogen has a negative
    // hardness); curcuma then falls back from its Cholesky to an LU solve
    // (eeq_solver.cpp:1448-2086).  Probe once at the setup geometry and keep the
    // choice for this molecule; enqueue() switches later if a geometry turns it.
    if (P.nred > 0) {
        DBuf<double> x;
        std::vector<double> h(m.xyz_setup);
        x.upload(h);
        enqueue(x.p, true);
        int st = 0;
        fetch(nullptr, nullptr, &st, nullptr);
        if (st == GFNFF_NOT_SPD) P.use_lu = true;
    }
}

bool Engine::switch_to_lu()
{
    if (p_->use_lu || p_->nred == 0) return false;
    p_->use_lu = true;
    return true;
}

void Engine::enqueue(const double* d_xyz, bool bohr)
{
    Impl& P = *p_;
    cudaStream_t s = P.stream;
    const int n = P.n;
    View V = P.view();
    P.mark(0);
    CK(cudaMemsetAsync(P.grad.p, 0, 3 * (size_t)n * sizeof(double), s));
    CK(cudaMemsetAsync(P.dEdcn.p, 0, (size_t)n * sizeof(double), s));
    CK(cudaMemsetAsync(P.msd.p, 0, sizeof(double), s));
    const double scale = bohr ? 1.0 : kAngToBohr;
    k_positions<<<nblk(n), kBlock, 0, s>>>(n, d_xyz, scale, P.pos.p, P.hbref.p, P.msd.p, P.E.p, P.status.p);
    P.mark(1);
    k_cn<<<nblk((long)n * 32), kBlock, 0, s>>>(V);
    P.mark(2);
    k_d4_weights<<<nblk(n), kBlock, 0, s>>>(V);
    // EEQ
    {
        P.mark(3);
        dim3 g(nblk(n), n);
        k_eeq_matrix<<<g, kBlock, 0, s>>>(V, P.A.p);
        k_eeq_residual<<<nblk((long)n * 32), kBlock, 0, s>>>(V, P.A.p, P.q0.p, P.rvec.p);
        P.mark(4);
        if (P.nred > 0) {
            dim3 g2(nblk(P.nred), P.nred);
            k_eeq_reduce<<<g2, kBlock, 0, s>>>(V, P.A.p, P.red2atom.p, P.anchor.p, P.rvec.p, P.M.p, P.bvec.p);
        }
        P.mark(5);
        if (P.nred > 0) {
            if (!P.use_lu) {
                CS(cusolverDnDpotrf(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, P.M.p, P.nred, P.work.p, P.lwork, P.info.p));
                CS(cusolverDnDpotrs(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, 1, P.M.p, P.nred, P.bvec.p, P.nred, P.info2.p));
            } else {
                CS(cusolverDnDgetrf(P.sol, P.nred, P.nred, P.M.p, P.nred, P.work.p, P.ipiv.p, P.info.p));
                CS(cusolverDnDgetrs(P.sol, CUBLAS_OP_N, P.nred, 1, P.M.p, P.nred, P.ipiv.p, P.bvec.p, P.nred, P.info2.p));
            }
        }
        k_eeq_expand<<<nblk(n), kBlock, 0, s>>>(V, P.q0.p, P.atom2red.p, P.frag_off.p, P.frag_atoms.p, P.anchor.p, P.bvec.p);
    }
    P.mark(6);
    if (P.nb) {
        BondSoA B{P.nb, P.b_i.p, P.b_j.p, P.b_h.p, P.b_off.p, P.b_hb.p, P.b_fc.p, P.b_al.p,
                  P.b_r0i.p, P.b_r0j.p, P.b_cki.p, P.b_ckj.p, P.b_sh.p, P.b_ff.p};
        k_bonds<<<nblk(P.nb), kBlock, 0, s>>>(V, B);
    }
    if (P.na) k_angles<<<nblk(P.na), kBlock, 0, s>>>(V, AngleSoA{P.na, P.a_i.p, P.a_j.p, P.a_k.p, P.a_fc.p, P.a_th.p});
    if (P.nt) k_torsions<<<nblk(P.nt), kBlock, 0, s>>>(V, TorsSoA{P.nt, P.t_i.p, P.t_j.p, P.t_k.p, P.t_l.p, P.t_V.p, P.t_n.p, P.t_p.p}, 0);
    if (P.ns) k_torsions<<<nblk(P.ns), kBlock, 0, s>>>(V, TorsSoA{P.ns, P.s_i.p, P.s_j.p, P.s_k.p, P.s_l.p, P.s_e.p, nullptr, nullptr}, 1);
    if (P.ninv) k_inversions<<<nblk(P.ninv), kBlock, 0, s>>>(V, InvSoA{P.ninv, P.v_i.p, P.v_j.p, P.v_k.p, P.v_l.p, P.v_t.p, P.v_fc.p, P.v_om.p});
    if (P.natm) k_atm<<<nblk(P.natm), kBlock, 0, s>>>(V, TripSoA{P.natm, P.at_i.p, P.at_j.p, P.at_k.p, P.at_c9.p, P.at_r0ij.p, P.at_r0ik.p, P.at_r0jk.p, P.at_sc.p});
    if (P.nbatm) k_batm<<<nblk(P.nbatm), kBlock, 0, s>>>(V, TripSoA{P.nbatm, P.ba_i.p, P.ba_j.p, P.ba_k.p, P.ba_c9.p, nullptr, nullptr, nullptr, nullptr});
    P.mark(7);
    if (P.nhb) {
        HBSoA H{P.nhb, P.h_a.p, P.h_h.p, P.h_b.p, P.h_c.p, P.h_pc.p, P.h_nbo.p, P.h_nb.p, P.h_nco.p, P.h_nc.p,
                P.h_ba.p, P.h_bb.p, P.h_aa.p, P.h_ab.p, P.h_QH.p, P.h_QA.p, P.h_QB.p, P.h_rv.p, P.h_zlp.p, P.h_nfl.p};
        k_hbonds<<<nblk(P.nhb), kBlock, 0, s>>>(V, H);
    }
    if (P.nxb) k_xbonds<<<nblk(P.nxb), kBlock, 0, s>>>(V, XBSoA{P.nxb, P.x_a.p, P.x_x.p, P.x_b.p, P.x_pre.p, P.x_rv.p});
    P.mark(8);
    k_repulsion<<<nblk((long)n * 32), kBlock, 0, s>>>(V, P.r_off.p, P.r_j.p, P.r_al.p, P.r_ab.p, P.r_kind.p);
    P.mark(9);
    k_pairs<<<nblk((long)n * 32), kBlock, 0, s>>>(V);
    P.mark(10);
    k_post<<<nblk(n), kBlock, 0, s>>>(V);
    k_cn_chain<<<nblk((long)n * 32), kBlock, 0, s>>>(V);
    P.mark(11);
    k_finish<<<1, 256, 0, s>>>(V, P.nred > 0 ? P.info.p : nullptr, P.e0, nullptr, nullptr);
    P.mark(12);
    CK(cudaGetLastError());
}

const double* Engine::d_terms() const { return p_->E.p; }
const double* Engine::d_grad() const { return p_->grad.p; }
const double* Engine::d_charges() const { return p_->q.p; }
const double* Engine::d_cn() const { return p_->cn.p; }
const int* Engine::d_status() const { return p_->status.p; }
const double* Engine::d_hb_msd() const { return p_->msd.p; }
double* Engine::d_xyz_scratch() { return p_->xyz_stage.p; }
void* Engine::stream() const { return (void*)p_->stream; }
int Engine::natoms() const { return p_->n; }
void Engine::sync() { CK(cudaStreamSynchronize(p_->stream)); }

void Engine::fetch(double* terms, double* grad, int* status, double* hb_msd)
{
    Impl& P = *p_;
    if (terms) CK(cudaMemcpyAsync(terms, P.E.p, kNumTerms * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (grad) CK(cudaMemcpyAsync(grad, P.grad.p, 3 * (size_t)P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (status) CK(cudaMemcpyAsync(status, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    if (hb_msd) CK(cudaMemcpyAsync(hb_msd, P.msd.p, sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
}

std::vector<int> Engine::device_dispersion_pairs()
{
    Impl& P = *p_;
    DBuf<unsigned long long> cnt;
    cnt.alloc(1);
    CK(cudaMemset(cnt.p, 0, sizeof(unsigned long long)));
    dim3 g(nblk(P.n), P.n);
    k_disp_count<<<g, kBlock, 0, P.stream>>>(P.n, P.pos0.p, cnt.p, nullptr, 0);
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, cnt.p, sizeof(c), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
    DBuf<int2> out;
    out.alloc(c);
    CK(cudaMemset(cnt.p, 0, sizeof(unsigned long long)));
    k_disp_count<<<g, kBlock, 0, P.stream>>>(P.n, P.pos0.p, cnt.p, out.p, c);
    std::vector<int2> h(c);
    if (c) CK(cudaMemcpyAsync(h.data(), out.p, c * sizeof(int2), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
    std::sort(h.begin(), h.end(), [](int2 a, int2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
    std::vector<int> v;
    v.reserve(2 * c);
    for (auto& p : h) { v.push_back(p.x); v.push_back(p.y); }
    return v;
}

void Engine::set_hb_reference(const double* xyz_bohr)
{
    std::vector<double> x(xyz_bohr, xyz_bohr + 3 * (size_t)p_->n);
    p_->hbref.upload(to4(x));
}

}  // namespace gfnff
