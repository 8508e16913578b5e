// Shared device-side definitions of the GFN-FF engine: error macros, device buffers,
// small vector helpers, the model view passed to every kernel and the per-molecule
// energy reduction.  Included inside namespace gfnff by engine.cu (one translation unit).
#pragma once

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
    T_HB, T_XB, T_ATM, T_BATM, T_SOLV, T_TOTAL
};

constexpr int kBlock = 128;
constexpr double kPi = 3.14159265358979323846;
// mixed form: the EEQ solution is refined until the FP64 residual ||b - M y||_inf of the
// reduced system is at most this (Hartree per charge unit)
constexpr double kRefineTol = 1e-10;

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
        if (v.empty()) return;
        CK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        // a copy from pageable memory may return before its DMA has landed, and the engine's
        // streams do not wait for the legacy stream: wait here
        CK(cudaStreamSynchronize(cudaStreamLegacy));
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
// 3-vector in the arithmetic type R of a kernel (double in the FP64 form, float for the
// FP32 arithmetic of the mixed form); D3 is the double version
template <class R>
struct V3 {
    R x, y, z;
};
using D3 = V3<double>;
__device__ __forceinline__ D3 mk(double x, double y, double z) { return {x, y, z}; }
template <class R>
__device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R>
__device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R>
__device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R>
__device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R>
__device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
__device__ __forceinline__ R nrm(V3<R> a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ D3 ld(const double4* p, int i)
{
    double4 v = p[i];
    return {v.x, v.y, v.z};
}
// position of atom i relative to the origin o, in the arithmetic type R (the FP64
// difference is taken first, so FP32 keeps the relative precision of short vectors)
template <class R>
__device__ __forceinline__ V3<R> ldr(const double4* p, int i, double4 o)
{
    const double4 v = p[i];
    return {(R)(v.x - o.x), (R)(v.y - o.y), (R)(v.z - o.z)};
}
template <class R>
__device__ __forceinline__ void agrad(double* g, int i, V3<R> v)
{
    atomicAdd(g + 3 * i, (double)v.x);
    atomicAdd(g + 3 * i + 1, (double)v.y);
    atomicAdd(g + 3 * i + 2, (double)v.z);
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
template <class R>
__device__ R dihedral(V3<R> ri, V3<R> rj, V3<R> rk, V3<R> rl, V3<R> g[4])
{
    using P3 = V3<R>;
    for (int a = 0; a < 4; ++a) g[a] = P3{R(0), R(0), R(0)};
    P3 v1 = rj - ri, v2 = rk - rj, v3 = rl - rk;
    P3 n1 = cross(v1, v2), n2 = cross(v2, v3);
    const R n1n = nrm(n1), n2n = nrm(n2), v2n = nrm(v2);
    if (n1n < R(1e-10) || n2n < R(1e-10) || v2n < R(1e-10)) return R(0);
    P3 h1 = (R(1) / n1n) * n1, h2 = (R(1) / n2n) * n2;
    const R cphi = dot(h1, h2);
    R sphi = (v2n * dot(h1, v3)) / n2n;
    sphi = fmax(R(-1), fmin(R(1), sphi));
    const R phi = atan2(sphi, cphi);
    const R nen = n1n * n2n * sin(phi);
    if (fabs(nen) < R(1e-14)) return phi;
    const R o = R(1) / nen;
    P3 rab = cross(n1, v2), rbb = cross(n2, v2), rac = cross(n1, v3), rbc = cross(n2, v3);
    P3 rba = cross(n2, v1), raa = cross(n1, v1);
    P3 rapb = v1 + v2, rbpc = v2 + v3;
    P3 rapba = cross(rapb, n1), rapbb = cross(rapb, n2), rbpca = cross(rbpc, n1), rbpcb = cross(rbpc, n2);
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
// periodic cell for the minimum-image convention (curcuma: cuda/gfnff_kernels.cu:92-119):
// h holds the lattice vectors a, b, c as columns, h[3*col + row] (bohr), hi its inverse in
// the same layout; on = 0 for an isolated system.  The displacement d = x_b - x_a becomes
// h (f - rint(f)) with the fractional f = hi d.
// ------------------------------------------------------------------------------------
struct Cell {
    double h[9], hi[9];
    int on;
};

__device__ __forceinline__ void mic(const Cell& c, double& dx, double& dy, double& dz)
{
    double fx = c.hi[0] * dx + c.hi[3] * dy + c.hi[6] * dz;
    double fy = c.hi[1] * dx + c.hi[4] * dy + c.hi[7] * dz;
    double fz = c.hi[2] * dx + c.hi[5] * dy + c.hi[8] * dz;
    fx -= rint(fx);
    fy -= rint(fy);
    fz -= rint(fz);
    dx = c.h[0] * fx + c.h[3] * fy + c.h[6] * fz;
    dy = c.h[1] * fx + c.h[4] * fy + c.h[7] * fz;
    dz = c.h[2] * fx + c.h[5] * fy + c.h[8] * fz;
}

// ------------------------------------------------------------------------------------
// device view of the model.  Atoms are stored in the engine's internal order (molecules
// contiguous, atoms of a molecule sorted along a Morton curve of the setup geometry);
// perm maps an internal index to the caller's index.
// ------------------------------------------------------------------------------------
struct View {
    int n, nfrag, K, nred, nmol;
    const int* mol;           // molecule of each atom
    const int2* jr;           // [first, last+1) atom range of the atom's molecule
    const int* perm;          // internal -> caller index
    const double4* pos;       // current geometry (bohr)
    const double4* pos0;      // setup geometry (bohr)
    const double* rcov_cn;
    const double* rcov43;     // 4/3 * covalent_rad_d3 (angle/torsion damping)
    const double* rcov_d3;
    const double* chi_base;
    const double* cnf;
    const double* gam;
    const double* alpeeq;
    const double* adiag;      // EEQ diagonal gam + sqrt(2/pi)/sqrt(alpha)
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
    double* E;                // nmol*16 term energies
    int* status;              // nmol
    // ALPB implicit solvation (brad null: gas phase): the Born matrix enters the EEQ matrix,
    // off-diagonal keps / f_GB(r, brad_a, brad_b) (P16), diagonal bdiag = keps / brad + 2 hbw
    const double* brad;
    const double* bdiag;
    double keps;
    // exact-gradient mode (see the gradient options of the C ABI)
    int exact;                // drop the D4 dC6/dCN term
    double* cfar;             // n: potential of the Coulomb pairs beyond 100 bohr, or null
    const double* u;          // n: EEQ charge response, or null
    // axis-aligned boxes of the runs of 32 consecutive atoms (current geometry)
    const double4* boxlo;
    const double4* boxhi;
    // periodic cell: the CN, bond, angle, HB, XB, repulsion, Coulomb and D4 pair distances
    // take the minimum image; torsions, inversions, ATM, BATM and the EEQ matrix do not
    Cell cell;
};

// minimum-image difference pos[b] - pos[a] in FP64 (the plain difference without a cell)
__device__ __forceinline__ D3 dmic(const View& V, int a, int b)
{
    const double4 x = V.pos[a], y = V.pos[b];
    double dx = y.x - x.x, dy = y.y - x.y, dz = y.z - x.z;
    if (V.cell.on) mic(V.cell, dx, dy, dz);
    return {dx, dy, dz};
}

// Adds v to term `term` of molecule `mol` (mol < 0: nothing to add).  Every thread of
// the block calls it.  Single-molecule models reduce over the block; batches reduce
// over the warp when its lanes share a molecule and add per thread otherwise.
__device__ __forceinline__ void eadd(const View& V, double v, int mol, int term)
{
    if (V.nmol == 1) {
        block_add(v, V.E + term);
        return;
    }
    const unsigned full = 0xffffffffu;
    const int m0 = __shfl_sync(full, mol, 0);
    if (__all_sync(full, mol == m0 || mol < 0)) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
        if ((threadIdx.x & 31) == 0 && m0 >= 0 && v != 0.0) atomicAdd(V.E + 16 * m0 + term, v);
    } else if (mol >= 0 && v != 0.0) {
        atomicAdd(V.E + 16 * mol + term, v);
    }
}

}  // namespace
