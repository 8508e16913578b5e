// Batched EEQ of the mixed form: FP32 Cholesky on the tensor cores with FP64 iterative
// refinement, one thread block per molecule (work items of k_eeq_batch).
//
// Replaces, for the mixed form, the per-molecule Cholesky of curcuma's Schur solve
// (eeq_solver.cpp:2087-2256, solveWithSchurCholesky): the reduced matrix M = B^T A B of the
// null-space substitution (k_eeq.cuh) is built from the geometry in FP64, once, and kept
//   * in FP64 in global scratch as 32 x 32 lower tiles (column-major inside a tile), for the
//     residuals of the refinement;
//   * in FP32 in shared memory as 16-column panels (rows 16q.. of panel q, 16 floats a row,
//     the four 4-float chunks of a row XOR-swizzled by bits 1-2 of the row so that the MMA
//     fragment loads of eight consecutive rows hit 32 different banks), with the right-hand
//     side appended as row nr.
// Blocked right-looking Cholesky per 16-column panel: one warp factors the 16 x 16 diagonal
// block in registers and forms its explicit inverse X = L11^-1; every thread solves one row of
// the panel below it (L21 = A21 X^T); the trailing lower triangle takes A22 -= L21 L21^T on the
// tensor cores (mma.sync m16n8k8 TF32, 3xTF32 split: a = a_hi + a_lo, products hi*hi + hi*lo +
// lo*hi with FP32 accumulation).  The appended row yields z = L^-1 b along the way.
// Refinement: y = L^-T z, then r = b - M y in FP64 from the FP64 tiles (every tile read once,
// its row and column contributions added), a correction solve with the FP32 factor
// (the diagonal blocks applied as their inverses), y += d, until ||r||_inf <= tol
// (1e-10: info 0) or kTcMaxRefine corrections were made (info 3, REFINE_NOT_CONVERGED).
// A pivot <= 0 of the FP32 factor gives info 1 (NOT_SPD).
// Included inside namespace gfnff by engine.cu (one translation unit), after k_eeq.cuh.
#pragma once

namespace {

constexpr int kTcNB = 16;                                    // panel width
constexpr int kTcMaxRows = 304;                              // nr rounded up to 16, at most
constexpr int kTcMaxRed = kTcMaxRows;                        // largest reduced system of this path
constexpr int kTcMaxPanels = (kTcMaxRed + kTcNB - 1) / kTcNB;
constexpr int kTcPanelFloats =
    kTcNB * (kTcMaxPanels * kTcMaxRows - kTcNB * kTcMaxPanels * (kTcMaxPanels - 1) / 2);
constexpr int kTcMaxRefine = 8;
// shared memory of one molecule (bytes): the staged atoms (later the diagonal-block
// inverses), b, y, the residual accumulator, the FP32 solve vector, the FP32 panels
constexpr int kTcStageBytes = (kStageDoubles + kStageInts / 2) * 8;
constexpr int kTcOffB = kTcStageBytes;
constexpr int kTcOffY = kTcOffB + kTcMaxRows * 8;
constexpr int kTcOffR = kTcOffY + kTcMaxRows * 8;
constexpr int kTcOffW = kTcOffR + kTcMaxRows * 8;
constexpr int kTcOffT = kTcOffW + kTcMaxRows * 4;
constexpr int kTcOffS = kTcOffT + 64;
constexpr int kTcSmemBytes = kTcOffS + kTcPanelFloats * 4;
static_assert(kTcMaxPanels * 256 * 4 <= kTcStageBytes, "diagonal inverses reuse the staging area");
static_assert(kTcMaxRed == kTcMaxRedFwd, "dispatch bound of k_eeq_batch");
static_assert(kTcSmemBytes <= 227 * 1024 - 1024, "tensor-core EEQ exceeds shared memory");

// element (r, c) of the FP32 panels, r >= 16 * (c / 16), r < nrp
struct TcPanels {
    float* S;
    int nrp;
    __device__ __forceinline__ int base(int q) const { return kTcNB * (q * nrp - kTcNB * q * (q - 1) / 2); }
    __device__ __forceinline__ int idx(int r, int c) const
    {
        const int q = c >> 4;
        return base(q) + (r - 16 * q) * 16 + ((c & 15) ^ (((r >> 1) & 3) << 2));
    }
    __device__ __forceinline__ float& operator()(int r, int c) const { return S[idx(r, c)]; }
};

__device__ __forceinline__ uint32_t tf32_bits(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// a = hi + lo with hi, lo representable in TF32
__device__ __forceinline__ void tf32_split(float a, uint32_t& hi, uint32_t& lo)
{
    hi = tf32_bits(a);
    lo = tf32_bits(a - __uint_as_float(hi));
}

// D = A B + D, A 16 x 8 (row), B 8 x 8 (col), TF32 in, FP32 accumulate
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A22 -= L21 L21^T for the rows [c0 + 16, nrows) and columns [c0 + 16, nr) (lower part) after
// panel c0 / 16 was factored.  A warp task is a 16 x 16 block (two n8 tiles) with K = 16 (two
// k8 steps), 3xTF32: 12 MMAs.  Entries above the diagonal inside diagonal 16 x 16 blocks are
// updated too; they exist in the panel storage and are never read.
__device__ void tc_trailing(const TcPanels& L, int nr, int nrows, int c0)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int first = c0 + 16;
    const int nrt = (nrows - first + 15) >> 4, nct = (nr - first + 15) >> 4;
    for (int task = warp; task < nrt * nct; task += nw) {
        const int a = task / nct, b = task % nct;
        if (b > a) continue;
        const int i0 = first + 16 * a, j0 = first + 16 * b;
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int k = c0 + 8 * s + t;
            const float v[4] = {L(i0 + g, k), L(i0 + g + 8, k), L(i0 + g, k + 4), L(i0 + g + 8, k + 4)};
#pragma unroll
            for (int e = 0; e < 4; ++e) tf32_split(-v[e], ah[s][e], al[s][e]);   // -L21: D = C - L L^T
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int jr = j0 + 8 * h;
            float d[4];
            const int cc = jr + 2 * t;
            d[0] = L(i0 + g, cc);
            d[1] = L(i0 + g, cc + 1);
            d[2] = L(i0 + g + 8, cc);
            d[3] = L(i0 + g + 8, cc + 1);
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int k = c0 + 8 * s + t;
                uint32_t bh[2], bl[2];
                tf32_split(L(jr + g, k), bh[0], bl[0]);
                tf32_split(L(jr + g, k + 4), bh[1], bl[1]);
                mma_tf32(d, al[s], bh);
                mma_tf32(d, ah[s], bl);
                mma_tf32(d, ah[s], bh);
            }
            L(i0 + g, cc) = d[0];
            L(i0 + g, cc + 1) = d[1];
            L(i0 + g + 8, cc) = d[2];
            L(i0 + g + 8, cc + 1) = d[3];
        }
    }
}

// Cholesky of the FP32 panels (rows and columns 0..nr-1; the last panel padded to 16 columns
// with the identity, so that every diagonal block is a full 16 x 16 SPD block); Xinv receives
// the inverse of every diagonal block (16 x 16 row-major).  Returns false (uniformly) when a
// pivot is not positive.  The diagonal block is straight-line code: every shuffle is executed
// by the whole warp, every register array is indexed by unrolled counters only.
__device__ bool tc_factor(const TcPanels& L, int nr, float* Xinv)
{
    __shared__ int s_bad;
    __shared__ float s_inv[16];
    const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
    const int Q = (nr + 15) >> 4;
    for (int p = 0; p < Q; ++p) {
        const int c0 = 16 * p;
        float* Pb = L.S + L.base(p);   // row c0 + i of the panel at Pb + 16 i (chunks swizzled)
        if (tid < 32) {
            // lane l < 16 (and l + 16, a copy) holds row c0 + l of the diagonal block
            const int row = lane & 15;
            const int sw = ((row >> 1) & 3) << 2;
            float* rp = Pb + 16 * row;
            float a[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = j <= row ? rp[j ^ sw] : 0.f;
            bool bad = false;
            float invd = 0.f;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float d = __shfl_sync(0xffffffffu, a[j], j);
                bad = bad || !(d > 0.f);
                const float is = rsqrtf(d);
                const float aj = (row == j ? d : a[j]) * is;   // L(row, j); rows above j hold zeros
                invd = row == j ? is : invd;
                a[j] = aj;
#pragma unroll
                for (int q = j + 1; q < 16; ++q) {
                    const float lqj = __shfl_sync(0xffffffffu, aj, q);
                    const float msk = row >= q ? 1.f : 0.f;   // a product, not a select: keeps a[] in registers
                    a[q] = fmaf(-aj * msk, lqj, a[q]);
                }
            }
            if (lane < 16) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (j <= row) rp[j ^ sw] = a[j];
                s_inv[lane] = invd;
            }
            if (lane == 0) s_bad = bad ? 1 : 0;
        }
        __syncthreads();
        if (s_bad) return false;
        // panel rows below the diagonal block: L21 = A21 L11^-T by forward substitution along
        // the row (L11 and 1/L_jj read as shared-memory broadcasts; two partial sums per entry)
        for (int r = c0 + 16 + tid; r < nr; r += nt) {
            float4* rp = reinterpret_cast<float4*>(Pb + 16 * (r - c0));
            const int sw = (r >> 1) & 3;
            float o[16];
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
                const float4 v = rp[ch ^ sw];
                o[4 * ch] = v.x; o[4 * ch + 1] = v.y; o[4 * ch + 2] = v.z; o[4 * ch + 3] = v.w;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float s0 = o[j], s1 = 0.f;
#pragma unroll
                for (int k = 0; k < j; ++k) {
                    const float ljk = Pb[16 * j + (k ^ (((j >> 1) & 3) << 2))];
                    if (k & 1) s1 = fmaf(-o[k], ljk, s1);
                    else s0 = fmaf(-o[k], ljk, s0);
                }
                o[j] = (s0 + s1) * s_inv[j];
            }
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) rp[ch ^ sw] = make_float4(o[4 * ch], o[4 * ch + 1], o[4 * ch + 2], o[4 * ch + 3]);
        }
        __syncthreads();
        if (c0 + 16 < nr) {
            tc_trailing(L, nr, nr, c0);
            __syncthreads();
        }
    }
    // X = L11^-1 of every diagonal block, a warp per block (lane k < 16 builds column k:
    // x_i = -(sum_{j<i} L_ij x_j) / L_ii, four partial sums), off the factorisation's path
    const int warp = tid >> 5, nw = nt >> 5;
    for (int p = warp; p < Q; p += nw) {
        const float* Pb = L.S + L.base(p);
        float* X = Xinv + 256 * p;
        if (lane < 16) {
            float x[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                float s4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int j = 0; j < i; ++j) s4[j & 3] = fmaf(Pb[16 * i + (j ^ (((i >> 1) & 3) << 2))], x[j], s4[j & 3]);
                const float sum = (s4[0] + s4[1]) + (s4[2] + s4[3]);
                const float rdi = 1.f / Pb[16 * i + (i ^ (((i >> 1) & 3) << 2))];
                x[i] = i == lane ? rdi : (i > lane ? -sum * rdi : 0.f);
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) X[16 * i + lane] = x[i];
        }
    }
    __syncthreads();
    return true;
}

// L w = w (forward) then L^T w = w (back) with the FP32 panels and the diagonal inverses, by
// one warp (warp-level synchronisation only); w has nr entries and is zero up to the end of
// the last panel.  Per panel: lanes 0..15 apply X (or X^T) to the panel's 16 entries, the
// result is broadcast by shuffles, and every lane updates its share of the rows below
// (forward: a float4 row of the panel per row) or of the columns before (back).
__device__ void tc_solve_warp(const TcPanels& L, const float* Xinv, int nr, float* w)
{
    const int lane = threadIdx.x & 31;
    const int Q = (nr + 15) >> 4;
    for (int p = 0; p < Q; ++p) {
        const int c0 = 16 * p;
        const float* X = Xinv + 256 * p;
        float t = 0.f;
        if (lane < 16) {
#pragma unroll
            for (int k = 0; k < 16; ++k) t = fmaf(X[16 * lane + k], w[c0 + k], t);   // X: zero above its diagonal
        }
        float tk[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) tk[k] = __shfl_sync(0xffffffffu, t, k);
        __syncwarp();
        if (lane < 16) w[c0 + lane] = t;
        const float4* Pb = reinterpret_cast<const float4*>(L.S + L.base(p));
        for (int r = c0 + 16 + lane; r < nr; r += 32) {   // rows below exist only under full panels
            const float4* rp = Pb + 4 * (r - c0);
            const int sw = (r >> 1) & 3;
            float s = 0.f;
#pragma unroll
            for (int ch = 0; ch < 4; ++ch) {
                const float4 v = rp[ch ^ sw];
                s = fmaf(v.x, tk[4 * ch], s);
                s = fmaf(v.y, tk[4 * ch + 1], s);
                s = fmaf(v.z, tk[4 * ch + 2], s);
                s = fmaf(v.w, tk[4 * ch + 3], s);
            }
            w[r] -= s;
        }
        __syncwarp();
    }
    for (int p = Q - 1; p >= 0; --p) {
        const int c0 = 16 * p;
        const float* X = Xinv + 256 * p;
        float t = 0.f;
        if (lane < 16) {
#pragma unroll
            for (int k = 0; k < 16; ++k) t = fmaf(X[16 * k + lane], w[c0 + k], t);   // X^T: zero below its diagonal
        }
        float tk[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) tk[k] = __shfl_sync(0xffffffffu, t, k);
        __syncwarp();
        if (lane < 16) w[c0 + lane] = t;
        for (int c = lane; c < c0; c += 32) {
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < 16; ++i) s = fmaf(L(c0 + i, c), tk[i], s);   // rows >= nr of the panel hold zeros
            w[c] -= s;
        }
        __syncwarp();
    }
}

// acc = M y over the FP64 lower tiles (T x T tile rows, tile (R, C) at G + 1024 (R(R+1)/2 + C),
// column-major inside): a warp per tile, lane = row; row sums directly, column sums by a
// butterfly over the warp (16 columns at a time).  acc must be zero on entry.
__device__ void tc_matvec64(const double* __restrict__ G, int nr, const double* y, double* acc)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int T = (nr + 31) >> 5;
    const int ntile = T * (T + 1) / 2;
    for (int tk = warp; tk < ntile; tk += nw) {
        int R = (int)((sqrtf(8.f * tk + 1.f) - 1.f) * 0.5f);
        while ((R + 1) * (R + 2) / 2 <= tk) ++R;
        while (R * (R + 1) / 2 > tk) --R;
        const int C = tk - R * (R + 1) / 2;
        const double* Tp = G + 1024ll * tk;
        const int r = 32 * R + lane;
        const bool rv = r < nr;
        const double yr = rv ? y[r] : 0.0;
        double rs = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double cs[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int cc = 16 * h + k, c = 32 * C + cc;
                const bool in = rv && c < nr && (R > C || cc <= lane);
                const double v = in ? Tp[32 * cc + lane] : 0.0;
                rs = fma(v, y[min(c, nr - 1)], rs);
                cs[k] = (R > C || cc < lane) ? v * yr : 0.0;
            }
            // lane l ends with the sum over all lanes of cs[l & 15]
#pragma unroll
            for (int s = 8; s >= 1; s >>= 1) {
                const bool up = lane & s;
#pragma unroll
                for (int i = 0; i < s; ++i) {
                    const double send = up ? cs[i] : cs[i + s];
                    const double keep = up ? cs[i + s] : cs[i];
                    cs[i] = keep + __shfl_xor_sync(0xffffffffu, send, s);
                }
            }
            cs[0] += __shfl_xor_sync(0xffffffffu, cs[0], 16);
            const int c = 32 * C + 16 * h + (lane & 15);
            if (lane < 16 && c < nr) atomicAdd(&acc[c], cs[0]);
        }
        if (rv) atomicAdd(&acc[r], rs);
    }
}

// one molecule of the batch: stage, build (FP64 tiles + FP32 panels), factor, refine
__device__ void tc_solve(const View& V, const EEQBatch& P, int m, double* S)
{
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    const int r0 = P.roff[m], nr = P.roff[m + 1] - r0;
    char* base = reinterpret_cast<char*>(S);
    double* b64 = reinterpret_cast<double*>(base + kTcOffB);
    double* y64 = reinterpret_cast<double*>(base + kTcOffY);
    double* acc = reinterpret_cast<double*>(base + kTcOffR);
    float* w = reinterpret_cast<float*>(base + kTcOffW);
    float* Xinv = reinterpret_cast<float*>(base);   // after the build (staging area)
    const int Q = (nr + 15) >> 4;
    const int nrp = 16 * Q;
    const TcPanels L{reinterpret_cast<float*>(base + kTcOffS), nrp};
    double* G = P.M64 + P.m64off[m];
    __shared__ double s_rmax[32];
    __shared__ int s_done;

    const MolStage MS = stage_molecule(V, P, r0, nr, S, reinterpret_cast<int*>(S + kStageDoubles));
    // zero the panels and the solve vector (padding rows and columns stay zero), b
    {
        float4* z4 = reinterpret_cast<float4*>(L.S);
        const int nz = L.base(Q) / 4;
        for (int k = tid; k < nz; k += nt) z4[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int k = tid; k < kTcMaxRows; k += nt) w[k] = 0.f;
        for (int k = tid; k < nr; k += nt) b64[k] = MS.rhs[k];
    }
    __syncthreads();
    // FP32 panels from the FP64 tiles (k_eeq_tc_tiles): a warp per tile, lane = row; the
    // padding columns of the last panel get a unit diagonal
    {
        const int T = (nr + 31) >> 5;
        const int ntile = T * (T + 1) / 2;
        for (int tk = warp; tk < ntile; tk += nw) {
            int R = (int)((sqrtf(8.f * tk + 1.f) - 1.f) * 0.5f);
            while ((R + 1) * (R + 2) / 2 <= tk) ++R;
            while (R * (R + 1) / 2 > tk) --R;
            const int C = tk - R * (R + 1) / 2;
            const double* Tp = G + 1024ll * tk;
            const int r = 32 * R + lane;
#pragma unroll 4
            for (int cc = 0; cc < 32; ++cc) {
                const int c = 32 * C + cc;
                if (r < nr && c < nr && r >= c) L(r, c) = (float)Tp[32 * cc + lane];
            }
        }
        for (int c = nr + tid; c < nrp; c += nt) L(c, c) = 1.f;
    }
    __syncthreads();
    bool ok = tc_factor(L, nr, Xinv);
    if (!ok) {
        if (tid == 0) P.info[m] = 1;
        return;
    }
    // y = M^-1 b with the FP32 factor (w is zero beyond nr: the fixed-length products of the
    // solves read to the end of the last panel)
    for (int c = tid; c < nr; c += nt) w[c] = (float)b64[c];
    __syncthreads();
    if (warp == 0) tc_solve_warp(L, Xinv, nr, w);
    __syncthreads();
    for (int c = tid; c < nr; c += nt) y64[c] = (double)w[c];
    int it = 0;
    bool conv = false;
    for (;;) {
        // r = b - M y (FP64)
        for (int c = tid; c < nr; c += nt) acc[c] = 0.0;
        __syncthreads();
        tc_matvec64(G, nr, y64, acc);
        __syncthreads();
        double mx = 0.0;
        for (int c = tid; c < nr; c += nt) {
            const double rr = b64[c] - acc[c];
            acc[c] = rr;
            mx = fmax(mx, fabs(rr));
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) s_rmax[warp] = mx;
        __syncthreads();
        if (tid == 0) {
            double g = 0.0;
            for (int k = 0; k < nw; ++k) g = fmax(g, s_rmax[k]);
            s_done = (g <= P.tol) ? 1 : (it >= kTcMaxRefine || !(g == g) ? 2 : 0);
        }
        __syncthreads();
        if (s_done) {
            conv = s_done == 1;
            break;
        }
        for (int c = tid; c < nr; c += nt) w[c] = (float)acc[c];
        __syncthreads();
        if (warp == 0) tc_solve_warp(L, Xinv, nr, w);
        __syncthreads();
        for (int c = tid; c < nr; c += nt) y64[c] += (double)w[c];
        ++it;
        __syncthreads();
    }
    double* y = P.y + r0;
    for (int c = tid; c < nr; c += nt) y[c] = y64[c];
    if (tid == 0) {
        P.info[m] = conv ? 0 : 3;
        if (P.refine) atomicMax(P.refine, it);
    }
}

// FP64 lower tiles of the reduced matrices of the tensor-core molecules, one block per
// 32 x 32 tile (the tile list {molecule, R, C} comes from the set-up), written column-major
// to M64 + m64off[m] + 1024 (R (R + 1) / 2 + C): the element formulas of eeq_aug (for a
// one-fragment molecule A(k, l) - A(k, a) - A(a, l) + A(a, a) with the anchor terms
// evaluated once per row and column), here at full occupancy instead of inside the
// one-block-per-molecule factorisation.
__global__ void __launch_bounds__(256) k_eeq_tc_tiles(View V, EEQBatch P, const int4* __restrict__ tiles)
{
    __shared__ double px[4][32], py[4][32], pz[4][32], pa[4][32], va[2][32];
    __shared__ int pid[4][32];
    __shared__ int s_single;
    const int4 t = tiles[blockIdx.x];
    const int m = t.x, R = t.y, C = t.z;
    const int r0 = P.roff[m], nr = P.roff[m + 1] - r0;
    const int tid = threadIdx.x;
    if (tid < 128) {
        const int w = tid >> 5, l = tid & 31;
        const int idx = (w < 2 ? 32 * R : 32 * C) + l;
        int a = -1;
        if (idx < nr) {
            const int k = P.red2atom[r0 + idx];
            a = (w & 1) ? P.anchor[k] : k;
        }
        pid[w][l] = a;
        if (a >= 0) {
            const double4 q = V.pos[a];
            px[w][l] = q.x; py[w][l] = q.y; pz[w][l] = q.z; pa[w][l] = V.alpeeq[a];
        }
    }
    if (tid == 0)
        s_single = P.anchor[P.red2atom[r0]] == P.anchor[P.red2atom[r0 + nr - 1]];
    __syncthreads();
    auto el = [&](int wa, int ia, int wb, int ib) {
        if (pid[wa][ia] == pid[wb][ib]) return V.adiag[pid[wa][ia]];
        const double dx = px[wa][ia] - px[wb][ib], dy = py[wa][ia] - py[wb][ib], dz = pz[wa][ia] - pz[wb][ib];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double s = pa[wa][ia] + pa[wb][ib];
        if (d2 >= 36.0 * s) return rsqrt(d2);
        const double r = sqrt(d2);
        return erf(r / sqrt(s)) / r;
    };
    const bool single = s_single;
    if (single && tid < 64) {   // A(k_r, a) of the rows (w = 0) and columns (w = 2)
        const int h = tid >> 5, l = tid & 31;
        if (pid[2 * h][l] >= 0) va[h][l] = el(2 * h, l, 2 * h + 1, l);
    }
    __syncthreads();
    double* Tp = P.M64 + P.m64off[m] + 1024ll * (R * (R + 1) / 2 + C);
    const int tx = tid & 31, ty = tid >> 5;
    const int r = 32 * R + tx;
    for (int cc = ty; cc < 32; cc += 8) {
        const int c = 32 * C + cc;
        double v = 0.0;
        if (r < nr && c < nr && r >= c) {
            if (single) v = ((el(0, tx, 2, cc) - va[0][tx]) - va[1][cc]) + V.adiag[pid[1][tx]];
            else v = el(0, tx, 2, cc) - el(0, tx, 3, cc) - el(1, tx, 2, cc) + el(1, tx, 3, cc);
        }
        Tp[32 * cc + tx] = v;
    }
}

}  // namespace
