// Block-Jacobi preconditioned conjugate gradients for the reduced EEQ system (FP64), in
// one persistent cooperative kernel.
//
// For systems of many small fragments (solvated clusters) the reduced matrix
// M = B^T A B is very well conditioned: the difference basis removes the long-range 1/r
// coupling, leaving dipole-like interactions (condition numbers near 2 for water
// clusters).  CG with the exact inverse of each fragment's diagonal block then reaches
// a residual of 1e-12 in about 15 iterations, each one symmetric matrix-vector product.
// Convergence is accepted only on the true residual b - M x, recomputed once the
// recursively updated residual meets the tolerance (CG restarts from it otherwise).
//
// Layout: M is the full symmetric reduced matrix, column-major with leading dimension
// lda (row r of M is contiguous as column r).  Every block owns a contiguous range of
// rows that covers whole preconditioner blocks; the search direction p is replicated in
// every block's shared memory and updated redundantly (identical arithmetic in every
// block), so one iteration needs two grid barriers.  Barrier waits are bounded; a wait
// that gives up sets info = 2, no convergence within max_iter sets info = 3.
// Included inside namespace gfnff by engine.cu (one translation unit).
#pragma once

namespace {

constexpr int kPcgThreads = 512;       // k_pcg: the whole SM (the tiled product wants the warps)
constexpr int kPcgPipeThreads = 256;   // k_pcg_pipe: half of an SM's registers, so that the
                                       // charge-independent term kernels run beside it
constexpr int kPcgMaxBlock = 64;   // largest preconditioner block

struct PCGArgs {
    const double* M;
    int lda, n;
    const double* b;
    double* x;            // solution
    double* z;            // preconditioned residual (shared between grid blocks)
    double* z2;           // k_pcg_pipe: second shared n-vector (published vectors alternate)
    const int2* blocks;   // preconditioner blocks {first row, size}
    const long long* boff;
    int maxrows;          // most rows owned by one grid block
    int maxinv;           // most inverse entries held by one grid block
    const int4* part;     // per grid block: rows [x, y), preconditioner blocks [z, w)
    const int* rblk;      // preconditioner block of every row
    double* partial;      // gridDim.x * 8
    unsigned int* bar;    // arrival count at [0], generation at [kBarGen]
    int* info;
    int* iters;           // [0] iterations; k_pcg_ir also [1]: FP64 matrix products
    int* warm;            // when non-null and *warm != 0, x holds the previous solution of the
                          // same system and is the initial guess; set to 1 on convergence
    const float* Mf;      // lower form in the mixed precision form: M stored in FP32 (M unused)
    const double* binv_pre;   // block inverses computed at set-up (global memory, boff layout), or null
    int lower;            // 1 or 2: only the lower triangle of M is stored; M p by tiles
                          // (matvec_tiles, streaming 4 or 8 columns per warp at once)
    double* yA;           // lower: n-vector the tiles add M p into (zero between uses)
    const int2* tiles;    // lower: tiles {first row I0, first column J0}, I0 >= J0
    int ntiles;
    int max_iter;
    double tol;           // converged when max|b - M x| <= tol * max|b| ...
    double tol_abs;       // ... or, when > 0, when max|b - M x| <= tol_abs (the mixed form's
                          // FP64 true-residual bar); the residual is always computed in FP64
    int max_outer;        // k_pcg_ir: FP64 residual corrections at most
    double inner_rel;     // k_pcg_ir: inner solve to ||r_inner||_inf <= inner_rel ||r||_inf
    float* p32[2];        // k_pcg_ir: the inner CG direction in FP32, two global n-vectors
                          // (16-byte aligned, length a multiple of 4) used in turn
};

// grid-wide barrier (all blocks co-resident); false when the wait gave up.  The block's
// threads meet at __syncthreads, then thread 0 alone arrives with a release atomic
// (covering the block's writes ordered before it by the block barrier) and polls with
// acquire loads.  The arrival
// counter bar[0] and the generation bar[kBarGen] sit on different 128-byte lines, so the
// polling reads do not queue behind the arrival atomics; the generation counter makes
// the barrier reusable without a reset in between.
__device__ __forceinline__ double pcg_threshold(const PCGArgs& A, double bmax)
{
    return A.tol_abs > 0.0 ? A.tol_abs : A.tol * bmax;
}

constexpr int kBarGen = 32;
__device__ __forceinline__ unsigned int atom_add_release(unsigned int* p, unsigned int v)
{
    unsigned int old;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ bool grid_sync(unsigned int* bar, unsigned int& gen)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok_s = 1;
        const unsigned int want = gen + 1;
        if (atom_add_release(bar, 1u) + 1u == gridDim.x) {
            atomicExch(bar, 0u);
            atom_add_release(bar + kBarGen, 1u);
        } else {
            long long polls = 0;
            while ((int)(ld_acquire(bar + kBarGen) - want) < 0) {
                if (++polls > (1ll << 24)) {
                    ok_s = 0;
                    break;
                }
            }
        }
        gen = want;
    }
    __syncthreads();
    return ok_s != 0;
}

// block reduction of (sum, max) into the block's two partial slots at out
__device__ void block_sum_max(double s, double m, double* out)
{
    __shared__ double rs[32], rm[32];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) { rs[w] = s; rm[w] = m; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += rs[k]; b = fmax(b, rm[k]); }
        __stcg(out, a);
        __stcg(out + 1, b);
    }
}

// the same totals in every block: thread k loads block k's partials (one round trip for
// all of them), then a fixed reduction tree combines them, so every block gets
// identical sums
__device__ void grid_totals(const double* partial, int slot, double& sum, double& mx)
{
    __shared__ double ws[32], wm[32];
    __syncthreads();
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
        a += __ldcg(partial + 8 * k + slot);
        b = fmax(b, __ldcg(partial + 8 * k + slot + 1));
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { ws[w] = a; wm[w] = b; }
    __syncthreads();
    a = 0.0;
    b = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += ws[k]; b = fmax(b, wm[k]); }
    sum = a;
    mx = b;
}

// p = z + beta p over all n entries (z from global memory, several loads in flight);
// beta == 0 overwrites p without reading it
__device__ void update_p(double* p, const double* z, int n, double beta)
{
    constexpr int U = 8;
    for (int c0 = threadIdx.x; c0 < n; c0 += U * blockDim.x) {
        double zv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * blockDim.x;
            zv[u] = c < n ? __ldcg(z + c) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * blockDim.x;
            if (c < n) p[c] = beta == 0.0 ? zv[u] : zv[u] + beta * p[c];
        }
    }
}

// z = P^-1 r on the owned rows (one thread per row, rblk[r] = its preconditioner block),
// everything in shared memory: r, z and the block inverses of this grid block; returns
// the thread's part of r.z
// meta[k] = {first local row of row k's block, block size, offset of row k's inverse row}
__device__ double apply_precond(int nrow, const int4* meta, const double* binv, const double* r, double* z)
{
    double rz = 0.0;
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        const int4 m = meta[k];
        const double* Bi = binv + m.z;
        const double* rb = r + m.x;
        double s = 0.0;
        for (int j = 0; j < m.y; ++j) s += Bi[j] * rb[j];
        z[k] = s;
        rz += s * r[k];
    }
    return rz;
}

// out[r - row0] = (M v)_r for the owned rows (warp per row).  Rows are read as 16-byte
// pairs (lda is even) with eight independent pairs in flight per lane, so that one
// row of L2-resident M costs a few L2 round trips rather than one per 32 elements.
// Returns the thread's part of sum_r v_r (M v)_r.
template <int U>   // double2 loads in flight per lane
__device__ double matvec_rows_u(const PCGArgs& A, const double* v, int row0, int row1, double* out)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int n2 = A.n >> 1;
    const double2* v2 = reinterpret_cast<const double2*>(v);
    double vmv = 0.0;
    for (int rr = row0 + warp; rr < row1; rr += nw) {
        const double* col = A.M + (size_t)rr * A.lda;
        const double2* c2 = reinterpret_cast<const double2*>(col);
        double s[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) s[u] = 0.0;
        int c = lane;
        for (; c + (U - 1) * 32 < n2; c += U * 32) {
            double2 m[U];
#pragma unroll
            for (int u = 0; u < U; ++u) m[u] = c2[c + 32 * u];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 w = v2[c + 32 * u];
                s[u & 7] += m[u].x * w.x + m[u].y * w.y;
            }
        }
        for (; c < n2; c += 32) {
            const double2 m = c2[c], w = v2[c];
            s[0] += m.x * w.x + m.y * w.y;
        }
        if ((A.n & 1) && lane == 0) s[0] += col[A.n - 1] * v[A.n - 1];
        double t = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) {
            out[rr - row0] = t;
            vmv += t * v[rr];
        }
    }
    return vmv;
}

// eight loads in flight per lane measured faster than sixteen (1000 waters: 0.188 vs 0.194 ms
// per solve)
__device__ double matvec_rows(const PCGArgs& A, const double* v, int row0, int row1, double* out)
{
    return matvec_rows_u<8>(A, v, row0, row1, out);
}

// element (r, c) of M, from the lower triangle when only that is stored
__device__ __forceinline__ double mget(const PCGArgs& A, int r, int c)
{
    const size_t e = (A.lower && r < c) ? (size_t)r * A.lda + c : (size_t)c * A.lda + r;
    return A.Mf ? (double)A.Mf[e] : A.M[e];
}

// Symmetric M p from the lower triangle, for matrices too large for L2: the tiles
// (kPcgT x kPcgT, I0 >= J0) are dealt round-robin to the grid blocks.  A warp takes
// columns c of the tile kPcgCols at a time (independent 8-byte loads per lane in flight,
// streamed past L2) and forms u_r += M(r, c) p_c for the tile's rows (registers) and
// v_c = sum_r M(r, c) p_r (warp sum); the transposed part v goes to y_J, the row part u
// (summed over the block's warps in shared memory) to y_I, both as FP64 atomics into
// A.yA.  Diagonal tiles use r >= c for u and r > c for v.  Returns the thread's part of
// p^T M p.  The caller reads y after a grid barrier and zeroes what it read.
constexpr int kPcgT = 128;
template <int kPcgCols, class TM>   // columns a warp streams at once; matrix storage type
__device__ double matvec_tiles_c(const PCGArgs& A, const TM* Mt, const double* p, double* red)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double pap = 0.0;
    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int2 tl = A.tiles[t];
        const int I0 = tl.x, J0 = tl.y;
        const bool diag = I0 == J0;
        const int ni = min(kPcgT, A.n - I0), nj = min(kPcgT, A.n - J0);
        double u[4], pr[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = lane + 32 * i;
            u[i] = 0.0;
            pr[i] = r < ni ? p[I0 + r] : 0.0;
        }
        for (int cb = warp * kPcgCols; cb < nj; cb += nw * kPcgCols) {
            TM m[kPcgCols][4];   // kept in the storage type (FP32: half the registers)
            double v[kPcgCols], pc[kPcgCols];
#pragma unroll
            for (int q = 0; q < kPcgCols; ++q) {
                const int c = cb + q;
                pc[q] = c < nj ? p[J0 + c] : 0.0;
                const TM* col = Mt + (size_t)(J0 + (c < nj ? c : 0)) * A.lda + I0;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = lane + 32 * i;
                    m[q][i] = (c < nj && r < ni && (!diag || r >= c)) ? __ldcs(col + r) : TM(0);
                }
            }
#pragma unroll
            for (int q = 0; q < kPcgCols; ++q) {
                const int c = cb + q;
                v[q] = 0.0;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = lane + 32 * i;
                    const double mv = (double)m[q][i];
                    u[i] += mv * pc[q];
                    if (!diag || r > c) v[q] += mv * pr[i];
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int q = 0; q < kPcgCols; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
            double vq = 0.0;
#pragma unroll
            for (int q = 0; q < kPcgCols; ++q)
                if (lane == q) vq = v[q];
            if (lane < kPcgCols) {
                const int c = cb + lane;
                if (c < nj && vq != 0.0) {
                    atomicAdd(A.yA + J0 + c, vq);
                    pap += p[J0 + c] * vq;
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) red[warp * kPcgT + lane + 32 * i] = u[i];
        __syncthreads();
        for (int r = threadIdx.x; r < ni; r += blockDim.x) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += red[w * kPcgT + r];
            atomicAdd(A.yA + I0 + r, s);
            pap += p[I0 + r] * s;
        }
        __syncthreads();
    }
    return pap;
}

__device__ double matvec_tiles(const PCGArgs& A, const double* p, double* red)
{
    if (A.Mf) return matvec_tiles_c<8>(A, A.Mf, p, red);   // 4-byte elements: twice the columns in flight
    return A.lower == 2 ? matvec_tiles_c<8>(A, A.M, p, red) : matvec_tiles_c<4>(A, A.M, p, red);
}

// Ap for the owned rows after matvec_tiles and a grid barrier: read y (L2) and zero it
__device__ void take_tiles_result(const PCGArgs& A, int row0, int nrow, double* Ap)
{
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        Ap[k] = __ldcg(A.yA + row0 + k);
        __stcg(A.yA + row0 + k, 0.0);
    }
    __syncthreads();
}

// element accessor of the stored matrix (full, lower, or FP32 lower)
struct MStored {
    const PCGArgs* A;
    __device__ __forceinline__ double operator()(int r, int c) const { return mget(*A, r, c); }
};

// inverse of a preconditioner block of at most kPcgSmall rows by one thread
// (Gauss-Jordan in registers-sized local storage)
constexpr int kPcgSmall = 4;
template <class Get>
__device__ void invert_small(const PCGArgs& A, int bk, double* I, Get get)
{
    const int2 bl = A.blocks[bk];
    const int s = bl.y;
    double g[kPcgSmall][kPcgSmall], inv[kPcgSmall][kPcgSmall];
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) {
            g[i][j] = get(bl.x + i, bl.x + j);
            inv[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int c = 0; c < s; ++c) {
        const double pv = 1.0 / g[c][c];
        for (int j = 0; j < s; ++j) { g[c][j] *= pv; inv[c][j] *= pv; }
        for (int i = 0; i < s; ++i) {
            if (i == c) continue;
            const double f = g[i][c];
            for (int j = 0; j < s; ++j) { g[i][j] -= f * g[c][j]; inv[i][j] -= f * inv[c][j]; }
        }
    }
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) I[i * s + j] = inv[i][j];
}

// in-place Gauss-Jordan inverse of a preconditioner block of kPcgSmall < s <= 32 rows by
// one warp: lane j owns column j, column c of the pivot step is staged in colc (32
// doubles per warp), __syncwarp only.  M is stored in full and symmetric, so row i of
// the block is read from column i of M (coalesced).
constexpr int kPcgWarpMax = 32;
template <class Get>
__device__ void invert_warp(const PCGArgs& A, int bk, double* I, double* colc, Get get)
{
    const int lane = threadIdx.x & 31;
    const int2 bl = A.blocks[bk];
    const int s = bl.y;
    if (lane < s)
        for (int i = 0; i < s; ++i) I[i * s + lane] = get(bl.x + lane, bl.x + i);
    __syncwarp();
    for (int c = 0; c < s; ++c) {
        colc[lane] = lane < s ? I[lane * s + c] : 0.0;
        __syncwarp();
        const double inv = 1.0 / colc[c];
        if (lane < s) {
            const int j = lane;
            const double rc = (j == c ? 1.0 : I[c * s + j]) * inv;
            I[c * s + j] = rc;
            for (int i = 0; i < s; ++i) {
                if (i == c) continue;
                I[i * s + j] = (j == c ? 0.0 : I[i * s + j]) - colc[i] * rc;
            }
        }
        __syncwarp();
    }
}

// inverses of the grid block's preconditioner blocks (Gauss-Jordan, SPD, no pivoting:
// up to kPcgSmall rows by one thread, up to kPcgWarpMax by one warp, larger ones by the
// whole block with G as scratch) and the per-row records of apply_precond
template <class Get>
__device__ void pcg_setup(const PCGArgs& A, int4 pt, long long boff0, double* G, double* Bs, int4* meta, Get get)
{
    __shared__ double piv;
    constexpr int GL = kPcgMaxBlock + 1;
    const int row0 = pt.x, nrow = pt.y - pt.x;
    if (A.binv_pre) {   // inverses from set-up: only the row records
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            const int rr = row0 + k, bk = A.rblk[rr];
            const int2 bl = A.blocks[bk];
            meta[k] = make_int4(bl.x - row0, bl.y, (int)(A.boff[bk] - boff0) + (rr - bl.x) * bl.y, 0);
        }
        __syncthreads();
        return;
    }
    // ---- inverse of every owned preconditioner block (Gauss-Jordan on [M_bb | I]; SPD,
    // no pivoting); small blocks one per thread, larger ones by the whole grid block
    for (int bk = pt.z + threadIdx.x; bk < pt.w; bk += blockDim.x)
        if (A.blocks[bk].y <= kPcgSmall) invert_small(A, bk, Bs + (A.boff[bk] - boff0), get);
    {
        __shared__ double colc[kPcgThreads / 32][32];
        const int warp = threadIdx.x >> 5;
        for (int bk = pt.z + warp; bk < pt.w; bk += (int)(blockDim.x >> 5)) {
            const int s = A.blocks[bk].y;
            if (s > kPcgSmall && s <= kPcgWarpMax) invert_warp(A, bk, Bs + (A.boff[bk] - boff0), colc[warp], get);
        }
    }
    for (int bk = pt.z; bk < pt.w; ++bk) {
        const int2 bl = A.blocks[bk];
        const int s = bl.y;
        if (s <= kPcgWarpMax) continue;
        double* I = Bs + (A.boff[bk] - boff0);
        __syncthreads();
        for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
            const int i = e / s, j = e % s;
            G[i * GL + j] = get(bl.x + i, bl.x + j);
            I[e] = i == j ? 1.0 : 0.0;
        }
        __syncthreads();
        for (int c = 0; c < s; ++c) {
            if (threadIdx.x == 0) piv = 1.0 / G[c * GL + c];
            __syncthreads();
            const double pv = piv;
            for (int j = threadIdx.x; j < s; j += blockDim.x) {
                G[c * GL + j] *= pv;
                I[c * s + j] *= pv;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
                const int i = e / s, j = e % s;
                if (i != c) I[i * s + j] -= G[i * GL + c] * I[c * s + j];
            }
            __syncthreads();
            for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
                const int i = e / s, j = e % s;
                if (i != c && j != c) G[i * GL + j] -= G[i * GL + c] * G[c * GL + j];
            }
            __syncthreads();
            for (int i = threadIdx.x; i < s; i += blockDim.x)
                if (i != c) G[i * GL + c] = 0.0;
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        const int rr = row0 + k, bk = A.rblk[rr];
        const int2 bl = A.blocks[bk];
        meta[k] = make_int4(bl.x - row0, bl.y, (int)(A.boff[bk] - boff0) + (rr - bl.x) * bl.y, 0);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg(PCGArgs A)
{
    extern __shared__ double sm[];
    constexpr int GL = kPcgMaxBlock + 1;
    const int4 pt = A.part[blockIdx.x];
    const int row0 = pt.x, row1 = pt.y, nrow = row1 - row0;
    const long long boff0 = pt.z < pt.w ? A.boff[pt.z] : 0;
    double* p = sm;                              // n: search direction, replicated
    double* G = p + ((A.n + 1) & ~1);            // kPcgMaxBlock x GL scratch (even offsets
                                                 // keep the int4 records 16-byte aligned)
    double* xs = G + kPcgMaxBlock * GL;          // owned rows: x, r, z, M p
    double* rs = xs + A.maxrows;
    double* zs = rs + A.maxrows;
    double* Ap = zs + A.maxrows;
    double* Bs = Ap + A.maxrows;                 // inverses of the owned blocks
    int4* meta = reinterpret_cast<int4*>(Bs + A.maxinv);   // per owned row, see apply_precond
    __shared__ unsigned int gen;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + kBarGen);
    pcg_setup(A, pt, boff0, G, Bs, meta, MStored{&A});
    const double* Bp = A.binv_pre ? A.binv_pre + boff0 : Bs;
    // ---- x = x0 (the previous solution, or 0), r = b - M x0, z = P^-1 r.  x0 is complete
    // in global memory since the previous launch, so no grid barrier is needed here.
    const bool warm = A.warm != nullptr && *A.warm != 0;
    bool ok = true;
    if (warm) {   // uniform over the grid: every block reads the same flag
        update_p(p, A.x, A.n, 0.0);
        __syncthreads();
        if (A.lower) {
            matvec_tiles(A, p, G);
            ok = grid_sync(A.bar, gen);
            take_tiles_result(A, row0, nrow, Ap);
        } else {
            matvec_rows(A, p, row0, row1, Ap);
        }
        __syncthreads();
    }
    double bmax_t = 0.0;
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        const double bv = A.b[row0 + k];
        xs[k] = warm ? p[row0 + k] : 0.0;
        rs[k] = warm ? bv - Ap[k] : bv;
        bmax_t = fmax(bmax_t, fabs(bv));
    }
    __syncthreads();
    double rz_t = apply_precond(nrow, meta, Bp, rs, zs);
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.z + row0 + k, zs[k]);
    // the start totals have a slot of their own: a fast block writes its first p.Mp
    // partial into slot 0 before a slow one has read these after the barrier
    block_sum_max(rz_t, bmax_t, A.partial + 8 * blockIdx.x + 4);
    ok = grid_sync(A.bar, gen) && ok;
    double rz = 0.0, bmax = 0.0;
    if (ok) grid_totals(A.partial, 4, rz, bmax);
    update_p(p, A.z, A.n, 0.0);
    int it = 0;
    bool conv = ok && bmax == 0.0;
    while (ok && !conv && it < A.max_iter) {
        ++it;
        __syncthreads();
        const double pap_t = A.lower ? matvec_tiles(A, p, G) : matvec_rows(A, p, row0, row1, Ap);
        block_sum_max(pap_t, 0.0, A.partial + 8 * blockIdx.x);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        if (A.lower) take_tiles_result(A, row0, nrow, Ap);
        double pap, unused;
        grid_totals(A.partial, 0, pap, unused);
        const double alpha = rz / pap;
        double rmax_t = 0.0;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            xs[k] += alpha * p[row0 + k];
            rs[k] -= alpha * Ap[k];
            rmax_t = fmax(rmax_t, fabs(rs[k]));
        }
        __syncthreads();
        rz_t = apply_precond(nrow, meta, Bp, rs, zs);
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.z + row0 + k, zs[k]);
        block_sum_max(rz_t, rmax_t, A.partial + 8 * blockIdx.x + 2);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        double rzn, rmax;
        grid_totals(A.partial, 2, rzn, rmax);
        if (rmax <= pcg_threshold(A, bmax)) {
            // accept only on the true residual r = b - M x; otherwise restart from it
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.x + row0 + k, xs[k]);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            update_p(p, A.x, A.n, 0.0);
            __syncthreads();
            if (A.lower) {
                matvec_tiles(A, p, G);
                ok = grid_sync(A.bar, gen);
                if (!ok) break;
                take_tiles_result(A, row0, nrow, Ap);
            } else {
                matvec_rows(A, p, row0, row1, Ap);
            }
            __syncthreads();
            rmax_t = 0.0;
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
                rs[k] = A.b[row0 + k] - Ap[k];
                rmax_t = fmax(rmax_t, fabs(rs[k]));
            }
            __syncthreads();
            rz_t = apply_precond(nrow, meta, Bp, rs, zs);
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.z + row0 + k, zs[k]);
            block_sum_max(rz_t, rmax_t, A.partial + 8 * blockIdx.x + 2);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            grid_totals(A.partial, 2, rzn, rmax);
            if (rmax <= pcg_threshold(A, bmax)) {
                conv = true;
                break;
            }
            rz = rzn;
            update_p(p, A.z, A.n, 0.0);
            continue;
        }
        const double beta = rzn / rz;
        rz = rzn;
        update_p(p, A.z, A.n, beta);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) A.x[row0 + k] = xs[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.info = !ok ? 2 : (conv ? 0 : 3);
        *A.iters = it;
        if (A.warm) *A.warm = (ok && conv) ? 1 : 0;
    }
}

// ------------------------------------------------------------------------------------
// Mixed form, large systems (the lower-triangle tiled form): block-Jacobi CG on the FP32 copy
// of M inside FP64 iterative refinement.  Outer step: the true residual r = b - M x with the
// FP64 lower triangle (A.M); stop when ||r||_inf <= tol_abs (info 0) or after max_outer
// corrections (info 3, REFINE_NOT_CONVERGED).  Otherwise CG on the FP32 lower triangle
// (A.Mf: half the bytes of every product, FP32 arithmetic inside a tile) solves M32 d = r
// from d = 0, and x += d.  The inner solve stops at inner_rel ||r||_inf, but not below half
// the bar: one correction cannot lower the true residual by more than the FP32 rounding of M
// allows (~1e-6 relative), so the next outer step finishes from there.  Preconditioner blocks
// as in k_pcg; the partial-sum slots follow k_pcg's rule (the outer totals have a slot of
// their own).  iters: the inner iterations of all outer steps.
// ------------------------------------------------------------------------------------
__device__ double matvec_tiles64(const PCGArgs& A, const double* p, double* red)
{
    return A.lower == 2 ? matvec_tiles_c<8>(A, A.M, p, red) : matvec_tiles_c<4>(A, A.M, p, red);
}

// The inner products of k_pcg_ir: the FP32 lower triangle with FP32 arithmetic inside a tile
// (elements, the direction and the partial sums stay FP32: the inner solve needs ~1e-6
// relative accuracy, a 128-term FP32 sum gives ~1e-7), the tile's row and column sums added
// to y as FP64 atomics, as in matvec_tiles_c.  The tiles stream through shared memory in
// halves of 64 columns (32 KB) by TMA (one cp.async.bulk.tensor.2d per half, issued by one
// thread; rows and columns past n are zero-filled), together with the direction's segments
// (cp.async.bulk, the direction is an FP32 n-vector in global memory), kPcgStages halves in
// flight, each stage completing on its own mbarrier: the copies run ahead of the products,
// the reductions and the atomics, and the threads issue no copy instructions.  Every wait on
// an mbarrier is bounded (kTmaPolls); a wait that gives up marks the product failed.  The
// staging ring shares its region with the FP64 vector of the outer products (pcg_ir_pregion).
constexpr int kPcgHalf = 64 * kPcgT;   // floats of half a tile
constexpr int kPcgStages = 4;          // halves in flight
constexpr int kPcgStageF = kPcgHalf + kPcgT + 64;   // floats per stage: elements, pr, pc
constexpr long long kTmaPolls = 1ll << 24;

__host__ __device__ inline int pcg_ir_pregion(int n)
{
    const int pd = (n + 1) & ~1;
    const int ring = kPcgStages * kPcgStageF / 2 + 16;   // doubles, with room to align to 128 bytes
    return pd > ring ? pd : ring;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// true once the phase with the given parity has completed; false after kTmaPolls polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    for (long long k = 0; k < kTmaPolls; ++k) {
        unsigned done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(smem_u32(bar)), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// TMA of half h's elements (box 128 rows x 64 columns at rows I0, columns J0 + 64 half) and
// bulk copies of the direction's row segment p[I0, +128) and column segment p[J0 + 64 half,
// +64) (clipped to the buffers' rounded length n4) into stage st, completing on bar
__device__ __forceinline__ void pcg_tma_half(const PCGArgs& A, const CUtensorMap* tmap, const float* p32, int t,
                                             int half, float* st, unsigned long long* bar)
{
    const int2 tl = A.tiles[t];
    const int I0 = tl.x, J0 = tl.y + 64 * half;
    const int n4 = (A.n + 3) & ~3;
    const unsigned pr_bytes = 4u * (unsigned)min(kPcgT, n4 - I0);
    const unsigned pc_bytes = J0 < n4 ? 4u * (unsigned)min(64, n4 - J0) : 0u;
    mbar_expect_tx(bar, 4u * kPcgHalf + pr_bytes + pc_bytes);
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(smem_u32(st)), "l"(tmap), "r"(I0), "r"(J0), "r"(smem_u32(bar))
        : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(st + kPcgHalf)), "l"(p32 + I0), "r"(pr_bytes), "r"(smem_u32(bar))
                 : "memory");
    if (pc_bytes)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                     ::"r"(smem_u32(st + kPcgHalf + kPcgT)), "l"(p32 + J0), "r"(pc_bytes), "r"(smem_u32(bar))
                     : "memory");
}

// bars: kPcgStages mbarriers (arrival count 1); uses: halves streamed so far by this block
// (stage = uses % kPcgStages, phase parity = (uses / kPcgStages) & 1), carried across calls;
// ok cleared when a wait gives up
__device__ double matvec_tiles_f32(const PCGArgs& A, const CUtensorMap* tmap, const float* p32, float* ring,
                                   float* red, unsigned long long* bars, unsigned& uses, bool& ok)
{
    constexpr int kCols = 4;   // 16 warps x 4 columns = one half tile
    static_assert(kPcgThreads / 32 * kCols == 64, "one pass per half tile");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double pap = 0.0;
    const int mine = blockIdx.x < A.ntiles ? (A.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int nh = 2 * mine;
    __shared__ int fail_s;
    // the ring's memory was last accessed by ordinary loads and stores (the FP64 vector, or
    // the previous product): ordered before the TMA writes
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        fail_s = 0;
        for (int h = 0; h < kPcgStages - 1 && h < nh; ++h) {
            const unsigned s = (uses + h) % kPcgStages;
            pcg_tma_half(A, tmap, p32, blockIdx.x + (h >> 1) * gridDim.x, h & 1, ring + s * kPcgStageF, bars + s);
        }
    }
    __syncthreads();
    float u[4], pr[4];
    for (int h = 0; h < nh; ++h) {
        const unsigned g = uses + h, s = g % kPcgStages;
        if (threadIdx.x == 0 && h + kPcgStages - 1 < nh) {
            const int hn = h + kPcgStages - 1;
            const unsigned sn = (uses + hn) % kPcgStages;
            pcg_tma_half(A, tmap, p32, blockIdx.x + (hn >> 1) * gridDim.x, hn & 1, ring + sn * kPcgStageF, bars + sn);
        }
        if (!mbar_wait(bars + s, (g / kPcgStages) & 1)) fail_s = 1;
        const float* st = ring + s * kPcgStageF;
        const int t = blockIdx.x + (h >> 1) * gridDim.x, half = h & 1;
        const int2 tl = A.tiles[t];
        const int I0 = tl.x, J0 = tl.y;
        const bool diag = I0 == J0;
        const int ni = min(kPcgT, A.n - I0), nj = min(kPcgT, A.n - J0);
        const bool full = !diag && ni == kPcgT && nj == kPcgT;
        if (half == 0) {
            const float4 p4 = *reinterpret_cast<const float4*>(st + kPcgHalf + 4 * lane);
            pr[0] = p4.x; pr[1] = p4.y; pr[2] = p4.z; pr[3] = p4.w;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                u[j] = 0.f;
                if (4 * lane + j >= ni) pr[j] = 0.f;
            }
        }
        float v[kCols];
        if (full) {
#pragma unroll
            for (int q = 0; q < kCols; ++q) {
                const int cl = warp * kCols + q;
                const float pc = st[kPcgHalf + kPcgT + cl];
                const float4 m4 = *reinterpret_cast<const float4*>(st + cl * kPcgT + 4 * lane);
                u[0] = fmaf(m4.x, pc, u[0]);
                u[1] = fmaf(m4.y, pc, u[1]);
                u[2] = fmaf(m4.z, pc, u[2]);
                u[3] = fmaf(m4.w, pc, u[3]);
                v[q] = m4.x * pr[0];
                v[q] = fmaf(m4.y, pr[1], v[q]);
                v[q] = fmaf(m4.z, pr[2], v[q]);
                v[q] = fmaf(m4.w, pr[3], v[q]);
            }
        } else {
#pragma unroll
            for (int q = 0; q < kCols; ++q) {
                const int cl = warp * kCols + q, c = 64 * half + cl;
                const float pc = c < nj ? st[kPcgHalf + kPcgT + cl] : 0.f;
                const float4 m4 = *reinterpret_cast<const float4*>(st + cl * kPcgT + 4 * lane);
                const float mm[4] = {m4.x, m4.y, m4.z, m4.w};
                v[q] = 0.f;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int r = 4 * lane + j;
                    const float m = (c < nj && r < ni && (!diag || r >= c)) ? mm[j] : 0.f;
                    u[j] = fmaf(m, pc, u[j]);
                    if (!diag || r > c) v[q] = fmaf(m, pr[j], v[q]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < kCols; ++q) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        float vq = 0.f;
#pragma unroll
        for (int q = 0; q < kCols; ++q)
            if (lane == q) vq = v[q];
        if (lane < kCols) {
            const int cl = warp * kCols + lane, c = 64 * half + cl;
            if (c < nj && vq != 0.f) {
                atomicAdd(A.yA + J0 + c, (double)vq);
                pap += (double)st[kPcgHalf + kPcgT + cl] * (double)vq;
            }
        }
        if (half == 1) {
#pragma unroll
            for (int j = 0; j < 4; ++j) red[warp * kPcgT + 4 * lane + j] = u[j];
            __syncthreads();
            for (int r = threadIdx.x; r < ni; r += blockDim.x) {
                double sr = 0.0;
                for (int w = 0; w < nw; ++w) sr += (double)red[w * kPcgT + r];
                atomicAdd(A.yA + I0 + r, sr);
                pap += (double)st[kPcgHalf + r] * sr;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();   // stage s is free for the copy issued next
    }
    uses += (unsigned)nh;
    if (fail_s) ok = false;
    return pap;
}

// dst = z + beta src over all n entries (z from global memory), written by every grid block
// (the same values): the direction of this inner iteration, read by the products of all
// blocks; src is the previous direction (the other buffer), beta == 0 ignores it
__device__ void update_p32(float* dst, const float* src, const double* z, int n, double beta)
{
    constexpr int U = 8;
    for (int c0 = threadIdx.x; c0 < n; c0 += U * blockDim.x) {
        double zv[U];
        float pv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * blockDim.x;
            zv[u] = c < n ? __ldcg(z + c) : 0.0;
            pv[u] = (c < n && beta != 0.0) ? __ldcg(src + c) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + u * blockDim.x;
            if (c < n) __stcg(dst + c, (float)(zv[u] + beta * (double)pv[u]));
        }
    }
    // the direction is read next by bulk copies (the async proxy)
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    __syncthreads();
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg_ir(PCGArgs A, const __grid_constant__ CUtensorMap tmap)
{
    extern __shared__ __align__(128) double sm[];
    __shared__ __align__(8) unsigned long long bars[kPcgStages];
    if (threadIdx.x == 0) {
        for (int s = 0; s < kPcgStages; ++s) mbar_init(bars + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    unsigned uses = 0;   // halves streamed through the ring (the stages' phases)
    bool tma_ok = true;
    constexpr int GL = kPcgMaxBlock + 1;
    const int4 pt = A.part[blockIdx.x];
    const int row0 = pt.x, row1 = pt.y, nrow = row1 - row0;
    const long long boff0 = pt.z < pt.w ? A.boff[pt.z] : 0;
    double* p = sm;                              // n, replicated: x of the FP64 residual
    float* ring = reinterpret_cast<float*>(      // inner iterations: the tile staging ring
        (reinterpret_cast<size_t>(sm) + 127) & ~static_cast<size_t>(127));
    double* G = p + pcg_ir_pregion(A.n);         // kPcgMaxBlock x GL scratch
    double* xs = G + kPcgMaxBlock * GL;          // owned rows: x, r, z, M p, d
    double* rs = xs + A.maxrows;
    double* zs = rs + A.maxrows;
    double* Ap = zs + A.maxrows;
    double* ds = Ap + A.maxrows;
    double* Bs = ds + ((A.maxrows + 1) & ~1);    // inverses of the owned blocks (an even offset
                                                 // keeps the int4 row records 16-byte aligned)
    int4* meta = reinterpret_cast<int4*>(Bs + A.maxinv);
    __shared__ unsigned int gen;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + kBarGen);
    pcg_setup(A, pt, boff0, G, Bs, meta, MStored{&A});
    const double* Bp = A.binv_pre ? A.binv_pre + boff0 : Bs;
    const bool warm = A.warm != nullptr && *A.warm != 0;   // uniform over the grid
    bool ok = true, conv = false;
    int it = 0, prod64 = 0;
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) xs[k] = warm ? __ldcg(A.x + row0 + k) : 0.0;
    for (int outer = 0; ok; ++outer) {
        // ---- FP64 true residual r = b - M x (x = 0 on a cold start: r = b); x is complete in
        // global memory (the previous launch, or the barrier after the last correction)
        const bool have_x = warm || outer > 0;
        if (have_x) {
            ++prod64;
            update_p(p, A.x, A.n, 0.0);
            __syncthreads();
            matvec_tiles64(A, p, G);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            take_tiles_result(A, row0, nrow, Ap);
        }
        double rmax_t = 0.0;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            const double r = A.b[row0 + k] - (have_x ? Ap[k] : 0.0);
            rs[k] = r;
            ds[k] = 0.0;
            rmax_t = fmax(rmax_t, fabs(r));
        }
        __syncthreads();
        double rz_t = apply_precond(nrow, meta, Bp, rs, zs);
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.z + row0 + k, zs[k]);
        block_sum_max(rz_t, rmax_t, A.partial + 8 * blockIdx.x + 4);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        double rz = 0.0, rmax = 0.0;
        grid_totals(A.partial, 4, rz, rmax);
        if (rmax <= A.tol_abs) {
            conv = true;
            break;
        }
        if (outer >= A.max_outer || it >= A.max_iter) break;
        const double stop = fmax(A.inner_rel * rmax, 0.5 * A.tol_abs);
        __syncthreads();   // the FP64 vector's region becomes the staging ring
        int cur = 0;       // the direction's buffer: A.p32[cur]
        update_p32(A.p32[cur], A.p32[1 - cur], A.z, A.n, 0.0);
        // ---- inner CG on the FP32 matrix: M32 d = r from d = 0
        while (it < A.max_iter) {
            ++it;
            __syncthreads();
            const double pap_t =
                matvec_tiles_f32(A, &tmap, A.p32[cur], ring, reinterpret_cast<float*>(G), bars, uses, tma_ok);
            block_sum_max(pap_t, 0.0, A.partial + 8 * blockIdx.x);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            take_tiles_result(A, row0, nrow, Ap);
            double pap, unused;
            grid_totals(A.partial, 0, pap, unused);
            const double alpha = rz / pap;
            double rin_t = 0.0;
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
                ds[k] += alpha * (double)__ldcg(A.p32[cur] + row0 + k);
                rs[k] -= alpha * Ap[k];
                rin_t = fmax(rin_t, fabs(rs[k]));
            }
            __syncthreads();
            rz_t = apply_precond(nrow, meta, Bp, rs, zs);
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(A.z + row0 + k, zs[k]);
            block_sum_max(rz_t, rin_t, A.partial + 8 * blockIdx.x + 2);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            double rzn, rin;
            grid_totals(A.partial, 2, rzn, rin);
            if (rin <= stop) break;
            const double beta = rzn / rz;
            rz = rzn;
            cur = 1 - cur;
            update_p32(A.p32[cur], A.p32[1 - cur], A.z, A.n, beta);
        }
        if (!ok) break;
        // ---- x += d, published for the next residual
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            xs[k] += ds[k];
            __stcg(A.x + row0 + k, xs[k]);
        }
        ok = grid_sync(A.bar, gen);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) A.x[row0 + k] = xs[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.info = (!ok || !tma_ok) ? 2 : (conv ? 0 : 3);
        A.iters[0] = it;
        A.iters[1] = prod64;
        if (A.warm) *A.warm = (ok && conv) ? 1 : 0;
    }
}

}  // namespace

namespace {

// block partials (sum a, sum b, max c) into out[0..2]
__device__ void block_sum3(double a, double b, double c, double* out)
{
    __shared__ double ra[32], rb[32], rc[32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c = fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) { ra[w] = a; rb[w] = b; rc[w] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0, z = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { x += ra[k]; y += rb[k]; z = fmax(z, rc[k]); }
        __stcg(out, x);
        __stcg(out + 1, y);
        __stcg(out + 2, z);
    }
}

// grid totals of block_sum3's partials (slot offset `set` in each block's 8 doubles),
// identical in every block (fixed reduction order)
__device__ void grid_totals3(const double* partial, int set, double& a, double& b, double& c)
{
    __shared__ double wa[32], wb[32], wc[32];
    __syncthreads();
    double x = 0.0, y = 0.0, z = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
        x += __ldcg(partial + 8 * k + set);
        y += __ldcg(partial + 8 * k + set + 1);
        z = fmax(z, __ldcg(partial + 8 * k + set + 2));
    }
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z = fmax(z, __shfl_xor_sync(0xffffffffu, z, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { wa[w] = x; wb[w] = y; wc[w] = z; }
    __syncthreads();
    x = y = z = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { x += wa[k]; y += wb[k]; z = fmax(z, wc[k]); }
    a = x;
    b = y;
    c = z;
}

// Pipelined block-Jacobi preconditioned CG (P. Ghysels, W. Vanroose, Parallel Computing
// 40 (2014) 224-238, the preconditioned pipelined CG): the iterates of k_pcg in exact
// arithmetic, rearranged so that both inner products of an iteration (r.u, w.u) are
// reduced together with the publication of m = P^-1 w, whose product n = M m is then
// formed locally.  One grid barrier per iteration (k_pcg needs two; the tiled product
// of large systems adds its own).  Published vectors and block partials alternate
// between two buffers with the barrier count: set k is written before barrier k and
// read right after it; the same buffer is written again (set k + 2) only after barrier
// k + 1, which no block passes before it has finished reading set k.  The result is
// accepted on the true residual b - M x; otherwise the recurrence restarts from it.
__global__ void __launch_bounds__(kPcgPipeThreads, 2) k_pcg_pipe(PCGArgs A)
{
    extern __shared__ double sm[];
    constexpr int GL = kPcgMaxBlock + 1;
    const int4 pt = A.part[blockIdx.x];
    const int row0 = pt.x, row1 = pt.y, nrow = row1 - row0;
    const long long boff0 = pt.z < pt.w ? A.boff[pt.z] : 0;
    const int R = A.maxrows;
    double* v = sm;                              // n: operand of the next product, replicated
    double* G = v + ((A.n + 1) & ~1);            // kPcgMaxBlock x GL scratch
    double* xs = G + kPcgMaxBlock * GL;          // owned rows of x r u w z q s p m n
    double* rs = xs + R;
    double* us = rs + R;
    double* ws = us + R;
    double* zs = ws + R;
    double* qs = zs + R;
    double* ss = qs + R;
    double* ps = ss + R;
    double* ms = ps + R;
    double* ns = ms + R;
    double* Bs = ns + R;                         // inverses of the owned blocks
    int4* meta = reinterpret_cast<int4*>(Bs + A.maxinv);
    __shared__ unsigned int gen;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + kBarGen);
    pcg_setup(A, pt, boff0, G, Bs, meta, MStored{&A});
    const double* Bp = A.binv_pre ? A.binv_pre + boff0 : Bs;
    bool ok = true;
    int phase = 0;   // barrier count: selects the published vector and partial set
    // out = (M v) for the owned rows, v replicated in shared memory
    auto product = [&](double* out) {
        if (A.lower) {
            matvec_tiles(A, v, G);
            ok = grid_sync(A.bar, gen) && ok;
            ++phase;
            take_tiles_result(A, row0, nrow, out);
        } else {
            matvec_rows(A, v, row0, row1, out);
            __syncthreads();
        }
    };
    // publish the owned rows of src, barrier, replicate the whole vector into v
    auto publish = [&](const double* src, double pa, double pb, double pc, double& ta, double& tb, double& tc) {
        double* pub = (phase & 1) ? A.z2 : A.z;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(pub + row0 + k, src[k]);
        block_sum3(pa, pb, pc, A.partial + 8 * blockIdx.x + 4 * (phase & 1));
        ok = grid_sync(A.bar, gen) && ok;
        grid_totals3(A.partial, 4 * (phase & 1), ta, tb, tc);
        update_p(v, pub, A.n, 0.0);
        ++phase;
        __syncthreads();
    };
    // ---- start: x0 (previous solution or 0), r = b - M x0, u = P^-1 r, w = M u
    const bool warm = A.warm != nullptr && *A.warm != 0;
    if (warm) {
        update_p(v, A.x, A.n, 0.0);
        __syncthreads();
        product(ns);
    }
    double bmax_t = 0.0;
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        const double bv = A.b[row0 + k];
        xs[k] = warm ? v[row0 + k] : 0.0;
        rs[k] = warm ? bv - ns[k] : bv;
        zs[k] = qs[k] = ss[k] = ps[k] = 0.0;
        bmax_t = fmax(bmax_t, fabs(bv));
    }
    __syncthreads();
    apply_precond(nrow, meta, Bp, rs, us);
    double bmax = 0.0, t1, t2;
    publish(us, 0.0, 0.0, bmax_t, t1, t2, bmax);
    product(ws);
    int it = 0;
    bool conv = ok && bmax == 0.0, first = true;
    double gam_prev = 1.0, alpha_prev = 1.0;
    while (ok && !conv && it < A.max_iter) {
        double g_t = 0.0, d_t = 0.0, rm_t = 0.0;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            g_t += rs[k] * us[k];
            d_t += ws[k] * us[k];
            rm_t = fmax(rm_t, fabs(rs[k]));
        }
        __syncthreads();
        apply_precond(nrow, meta, Bp, ws, ms);
        double gam, del, rmax;
        publish(ms, g_t, d_t, rm_t, gam, del, rmax);
        if (!ok) break;
        if (rmax <= pcg_threshold(A, bmax)) {
            // accept only on the true residual r = b - M x; otherwise restart from it
            double u1, u2;
            publish(xs, 0.0, 0.0, 0.0, u1, u2, u1);
            if (!ok) break;
            product(ns);
            double rt = 0.0;
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
                rs[k] = A.b[row0 + k] - ns[k];
                rt = fmax(rt, fabs(rs[k]));
            }
            __syncthreads();
            apply_precond(nrow, meta, Bp, rs, us);
            double rtrue;
            publish(us, 0.0, 0.0, rt, u1, u2, rtrue);
            if (!ok) break;
            if (rtrue <= pcg_threshold(A, bmax)) {
                conv = true;
                break;
            }
            product(ws);
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) zs[k] = qs[k] = ss[k] = ps[k] = 0.0;
            __syncthreads();
            first = true;
            continue;
        }
        ++it;
        product(ns);
        double beta, alpha;
        if (first) {
            beta = 0.0;
            alpha = gam / del;
        } else {
            beta = gam / gam_prev;
            alpha = gam / (del - beta * gam / alpha_prev);
        }
        first = false;
        gam_prev = gam;
        alpha_prev = alpha;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            const double z = ns[k] + beta * zs[k], q = ms[k] + beta * qs[k];
            const double sv = ws[k] + beta * ss[k], pv = us[k] + beta * ps[k];
            zs[k] = z; qs[k] = q; ss[k] = sv; ps[k] = pv;
            xs[k] += alpha * pv;
            rs[k] -= alpha * sv;
            us[k] -= alpha * q;
            ws[k] -= alpha * z;
        }
        __syncthreads();
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) A.x[row0 + k] = xs[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.info = !ok ? 2 : (conv ? 0 : 3);
        *A.iters = it;
        if (A.warm) *A.warm = (ok && conv) ? 1 : 0;
    }
}

}  // namespace

namespace {

// ------------------------------------------------------------------------------------
// Shared-memory resident PCG for reduced systems whose lower triangle fits the SMs'
// shared memory (up to ~2400 unknowns on 148 SMs).  Each block builds its 64x64 lower
// tiles of M straight from the atoms at launch (no HBM matrix, no separate build kernel)
// and keeps them for every product of the solve; a product adds each tile's row part and
// transposed part into an L2 vector with FP64 atomics (one barrier), as matvec_tiles does
// from HBM.  The iteration is the pipelined CG of k_pcg_pipe; the preconditioner blocks
// are formed from the atoms too.
// ------------------------------------------------------------------------------------
struct PCGRes {
    View V;
    const int* red2atom;
    const int* anchor;
    const int2* tiles;   // 64 x 64 lower tiles {I0, J0}, dealt round-robin to the blocks
    int ntiles;
    int ntl;             // tiles per block (the most any block holds)
    int gscratch;        // 1: preconditioner blocks beyond kPcgWarpMax need the G scratch
};
constexpr int kResT = 64, kResLd = kResT + 1;

// element (r, c) of the reduced matrix from the atoms (same operations as k_eeq_M_tiles)
struct MAtoms {
    const PCGRes* R;
    __device__ __forceinline__ double operator()(int r, int c) const
    {
        const View& V = R->V;
        const int k = R->red2atom[r], ak = R->anchor[k], l = R->red2atom[c], al = R->anchor[l];
        return eeq_a(V, k, l) - eeq_a(V, k, al) - eeq_a(V, ak, l) + eeq_a(V, ak, al);
    }
};

// builds tile (I0, J0) into T (column-major, leading dimension kResLd); the tile's row
// and column atoms (and anchors) are staged in shared memory first
__device__ void res_build_tile(const PCGRes& R, int n, int I0, int J0, double* T)
{
    __shared__ double bx[4][kResT], by[4][kResT], bz[4][kResT], ba[4][kResT], bd[4][kResT];
    __shared__ int bid[4][kResT];
    const View& V = R.V;
    __syncthreads();
    for (int e = threadIdx.x; e < 4 * kResT; e += blockDim.x) {
        const int w = e / kResT, t = e % kResT;
        const int idx = (w < 2 ? I0 : J0) + t;
        int a = -1;
        if (idx < n) {
            const int k = R.red2atom[idx];
            a = (w & 1) ? R.anchor[k] : k;
        }
        bid[w][t] = a;
        if (a >= 0) {
            const double4 p = V.pos[a];
            bx[w][t] = p.x; by[w][t] = p.y; bz[w][t] = p.z;
            ba[w][t] = V.alpeeq[a];
            bd[w][t] = V.adiag[a];
        }
    }
    __syncthreads();
    auto el = [&](int wa, int ia, int wb, int ib) {
        if (bid[wa][ia] == bid[wb][ib]) return bd[wa][ia];
        const double dx = bx[wa][ia] - bx[wb][ib], dy = by[wa][ia] - by[wb][ib], dz = bz[wa][ia] - bz[wb][ib];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double s = ba[wa][ia] + ba[wb][ib];
        if (d2 >= 36.0 * s) return rsqrt(d2);
        const double r = sqrt(d2);
        return erf(r / sqrt(s)) / r;
    };
    const bool diag = I0 == J0;
    for (int e = threadIdx.x; e < kResT * kResT; e += blockDim.x) {
        const int c = e / kResT, r = e % kResT;
        double v = 0.0;
        if (I0 + r < n && J0 + c < n && (!diag || r >= c))
            v = el(0, r, 2, c) - el(0, r, 3, c) - el(1, r, 2, c) + el(1, r, 3, c);
        T[c * kResLd + r] = v;
    }
}

// y += M v over the block's resident tiles: two tile groups of 128 threads, in each the
// first 64 threads form the row sums u_r, the next 64 the column sums w_c
__device__ void res_product(const PCGArgs& A, const PCGRes& R, const double* tl, int ntl, const double* v)
{
    const int g = threadIdx.x >> 7, t = threadIdx.x & 127, ng = blockDim.x >> 7;
    for (int k = g; k < ntl; k += ng) {
        const int2 tp = R.tiles[blockIdx.x + k * gridDim.x];
        const int I0 = tp.x, J0 = tp.y;
        const bool diag = I0 == J0;
        const int ni = min(kResT, A.n - I0), nj = min(kResT, A.n - J0);
        const double* T = tl + (size_t)k * kResT * kResLd;
        if (t < kResT) {
            const int r = t;
            if (r < ni) {
                double u0 = 0.0, u1 = 0.0;
                const int cmax = diag ? r + 1 : nj;
                int c = 0;
                for (; c + 1 < cmax; c += 2) {
                    u0 += T[c * kResLd + r] * v[J0 + c];
                    u1 += T[(c + 1) * kResLd + r] * v[J0 + c + 1];
                }
                if (c < cmax) u0 += T[c * kResLd + r] * v[J0 + c];
                atomicAdd(A.yA + I0 + r, u0 + u1);
            }
        } else {
            const int c = t - kResT;
            if (c < nj) {
                double w0 = 0.0, w1 = 0.0;
                int r = diag ? c + 1 : 0;
                for (; r + 1 < ni; r += 2) {
                    w0 += T[c * kResLd + r] * v[I0 + r];
                    w1 += T[c * kResLd + r + 1] * v[I0 + r + 1];
                }
                if (r < ni) w0 += T[c * kResLd + r] * v[I0 + r];
                if (w0 + w1 != 0.0) atomicAdd(A.yA + J0 + c, w0 + w1);
            }
        }
    }
}

__global__ void __launch_bounds__(kPcgPipeThreads, 1) k_pcg_res(PCGArgs A, PCGRes R)
{
    extern __shared__ double sm[];
    constexpr int GL = kPcgMaxBlock + 1;
    const int4 pt = A.part[blockIdx.x];
    const int row0 = pt.x, row1 = pt.y, nrow = row1 - row0;
    const long long boff0 = pt.z < pt.w ? A.boff[pt.z] : 0;
    const int RR = A.maxrows;
    double* v = sm;                                      // n: operand, replicated
    double* tl = v + ((A.n + 1) & ~1);                   // R.ntl resident tiles
    double* G = tl + (size_t)R.ntl * kResT * kResLd;     // scratch for large preconditioner blocks
    double* xs = G + (R.gscratch ? kPcgMaxBlock * GL : 0);
    double* rs = xs + RR;
    double* us = rs + RR;
    double* ws = us + RR;
    double* zs = ws + RR;
    double* qs = zs + RR;
    double* ss = qs + RR;
    double* ps = ss + RR;
    double* ms = ps + RR;
    double* ns = ms + RR;
    double* Bs = ns + RR;
    int4* meta = reinterpret_cast<int4*>(Bs + A.maxinv);
    __shared__ unsigned int gen;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + kBarGen);
    int ntl = 0;
    for (int t = blockIdx.x; t < R.ntiles; t += gridDim.x, ++ntl) {
        const int2 tp = R.tiles[t];
        res_build_tile(R, A.n, tp.x, tp.y, tl + (size_t)ntl * kResT * kResLd);
    }
    pcg_setup(A, pt, boff0, G, Bs, meta, MAtoms{&R});
    const double* Bp = A.binv_pre ? A.binv_pre + boff0 : Bs;
    bool ok = true;
    int phase = 0;
    auto product = [&](double* out) {
        res_product(A, R, tl, ntl, v);
        ok = grid_sync(A.bar, gen) && ok;
        ++phase;
        take_tiles_result(A, row0, nrow, out);
    };
    auto publish = [&](const double* src, double pa, double pb, double pc, double& ta, double& tb, double& tc) {
        double* pub = (phase & 1) ? A.z2 : A.z;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) __stcg(pub + row0 + k, src[k]);
        block_sum3(pa, pb, pc, A.partial + 8 * blockIdx.x + 4 * (phase & 1));
        ok = grid_sync(A.bar, gen) && ok;
        grid_totals3(A.partial, 4 * (phase & 1), ta, tb, tc);
        update_p(v, pub, A.n, 0.0);
        ++phase;
        __syncthreads();
    };
    // ---- start: x0 (previous solution or 0), r = b - M x0, u = P^-1 r, w = M u
    const bool warm = A.warm != nullptr && *A.warm != 0;
    if (warm) {
        update_p(v, A.x, A.n, 0.0);
        __syncthreads();
        product(ns);
    }
    double bmax_t = 0.0;
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
        const double bv = A.b[row0 + k];
        xs[k] = warm ? v[row0 + k] : 0.0;
        rs[k] = warm ? bv - ns[k] : bv;
        zs[k] = qs[k] = ss[k] = ps[k] = 0.0;
        bmax_t = fmax(bmax_t, fabs(bv));
    }
    __syncthreads();
    apply_precond(nrow, meta, Bp, rs, us);
    double bmax = 0.0, t1, t2;
    publish(us, 0.0, 0.0, bmax_t, t1, t2, bmax);
    product(ws);
    int it = 0;
    bool conv = ok && bmax == 0.0, first = true;
    double gam_prev = 1.0, alpha_prev = 1.0;
    while (ok && !conv && it < A.max_iter) {
        double g_t = 0.0, d_t = 0.0, rm_t = 0.0;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            g_t += rs[k] * us[k];
            d_t += ws[k] * us[k];
            rm_t = fmax(rm_t, fabs(rs[k]));
        }
        __syncthreads();
        apply_precond(nrow, meta, Bp, ws, ms);
        double gam, del, rmax;
        publish(ms, g_t, d_t, rm_t, gam, del, rmax);
        if (!ok) break;
        if (rmax <= pcg_threshold(A, bmax)) {
            double u1, u2;
            publish(xs, 0.0, 0.0, 0.0, u1, u2, u1);
            if (!ok) break;
            product(ns);
            double rt = 0.0;
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
                rs[k] = A.b[row0 + k] - ns[k];
                rt = fmax(rt, fabs(rs[k]));
            }
            __syncthreads();
            apply_precond(nrow, meta, Bp, rs, us);
            double rtrue;
            publish(us, 0.0, 0.0, rt, u1, u2, rtrue);
            if (!ok) break;
            if (rtrue <= pcg_threshold(A, bmax)) {
                conv = true;
                break;
            }
            product(ws);
            for (int k = threadIdx.x; k < nrow; k += blockDim.x) zs[k] = qs[k] = ss[k] = ps[k] = 0.0;
            __syncthreads();
            first = true;
            continue;
        }
        ++it;
        product(ns);
        double beta, alpha;
        if (first) {
            beta = 0.0;
            alpha = gam / del;
        } else {
            beta = gam / gam_prev;
            alpha = gam / (del - beta * gam / alpha_prev);
        }
        first = false;
        gam_prev = gam;
        alpha_prev = alpha;
        for (int k = threadIdx.x; k < nrow; k += blockDim.x) {
            const double z = ns[k] + beta * zs[k], q = ms[k] + beta * qs[k];
            const double sv = ws[k] + beta * ss[k], pv = us[k] + beta * ps[k];
            zs[k] = z; qs[k] = q; ss[k] = sv; ps[k] = pv;
            xs[k] += alpha * pv;
            rs[k] -= alpha * sv;
            us[k] -= alpha * q;
            ws[k] -= alpha * z;
        }
        __syncthreads();
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nrow; k += blockDim.x) A.x[row0 + k] = xs[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.info = !ok ? 2 : (conv ? 0 : 3);
        *A.iters = it;
        if (A.warm) *A.warm = (ok && conv) ? 1 : 0;
    }
}

}  // namespace
