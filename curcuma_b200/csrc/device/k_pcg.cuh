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

constexpr int kPcgThreads = 512;
constexpr int kPcgMaxBlock = 64;   // largest preconditioner block

struct PCGArgs {
    const double* M;
    int lda, n;
    const double* b;
    double* x;            // solution
    double* r;            // residual
    double* z;            // preconditioned residual
    const int2* blocks;   // preconditioner blocks {first row, size}
    const long long* boff;
    double* binv;         // inverse of every block (row-major, size^2)
    const int4* part;     // per grid block: rows [x, y), preconditioner blocks [z, w)
    const int* rblk;      // preconditioner block of every row
    double* partial;      // gridDim.x * 4
    unsigned int* bar;    // {arrival count, generation}
    int* info;
    int* iters;
    int max_iter;
    double tol;           // converged when max|b - M x| <= tol * max|b|
};

// grid-wide barrier (all blocks co-resident); false when the wait gave up
__device__ bool grid_sync(unsigned int* bar, unsigned int& gen)
{
    __shared__ int ok_s;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        ok_s = 1;
        const unsigned int want = gen + 1;
        if (atomicAdd(bar, 1u) + 1u == gridDim.x) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long polls = 0;
            while ((int)(*(volatile unsigned int*)(bar + 1) - want) < 0) {
                if (++polls > (1ll << 22)) {
                    ok_s = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
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

// the same totals in every block: warp 0 reads the partials (lane l takes blocks l,
// l + 32, ...) and combines them in a fixed order, so every block gets identical sums
__device__ void grid_totals(const double* partial, int slot, double& sum, double& mx)
{
    __shared__ double t0, t1;
    __syncthreads();
    if (threadIdx.x < 32) {
        double a = 0.0, b = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) {
            a += __ldcg(partial + 4 * k + slot);
            b = fmax(b, __ldcg(partial + 4 * k + slot + 1));
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if (threadIdx.x == 0) {
            t0 = a;
            t1 = b;
        }
    }
    __syncthreads();
    sum = t0;
    mx = t1;
}

// z = P^-1 r on the owned rows (one thread per row, rblk[r] = its preconditioner block);
// returns the thread's part of r.z
__device__ double apply_precond(const PCGArgs& A, int row0, int row1)
{
    double rz = 0.0;
    for (int rr = row0 + threadIdx.x; rr < row1; rr += blockDim.x) {
        const int bk = A.rblk[rr];
        const int2 bl = A.blocks[bk];
        const double* Bi = A.binv + A.boff[bk] + (size_t)(rr - bl.x) * bl.y;
        double s = 0.0;
        for (int j = 0; j < bl.y; ++j) s += __ldcg(Bi + j) * __ldcg(A.r + bl.x + j);
        __stcg(A.z + rr, s);
        rz += s * __ldcg(A.r + rr);
    }
    return rz;
}

// out[r - row0] = (M v)_r for the owned rows; the rows are shared out to the warps, each
// lane keeps four independent partial sums so that several loads are in flight.
// Returns the thread's part of sum_r v_r (M v)_r.
__device__ double matvec_rows(const PCGArgs& A, const double* v, int row0, int row1, double* out)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double vmv = 0.0;
    for (int rr = row0 + warp; rr < row1; rr += nw) {
        const double* col = A.M + (size_t)rr * A.lda;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int c = lane;
        for (; c + 96 < A.n; c += 128) {
            s0 += col[c] * v[c];
            s1 += col[c + 32] * v[c + 32];
            s2 += col[c + 64] * v[c + 64];
            s3 += col[c + 96] * v[c + 96];
        }
        for (; c < A.n; c += 32) s0 += col[c] * v[c];
        double s = (s0 + s1) + (s2 + s3);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            out[rr - row0] = s;
            vmv += s * v[rr];
        }
    }
    return vmv;
}

// inverse of a preconditioner block of at most kPcgSmall rows by one thread
// (Gauss-Jordan in registers-sized local storage)
constexpr int kPcgSmall = 4;
__device__ void invert_small(const PCGArgs& A, int bk)
{
    const int2 bl = A.blocks[bk];
    const int s = bl.y;
    double g[kPcgSmall][kPcgSmall], inv[kPcgSmall][kPcgSmall];
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) {
            g[i][j] = A.M[(size_t)(bl.x + j) * A.lda + bl.x + i];
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
    double* I = A.binv + A.boff[bk];
    for (int i = 0; i < s; ++i)
        for (int j = 0; j < s; ++j) __stcg(I + i * s + j, inv[i][j]);
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg(PCGArgs A)
{
    extern __shared__ double sm[];
    constexpr int GL = kPcgMaxBlock + 1;
    double* p = sm;                              // n
    double* G = sm + A.n;                        // kPcgMaxBlock x GL
    double* Ap = G + kPcgMaxBlock * GL;          // rows of this block
    __shared__ unsigned int gen;
    __shared__ double piv;
    const int4 pt = A.part[blockIdx.x];
    const int row0 = pt.x, row1 = pt.y;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + 1);
    // ---- inverse of every owned preconditioner block (Gauss-Jordan on [M_bb | I]; SPD,
    // no pivoting): M_bb in shared memory, the inverse built in place in binv
    for (int bk = pt.z + threadIdx.x; bk < pt.w; bk += blockDim.x)
        if (A.blocks[bk].y <= kPcgSmall) invert_small(A, bk);
    for (int bk = pt.z; bk < pt.w; ++bk) {
        const int2 bl = A.blocks[bk];
        const int s = bl.y;
        if (s <= kPcgSmall) continue;
        double* I = A.binv + A.boff[bk];
        __syncthreads();
        for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
            const int i = e / s, j = e % s;
            G[i * GL + j] = A.M[(size_t)(bl.x + j) * A.lda + bl.x + i];
            __stcg(I + e, i == j ? 1.0 : 0.0);
        }
        __syncthreads();
        for (int c = 0; c < s; ++c) {
            if (threadIdx.x == 0) piv = 1.0 / G[c * GL + c];
            __syncthreads();
            const double pv = piv;
            for (int j = threadIdx.x; j < s; j += blockDim.x) {
                G[c * GL + j] *= pv;
                __stcg(I + c * s + j, __ldcg(I + c * s + j) * pv);
            }
            __syncthreads();
            for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
                const int i = e / s, j = e % s;
                if (i == c) continue;
                __stcg(I + i * s + j, __ldcg(I + i * s + j) - G[i * GL + c] * __ldcg(I + c * s + j));
            }
            __syncthreads();
            for (int e = threadIdx.x; e < s * s; e += blockDim.x) {
                const int i = e / s, j = e % s;
                if (i == c || j == c) continue;
                G[i * GL + j] -= G[i * GL + c] * G[c * GL + j];
            }
            __syncthreads();
            for (int i = threadIdx.x; i < s; i += blockDim.x)
                if (i != c) G[i * GL + c] = 0.0;
            __syncthreads();
        }
    }
    __syncthreads();
    // ---- x = 0, r = b, z = P^-1 r
    double bmax_t = 0.0;
    for (int rr = row0 + threadIdx.x; rr < row1; rr += blockDim.x) {
        const double bv = A.b[rr];
        __stcg(A.x + rr, 0.0);
        __stcg(A.r + rr, bv);
        bmax_t = fmax(bmax_t, fabs(bv));
    }
    __syncthreads();
    double rz_t = apply_precond(A, row0, row1);
    block_sum_max(rz_t, bmax_t, A.partial + 4 * blockIdx.x);
    bool ok = grid_sync(A.bar, gen);
    double rz = 0.0, bmax = 0.0;
    if (ok) grid_totals(A.partial, 0, rz, bmax);
    for (int c = threadIdx.x; c < A.n; c += blockDim.x) p[c] = __ldcg(A.z + c);
    int it = 0;
    bool conv = ok && bmax == 0.0;
    while (ok && !conv && it < A.max_iter) {
        ++it;
        __syncthreads();
        const double pap_t = matvec_rows(A, p, row0, row1, Ap);
        block_sum_max(pap_t, 0.0, A.partial + 4 * blockIdx.x);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        double pap, unused;
        grid_totals(A.partial, 0, pap, unused);
        const double alpha = rz / pap;
        double rmax_t = 0.0;
        for (int rr = row0 + threadIdx.x; rr < row1; rr += blockDim.x) {
            __stcg(A.x + rr, __ldcg(A.x + rr) + alpha * p[rr]);
            const double nr = __ldcg(A.r + rr) - alpha * Ap[rr - row0];
            __stcg(A.r + rr, nr);
            rmax_t = fmax(rmax_t, fabs(nr));
        }
        __syncthreads();
        rz_t = apply_precond(A, row0, row1);
        block_sum_max(rz_t, rmax_t, A.partial + 4 * blockIdx.x + 2);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        double rzn, rmax;
        grid_totals(A.partial, 2, rzn, rmax);
        if (rmax <= A.tol * bmax) {
            // accept only on the true residual r = b - M x; otherwise restart from it
            for (int c = threadIdx.x; c < A.n; c += blockDim.x) p[c] = __ldcg(A.x + c);
            __syncthreads();
            matvec_rows(A, p, row0, row1, Ap);
            __syncthreads();
            rmax_t = 0.0;
            for (int rr = row0 + threadIdx.x; rr < row1; rr += blockDim.x) {
                const double tr = A.b[rr] - Ap[rr - row0];
                __stcg(A.r + rr, tr);
                rmax_t = fmax(rmax_t, fabs(tr));
            }
            __syncthreads();
            rz_t = apply_precond(A, row0, row1);
            block_sum_max(rz_t, rmax_t, A.partial + 4 * blockIdx.x + 2);
            ok = grid_sync(A.bar, gen);
            if (!ok) break;
            grid_totals(A.partial, 2, rzn, rmax);
            if (rmax <= A.tol * bmax) {
                conv = true;
                break;
            }
            rz = rzn;
            for (int c = threadIdx.x; c < A.n; c += blockDim.x) p[c] = __ldcg(A.z + c);
            continue;
        }
        const double beta = rzn / rz;
        rz = rzn;
        for (int c = threadIdx.x; c < A.n; c += blockDim.x) p[c] = __ldcg(A.z + c) + beta * p[c];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.info = !ok ? 2 : (conv ? 0 : 3);
        *A.iters = it;
    }
}

}  // namespace
