// Dense solves of the reduced EEQ system without a library:
//  * k_lu_factor + k_lu_back: LU with partial pivoting for an indefinite reduced matrix
//    (curcuma falls back from its Cholesky to a pivoted LU, eeq_solver.cpp:1448-2086); the
//    right-hand side is eliminated along with the matrix, so the back substitution finishes
//    the solve;
//  * k_lu_solve_rhs, k_chol_solve_rhs: a further right-hand side (the exact-gradient mode's
//    charge response) with the LU factor and pivots, or with a Cholesky factor L in M.
// M is column-major with leading dimension lda (element (r, c) at M[c * lda + r]).  These
// paths are rare (an indefinite matrix; exact-gradient mode after a direct factorisation), so
// they favour simplicity: an unblocked right-looking LU in one cooperative kernel (four grid
// barriers per pivot, bounded waits), single-block substitutions.
// Included inside namespace gfnff by engine.cu, after k_pcg.cuh (grid_sync, kBarGen).
#pragma once

namespace {

constexpr int kLuThreads = 512;

struct LUArgs {
    double* M;
    int lda, n;
    double* b;              // right-hand side, eliminated with the matrix (-> L^-1 P b)
    int* ipiv;              // n: row exchanged with row k at step k
    int* info;              // 0 ok, 1 singular (a zero pivot column), 2 a barrier wait gave up
    double* partial;        // 2 per grid block: pivot candidate (|value|, row)
    unsigned int* bar;      // grid barrier: arrival count at [0], generation at [kBarGen]
};

// LU with partial pivoting, one cooperative launch of gridDim.x blocks (all co-resident).
// Step k: pivot search over rows >= k of column k (largest magnitude, ties to the smaller
// row; every block reduces the blocks' candidates in the same order), row exchange across all
// columns and b, scaling of column k below the diagonal, rank-1 update of the trailing columns
// (block-cyclic over columns, threads over rows) and of b.
__global__ void __launch_bounds__(kLuThreads) k_lu_factor(LUArgs A)
{
    __shared__ unsigned int gen;
    __shared__ double wv[kLuThreads / 32];
    __shared__ int wi[kLuThreads / 32];
    __shared__ double s_amax;
    __shared__ int s_piv;
    if (threadIdx.x == 0) gen = *(volatile unsigned int*)(A.bar + kBarGen);
    __syncthreads();
    const int n = A.n, lda = A.lda;
    const long gt = (long)blockIdx.x * blockDim.x + threadIdx.x, gs = (long)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool ok = true;
    int info = 0;
    for (int k = 0; k < n; ++k) {
        double* ck = A.M + (size_t)k * lda;
        // ---- pivot search
        double bv = -1.0;
        int bi = n;
        for (long i = k + gt; i < n; i += gs) {
            const double v = fabs(__ldcg(ck + i));
            if (v > bv) {
                bv = v;
                bi = (int)i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            wv[warp] = bv;
            wi[warp] = bi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
                if (wv[w] > bv || (wv[w] == bv && wi[w] < bi)) {
                    bv = wv[w];
                    bi = wi[w];
                }
            __stcg(A.partial + 2 * blockIdx.x, bv);
            __stcg(A.partial + 2 * blockIdx.x + 1, (double)bi);
        }
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        if (threadIdx.x == 0) {
            double v = -1.0;
            int r = n;
            for (int g = 0; g < (int)gridDim.x; ++g) {
                const double gv = __ldcg(A.partial + 2 * g);
                const int gr = (int)__ldcg(A.partial + 2 * g + 1);
                if (gv > v || (gv == v && gr < r)) {
                    v = gv;
                    r = gr;
                }
            }
            s_amax = v;
            s_piv = r;
        }
        __syncthreads();
        const int piv = s_piv;
        if (!(s_amax > 0.0)) {   // uniform: every block reduced the same candidates
            info = 1;
            break;
        }
        if (gt == 0) A.ipiv[k] = piv;
        // ---- row exchange k <-> piv in every column and in b
        if (piv != k) {
            for (long c = gt; c <= n; c += gs) {
                double* col = c < n ? A.M + (size_t)c * lda : A.b;
                const double x = __ldcg(col + k), y = __ldcg(col + piv);
                __stcg(col + k, y);
                __stcg(col + piv, x);
            }
        }
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        // ---- column k below the diagonal: l_ik = a_ik / a_kk
        const double akk = __ldcg(ck + k);
        for (long i = k + 1 + gt; i < n; i += gs) __stcg(ck + i, __ldcg(ck + i) / akk);
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
        // ---- trailing columns (j = n is b): a_ij -= l_ik a_kj for i > k
        for (long j = k + 1 + blockIdx.x; j <= n; j += gridDim.x) {
            double* cj = j < n ? A.M + (size_t)j * lda : A.b;
            const double akj = __ldcg(cj + k);
            if (akj != 0.0)
                for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) __stcg(cj + i, __ldcg(cj + i) - __ldcg(ck + i) * akj);
        }
        ok = grid_sync(A.bar, gen);
        if (!ok) break;
    }
    if (gt == 0) *A.info = !ok ? 2 : info;
}

// U x = y in place on y (U: the upper triangle of the LU factor), one block
__device__ void lu_back_block(const double* M, int lda, int n, double* y)
{
    __shared__ double xk;
    for (int k = n - 1; k >= 0; --k) {
        __syncthreads();
        if (threadIdx.x == 0) {
            xk = y[k] / M[(size_t)k * lda + k];
            y[k] = xk;
        }
        __syncthreads();
        const double* ck = M + (size_t)k * lda;
        for (int i = threadIdx.x; i < k; i += blockDim.x) y[i] -= ck[i] * xk;
    }
    __syncthreads();
}

// back substitution of the solve (the factor is valid only when info == 0)
__global__ void __launch_bounds__(1024) k_lu_back(const double* M, int lda, int n, double* y, const int* info)
{
    if (*info != 0) return;
    lu_back_block(M, lda, n, y);
}

// a further right-hand side r with the LU factor: r <- P r, L z = r (unit L), U x = z
__global__ void __launch_bounds__(1024) k_lu_solve_rhs(const double* M, int lda, int n, const int* ipiv,
                                                       double* r, const int* info)
{
    if (*info != 0) return;
    if (threadIdx.x == 0)
        for (int k = 0; k < n; ++k) {
            const int p = ipiv[k];
            if (p != k) {
                const double t = r[k];
                r[k] = r[p];
                r[p] = t;
            }
        }
    for (int k = 0; k < n; ++k) {
        __syncthreads();
        const double rk = r[k];
        const double* ck = M + (size_t)k * lda;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) r[i] -= ck[i] * rk;
    }
    lu_back_block(M, lda, n, r);
}

// a further right-hand side r with a Cholesky factor L (lower triangle of M, L_kk on the
// diagonal): L z = r, then L^T x = z (row k of L read across the columns)
__global__ void __launch_bounds__(1024) k_chol_solve_rhs(const double* M, int lda, int n, double* r, const int* info)
{
    if (*info != 0) return;
    __shared__ double xk;
    for (int k = 0; k < n; ++k) {
        __syncthreads();
        if (threadIdx.x == 0) {
            xk = r[k] / M[(size_t)k * lda + k];
            r[k] = xk;
        }
        __syncthreads();
        const double* ck = M + (size_t)k * lda;
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) r[i] -= ck[i] * xk;
    }
    for (int k = n - 1; k >= 0; --k) {
        __syncthreads();
        if (threadIdx.x == 0) {
            xk = r[k] / M[(size_t)k * lda + k];
            r[k] = xk;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < k; j += blockDim.x) r[j] -= M[(size_t)j * lda + k] * xk;
    }
}

}  // namespace
