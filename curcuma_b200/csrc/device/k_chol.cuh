// Dense SPD solve of the reduced EEQ system in one persistent kernel (FP64).
//
// The matrix is stored column-major (lower triangle used) with one extra row holding the
// right-hand side b: factoring [[M, .], [b^T, .]] produces L in the first n rows and
// z = L^-1 b in row n, so the forward substitution comes free with the factorisation.
// The backward substitution L^T y = z follows as the last tasks.
//
// Work is split into 64 x 64 tiles and tasks (POTRF of a diagonal tile, TRSM of a tile
// below it, GEMM update of a trailing tile, BSOLVE of one tile of y).  Every block of a
// cooperative launch (all blocks co-resident) takes the next task of a host-built list
// in topological order and waits on per-tile counters for the tiles it needs.  Because a
// task only depends on tasks listed before it, the oldest unfinished task can always
// run, so the schedule cannot deadlock; the list puts the next panel's factorisation
// right after the updates it needs (look-ahead), so the critical path of diagonal
// factorisations overlaps the trailing updates.  Every wait gives up after a bounded
// number of polls and reports it in err.
// Included inside namespace gfnff by engine.cu (one translation unit).
#pragma once

namespace {

constexpr int CB = 64;          // tile edge
constexpr int CLD = CB + 1;     // padded shared-memory leading dimension
constexpr int kCholThreads = 256;
enum { TASK_POTRF = 0, TASK_TRSM = 1, TASK_GEMM = 2, TASK_BSOLVE = 3 };

struct CholArgs {
    double* M;          // column-major, lda rows; row n holds b
    int lda, n, nt;     // n pivots, nt tiles per side of the (n+1) x n augmented matrix
    const int4* tasks;  // {type, i, j, k}
    int ntasks;
    int* next;          // task counter
    int* cnt;           // nt*nt: updates applied to tile (i, j)
    int* fin;           // nt*nt: tile (i, j) of L final
    int* ydone;         // nt: tile k of y final
    double* rdiag;      // n: 1 / L_cc
    double* y;          // n: solution
    int* err;           // bit 0: not positive definite, bit 1: wait gave up
};

constexpr long long kMaxPolls = 1ll << 22;   // x ~0.5 us per poll

// rows of tile i (the augmented row included), pivot columns of tile k
__device__ __forceinline__ int tile_rows(const CholArgs& A, int i) { return min(CB, A.n + 1 - i * CB); }
__device__ __forceinline__ int tile_cols(const CholArgs& A, int k) { return max(0, min(CB, A.n - k * CB)); }

// thread 0 waits until *flag >= want; false when it gave up
__device__ bool wait_flag(const int* flag, int want, int* err)
{
    long long polls = 0;
    while (*(volatile const int*)flag < want) {
        if (++polls > kMaxPolls) {
            atomicOr(err, 2);
            return false;
        }
        __nanosleep(64);
    }
    __threadfence();
    return true;
}

// every thread fences its own global stores, then thread 0 raises the flag
__device__ __forceinline__ void publish(int* flag, int v)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(flag, v);
}

// tile (i, j) -> shared memory S[c*CLD + r] (rows x cols, zero elsewhere)
__device__ void load_tile(const CholArgs& A, int i, int j, int rows, int cols, double* S)
{
    const double* src = A.M + (size_t)(j * CB) * A.lda + i * CB;
    for (int e = threadIdx.x; e < CB * CB; e += blockDim.x) {
        const int r = e & (CB - 1), c = e >> 6;
        S[c * CLD + r] = (r < rows && c < cols) ? __ldcg(src + (size_t)c * A.lda + r) : 0.0;
    }
}

__device__ void store_tile(const CholArgs& A, int i, int j, int rows, int cols, const double* S)
{
    double* dst = A.M + (size_t)(j * CB) * A.lda + i * CB;
    for (int e = threadIdx.x; e < CB * CB; e += blockDim.x) {
        const int r = e & (CB - 1), c = e >> 6;
        if (r < rows && c < cols) __stcg(dst + (size_t)c * A.lda + r, S[c * CLD + r]);
    }
}

// Cholesky of the diagonal tile in shared memory (Crout order, four threads per row);
// rows beyond the pivot columns (the augmented row) get their L entries as well
__device__ bool potrf_tile(double* S, int rows, int cols, double* rdiag_out)
{
    __shared__ double piv;
    __shared__ int bad;
    const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    for (int c = 0; c < cols; ++c) {
        double s = 0.0;
        if (r >= c && r < rows)
            for (int p = q; p < c; p += 4) s += S[p * CLD + r] * S[p * CLD + c];
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        const double a = (r >= c && r < rows) ? S[c * CLD + r] - s : 0.0;
        if (r == c && q == 0) {
            if (!(a > 0.0)) {
                bad = 1;
                piv = 1.0;
            } else {
                piv = 1.0 / sqrt(a);
            }
        }
        __syncthreads();
        const double inv = piv;
        if (q == 0 && r < rows && r >= c) S[c * CLD + r] = (r == c) ? 1.0 / inv : a * inv;
        if (threadIdx.x == 0) rdiag_out[c] = inv;
        __syncthreads();
    }
    return bad == 0;
}

// X (rows x cols) <- X L^-T with L the factored diagonal tile (four threads per row)
__device__ void trsm_tile(double* X, const double* L, const double* rd, int rows, int cols)
{
    const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
    const bool act = r < rows;
    for (int c = 0; c < cols; ++c) {
        double s = 0.0;
        if (act)
            for (int p = q; p < c; p += 4) s += X[p * CLD + r] * L[p * CLD + c];
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (act && q == 0) X[c * CLD + r] = (X[c * CLD + r] - s) * rd[c];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(kCholThreads) k_chol(CholArgs A)
{
    extern __shared__ double smem[];
    double* S0 = smem;                  // CB x CLD
    double* S1 = smem + CB * CLD;       // CB x CLD
    double* rd = smem + 2 * CB * CLD;   // CB
    __shared__ int task_id, ok;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            task_id = atomicAdd(A.next, 1);
            ok = (*(volatile int*)A.err & 2) == 0;
        }
        __syncthreads();
        if (task_id >= A.ntasks || !ok) return;
        const int4 t = A.tasks[task_id];
        const int type = t.x, i = t.y, j = t.z, k = t.w;
        if (type == TASK_POTRF) {
            if (threadIdx.x == 0) ok = wait_flag(A.cnt + k * A.nt + k, k, A.err);
            __syncthreads();
            if (!ok) return;
            const int rows = tile_rows(A, k), cols = tile_cols(A, k);
            load_tile(A, k, k, rows, cols, S0);
            __syncthreads();
            const bool spd = potrf_tile(S0, rows, cols, rd);
            if (!spd && threadIdx.x == 0) atomicOr(A.err, 1);
            store_tile(A, k, k, rows, cols, S0);
            for (int c = threadIdx.x; c < cols; c += blockDim.x) __stcg(A.rdiag + k * CB + c, rd[c]);
            publish(A.fin + k * A.nt + k, 1);
        } else if (type == TASK_TRSM) {
            if (threadIdx.x == 0)
                ok = wait_flag(A.fin + k * A.nt + k, 1, A.err) && wait_flag(A.cnt + i * A.nt + k, k, A.err);
            __syncthreads();
            if (!ok) return;
            const int rows = tile_rows(A, i), cols = tile_cols(A, k);
            load_tile(A, k, k, tile_rows(A, k), cols, S1);
            load_tile(A, i, k, rows, cols, S0);
            for (int c = threadIdx.x; c < cols; c += blockDim.x) rd[c] = __ldcg(A.rdiag + k * CB + c);
            __syncthreads();
            trsm_tile(S0, S1, rd, rows, cols);
            __syncthreads();
            store_tile(A, i, k, rows, cols, S0);
            publish(A.fin + i * A.nt + k, 1);
        } else if (type == TASK_GEMM) {
            if (threadIdx.x == 0)
                ok = wait_flag(A.fin + i * A.nt + k, 1, A.err) && wait_flag(A.fin + j * A.nt + k, 1, A.err) &&
                     wait_flag(A.cnt + i * A.nt + j, k, A.err);
            __syncthreads();
            if (!ok) return;
            const int kc = tile_cols(A, k);
            const int rows = tile_rows(A, i), cols = tile_cols(A, j);
            load_tile(A, i, k, rows, kc, S0);                 // L_ik
            load_tile(A, j, k, tile_rows(A, j), kc, S1);      // L_jk
            __syncthreads();
            // C(rows x cols) -= L_ik L_jk^T; thread owns rows tr + 16a and columns tc + 16b
            const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
            double acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
            for (int p = 0; p < kc; ++p) {
                double av[4], bv[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) { av[a] = S0[p * CLD + tr + 16 * a]; bv[a] = S1[p * CLD + tc + 16 * a]; }
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
            }
            double* C = A.M + (size_t)(j * CB) * A.lda + i * CB;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int c = tc + 16 * b;
                if (c >= cols) continue;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const int r = tr + 16 * a;
                    if (r < rows) {
                        double* p = C + (size_t)c * A.lda + r;
                        __stcg(p, __ldcg(p) - acc[a][b]);
                    }
                }
            }
            publish(A.cnt + i * A.nt + j, k + 1);
        } else {   // TASK_BSOLVE: y_k = L_kk^-T (z_k - sum_{i>k} L_ik^T y_i)
            const int cols = tile_cols(A, k);
            const int kb = k * CB;
            double* part = S1;   // 4 x CB partial sums
            const int c = threadIdx.x & (CB - 1), q = threadIdx.x >> 6;
            double s = 0.0;
            for (int ti = A.nt - 1; ti > k; --ti) {
                if (tile_cols(A, ti) == 0) continue;   // only the augmented row
                if (threadIdx.x == 0) ok = wait_flag(A.ydone + ti, 1, A.err) && wait_flag(A.fin + ti * A.nt + k, 1, A.err);
                __syncthreads();
                if (!ok) return;
                const int r0 = ti * CB, r1 = min(A.n, r0 + CB);
                if (c < cols)
                    for (int r = r0 + q; r < r1; r += 4) s += __ldcg(A.M + (size_t)(kb + c) * A.lda + r) * __ldcg(A.y + r);
            }
            if (threadIdx.x == 0) ok = wait_flag(A.fin + (A.nt - 1) * A.nt + k, 1, A.err) && wait_flag(A.fin + k * A.nt + k, 1, A.err);
            part[q * CB + c] = s;
            __syncthreads();
            if (!ok) return;
            if (threadIdx.x < cols) {
                const int cc = threadIdx.x;
                // z_k sits in the augmented row n
                const double z = __ldcg(A.M + (size_t)(kb + cc) * A.lda + A.n);
                rd[cc] = z - (part[cc] + part[CB + cc] + part[2 * CB + cc] + part[3 * CB + cc]);
            }
            load_tile(A, k, k, tile_rows(A, k), cols, S0);
            __syncthreads();
            // back substitution inside the tile by warp 0
            if (threadIdx.x < 32) {
                const int lane = threadIdx.x;
                for (int cc = cols - 1; cc >= 0; --cc) {
                    double a = 0.0;
                    for (int p = cc + 1 + lane; p < cols; p += 32) a += S0[cc * CLD + p] * rd[p];
                    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
                    if (lane == 0) rd[cc] = (rd[cc] - a) / S0[cc * CLD + cc];
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int cc = threadIdx.x; cc < cols; cc += blockDim.x) __stcg(A.y + kb + cc, rd[cc]);
            publish(A.ydone + k, 1);
        }
    }
}

// host: task list in the order described above
inline std::vector<int4> chol_tasks(int n)
{
    const int nt = (n + 1 + CB - 1) / CB;
    const int ntp = (n + CB - 1) / CB;   // tiles with pivot columns
    std::vector<int4> T;
    auto add = [&](int ty, int i, int j, int k) { T.push_back(make_int4(ty, i, j, k)); };
    if (ntp == 0) return T;
    add(TASK_POTRF, 0, 0, 0);
    for (int i = 1; i < nt; ++i) add(TASK_TRSM, i, 0, 0);
    for (int k = 0; k + 1 < ntp; ++k) {
        for (int i = k + 1; i < nt; ++i) add(TASK_GEMM, i, k + 1, k);
        add(TASK_POTRF, k + 1, k + 1, k + 1);
        for (int i = k + 2; i < nt; ++i) add(TASK_TRSM, i, k + 1, k + 1);
        for (int j = k + 2; j < ntp; ++j)
            for (int i = j; i < nt; ++i) add(TASK_GEMM, i, j, k);
    }
    for (int k = ntp - 1; k >= 0; --k) add(TASK_BSOLVE, k, k, k);
    return T;
}

}  // namespace
