// EEQ charges (eeq_solver.cpp:3201-3700 of curcuma): A_ij = erf(r_ij/sqrt(a_i+a_j))/r_ij,
// A_ii = gam_i + sqrt(2/pi)/sqrt(a_i), x_i = chi_i + cnf_i sqrt(CN_i), one total-charge
// constraint per fragment.  The constraints are removed by the substitution q = q0 + B y,
// q0 = qfrag/n_f on the fragment's atoms and B the per-fragment difference basis
// (e_k - e_anchor, anchor = the fragment's first atom).  The reduced matrix
// M = B^T A B is SPD whenever A is on the constraint space and gives the same charges as
// curcuma's Schur-complement solve (:2087-2256) with one factorisation of size
// N - nfrag instead of N plus nfrag right-hand sides.  M is built element by element
// from the geometry (four A elements per entry), never from a stored A.
// Included inside namespace gfnff by engine.cu (one translation unit).
#pragma once

namespace {

// one element of A.  erf(r/sqrt(s)) == 1 in double once r^2 >= 36 s (erfc(6) < 2^-54).
__device__ __forceinline__ double eeq_a(const View& V, int a, int b)
{
    if (a == b) return V.adiag[a];
    const double4 pa = V.pos[a], pb = V.pos[b];
    const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double s = V.alpeeq[a] + V.alpeeq[b];
    if (d2 >= 36.0 * s) return rsqrt(d2);
    const double r = sqrt(d2);
    return erf(r / sqrt(s)) / r;
}

// reduced matrix, column-major with leading dimension lda: M[c*lda + r]; lower triangle
// only unless full.  Each thread keeps its row's atoms in registers and walks the
// columns blockIdx.y, blockIdx.y + gridDim.y, ...
__global__ void k_eeq_M(View V, const int* __restrict__ red2atom, const int* __restrict__ anchor, double* M,
                        int lda, int full)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= V.nred) return;
    const int k = red2atom[r], ak = anchor[k];
    for (int c = blockIdx.y; c < V.nred; c += gridDim.y) {
        if (!full && r < c) continue;
        const int l = red2atom[c], al = anchor[l];
        M[(size_t)c * lda + r] = eeq_a(V, k, l) - eeq_a(V, k, al) - eeq_a(V, ak, l) + eeq_a(V, ak, al);
    }
}

// x_i - sum_j A_ij q0_j over the atoms of charged fragments of i's molecule
__device__ __forceinline__ double eeq_rhs_atom(const View& V, int i, const int* qlist, int nq, const double* q0)
{
    double x = V.chi_base[i] + V.cnf[i] * sqrt(V.cn[i]);
    const int m = V.mol[i];
    for (int p = 0; p < nq; ++p) {
        const int j = qlist[p];
        if (V.mol[j] == m) x -= eeq_a(V, i, j) * q0[j];
    }
    return x;
}

// reduced right-hand side b = B^T (x - A q0); also written with stride lda to aug (the
// augmented row of the matrix) when aug is non-null
__global__ void k_eeq_rhs(View V, const int* __restrict__ red2atom, const int* __restrict__ anchor,
                          const int* __restrict__ qlist, int nq, const double* __restrict__ q0, double* b,
                          double* aug, int lda)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= V.nred) return;
    const int k = red2atom[r];
    const double v = eeq_rhs_atom(V, k, qlist, nq, q0) - eeq_rhs_atom(V, anchor[k], qlist, nq, q0);
    b[r] = v;
    if (aug) aug[(size_t)r * lda] = v;
}

// status of the persistent Cholesky: info = 1 not positive definite, 2 a wait gave up
__global__ void k_chol_info(const int* err, int* info)
{
    const int e = *err;
    *info = (e & 2) ? 2 : ((e & 1) ? 1 : 0);
}

// q = q0 + B y
__global__ void k_eeq_expand(View V, const double* q0, const int* atom2red, const int* frag_off,
                             const int* frag_atoms, const double* y)
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
            const int ra = atom2red[frag_atoms[p]];
            if (ra >= 0) s += y[ra];
        }
        V.q[i] = q0[i] - s;
    }
}

// ------------------------------------------------------------------------------------
// Batched block-diagonal EEQ: one block per molecule builds its reduced matrix (column-
// major lower triangle at M + moff[m]), factors it (right-looking Cholesky) and solves
// for y in place of b.  info[m] = 1 when the molecule's matrix is not positive definite.
// ------------------------------------------------------------------------------------
struct EEQBatch {
    const int* roff;        // nmol+1 reduced-index offsets
    const long long* moff;  // nmol matrix offsets (doubles)
    const int* red2atom;
    const int* anchor;
    const int* qlist;
    int nq;
    const double* q0;
    double* M;
    double* b;
    int* info;
};

__global__ void __launch_bounds__(256) k_eeq_batch(View V, EEQBatch P)
{
    const int m = blockIdx.x;
    const int r0 = P.roff[m], nr = P.roff[m + 1] - r0;
    double* M = P.M + P.moff[m];
    double* b = P.b + r0;
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    __shared__ double inv;
    __shared__ int bad;
    if (tid == 0) bad = 0;
    // build
    for (long long e = tid; e < (long long)nr * nr; e += nt) {
        const int c = (int)(e / nr), r = (int)(e % nr);
        if (r < c) continue;
        const int k = P.red2atom[r0 + r], l = P.red2atom[r0 + c];
        const int ak = P.anchor[k], al = P.anchor[l];
        M[(size_t)c * nr + r] = eeq_a(V, k, l) - eeq_a(V, k, al) - eeq_a(V, ak, l) + eeq_a(V, ak, al);
    }
    for (int r = tid; r < nr; r += nt) {
        const int k = P.red2atom[r0 + r];
        b[r] = eeq_rhs_atom(V, k, P.qlist, P.nq, P.q0) - eeq_rhs_atom(V, P.anchor[k], P.qlist, P.nq, P.q0);
    }
    __syncthreads();
    // factor: column k of L below the diagonal lives at M[k*nr + r], r > k
    for (int k = 0; k < nr; ++k) {
        if (tid == 0) {
            const double d = M[(size_t)k * nr + k];
            if (!(d > 0.0)) {
                bad = 1;
            } else {
                const double L = sqrt(d);
                M[(size_t)k * nr + k] = L;
                inv = 1.0 / L;
            }
        }
        __syncthreads();
        if (bad) break;
        for (int r = k + 1 + tid; r < nr; r += nt) M[(size_t)k * nr + r] *= inv;
        __syncthreads();
        for (int c = k + 1 + warp; c < nr; c += nw) {
            const double lc = M[(size_t)k * nr + c];
            for (int r = c + lane; r < nr; r += 32) M[(size_t)c * nr + r] -= M[(size_t)k * nr + r] * lc;
        }
        __syncthreads();
    }
    if (bad) {
        if (tid == 0) P.info[m] = 1;
        return;
    }
    // L z = b (column sweep), then L^T y = z (row sweep over the columns of L)
    for (int k = 0; k < nr; ++k) {
        if (tid == 0) b[k] /= M[(size_t)k * nr + k];
        __syncthreads();
        const double zk = b[k];
        for (int r = k + 1 + tid; r < nr; r += nt) b[r] -= M[(size_t)k * nr + r] * zk;
        __syncthreads();
    }
    for (int k = nr - 1; k >= 0; --k) {
        if (warp == 0) {
            double s = 0.0;
            for (int r = k + 1 + lane; r < nr; r += 32) s += M[(size_t)k * nr + r] * b[r];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) b[k] = (b[k] - s) / M[(size_t)k * nr + k];
        }
        __syncthreads();
    }
    if (tid == 0) P.info[m] = 0;
}

}  // namespace
