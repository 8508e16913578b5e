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
// Born (P16) element keps / (r + ab (ab / (ab + zeta r / 16))^16), ab = sqrt(brad_a brad_b)
__device__ __forceinline__ double born_p16(double keps, double r, double ba, double bb)
{
    const double ab = sqrt(ba * bb);
    double t = ab / (ab + gfnff::alpb::kZetaP16o16 * r);
    t *= t;
    t *= t;
    t *= t;
    t *= t;
    return keps / (r + ab * t);
}

__device__ __forceinline__ double eeq_a(const View& V, int a, int b)
{
    if (a == b) return V.adiag[a] + (V.brad ? V.bdiag[a] : 0.0);
    const double4 pa = V.pos[a], pb = V.pos[b];
    const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double s = V.alpeeq[a] + V.alpeeq[b];
    const double r = sqrt(d2);
    const double born = V.brad ? born_p16(V.keps, r, V.brad[a], V.brad[b]) : 0.0;
    if (d2 >= 36.0 * s) return rsqrt(d2) + born;
    return erf(r / sqrt(s)) / r + born;
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

// Reduced matrix by 32 x 32 tiles of the lower triangle (block (tr, tc), tr >= tc): the
// tile's row and column atoms (and their anchors) are staged in shared memory, every
// entry is computed once and written to (r, c) and, when full, to (c, r) through a
// shared-memory transpose so that both writes are coalesced.
constexpr int kMT = 32;
// BORN: the ALPB Born matrix enters (V.brad, V.bdiag); the gas-phase instantiation has none of
// its code
template <class TM, bool BORN = false>   // storage type of M: double, or float for the FP32-stored PCG matrix
__global__ void __launch_bounds__(256) k_eeq_M_tiles(View V, const int* __restrict__ red2atom,
                                                    const int* __restrict__ anchor, TM* M, int lda, int full,
                                                    float* M32 = nullptr)   // optional FP32 copy (k_pcg_ir)
{
    __shared__ double px[4][kMT], py[4][kMT], pz[4][kMT], pa[4][kMT];   // rows k, rows ak, cols l, cols al
    __shared__ double pbr[4][BORN ? kMT : 1];                            // Born radii (solvation)
    __shared__ int pid[4][kMT];
    __shared__ double T[kMT][kMT + 1];
    // triangular block index -> (tr, tc)
    const long long b = blockIdx.x;
    int tr = (int)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((long long)(tr + 1) * (tr + 2) / 2 <= b) ++tr;
    while ((long long)tr * (tr + 1) / 2 > b) --tr;
    const int tc = (int)(b - (long long)tr * (tr + 1) / 2);
    const int r0 = tr * kMT, c0 = tc * kMT, n = V.nred;
    if (threadIdx.x < 4 * kMT) {
        const int w = threadIdx.x / kMT, t = threadIdx.x % kMT;
        const int idx = (w < 2 ? r0 : c0) + t;
        int a = -1;
        if (idx < n) {
            const int k = red2atom[idx];
            a = (w & 1) ? anchor[k] : k;
        }
        pid[w][t] = a;
        if (a >= 0) {
            const double4 p = V.pos[a];
            px[w][t] = p.x; py[w][t] = p.y; pz[w][t] = p.z; pa[w][t] = V.alpeeq[a];
            if constexpr (BORN) pbr[w][t] = V.brad[a];
        }
    }
    __syncthreads();
    auto el = [&](int wa, int ia, int wb, int ib) {
        if (pid[wa][ia] == pid[wb][ib]) {
            if constexpr (BORN) return V.adiag[pid[wa][ia]] + V.bdiag[pid[wa][ia]];
            else return V.adiag[pid[wa][ia]];
        }
        const double dx = px[wa][ia] - px[wb][ib], dy = py[wa][ia] - py[wb][ib], dz = pz[wa][ia] - pz[wb][ib];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double s = pa[wa][ia] + pa[wb][ib];
        if constexpr (!BORN) {
            if (d2 >= 36.0 * s) return rsqrt(d2);
            const double r = sqrt(d2);
            return erf(r / sqrt(s)) / r;
        } else {
            const double born = born_p16(V.keps, sqrt(d2), pbr[wa][ia], pbr[wb][ib]);
            if (d2 >= 36.0 * s) return rsqrt(d2) + born;
            const double r = sqrt(d2);
            return erf(r / sqrt(s)) / r + born;
        }
    };
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    for (int cc = ty; cc < kMT; cc += 8) {
        const int r = r0 + tx, c = c0 + cc;
        double v = 0.0;
        if (r < n && c < n) v = el(0, tx, 2, cc) - el(0, tx, 3, cc) - el(1, tx, 2, cc) + el(1, tx, 3, cc);
        T[cc][tx] = v;
        if (r < n && c < n && (full || r >= c)) {
            M[(size_t)c * lda + r] = (TM)v;
            if (M32) M32[(size_t)c * lda + r] = (float)v;
        }
    }
    if (!full || tr == tc) return;
    __syncthreads();
    for (int rr = ty; rr < kMT; rr += 8) {   // (c, r) entries: row c0 + tx of column r0 + rr
        const int r = r0 + rr, c = c0 + tx;
        if (r < n && c < n) {
            M[(size_t)r * lda + c] = (TM)T[tx][rr];
            if (M32) M32[(size_t)r * lda + c] = (float)T[tx][rr];
        }
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

// info = max(info, other) (status of a second solve in the same evaluation)
__global__ void k_merge_info(int* info, const int* other)
{
    if (*other > *info) *info = *other;
}

// status of the persistent Cholesky: info = 1 not positive definite, 2 a wait gave up
__global__ void k_chol_info(const int* err, int* info)
{
    const int e = *err;
    *info = (e & 2) ? 2 : ((e & 1) ? 1 : 0);
}

// out = q0 + B y (q0 null: B y)
__global__ void k_eeq_expand(int nfrag, const double* q0, const int* atom2red, const int* frag_off,
                             const int* frag_atoms, const double* y, double* out)
{
    // one warp per fragment; frag_atoms[frag_off[f]] is the fragment's anchor (its first atom)
    const int f = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (f >= nfrag) return;   // whole warps
    const int p0 = frag_off[f], p1 = frag_off[f + 1];
    double s = 0.0;
    for (int p = p0 + 1 + lane; p < p1; p += 32) {
        const int a = frag_atoms[p];
        const double v = y[atom2red[a]];
        out[a] = (q0 ? q0[a] : 0.0) + v;
        s += v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        // anchor: minus the sum of its fragment's reduced variables
        const int a = frag_atoms[p0];
        out[a] = (q0 ? q0[a] : 0.0) - s;
    }
}

// rhs of the charge-response solve, B^T w with w_i = -cfar_i
__global__ void k_resp_rhs(View V, const int* __restrict__ red2atom, const int* __restrict__ anchor, double* b)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= V.nred) return;
    const int k = red2atom[r];
    b[r] = V.cfar[anchor[k]] - V.cfar[k];
}

// ------------------------------------------------------------------------------------
// Batched block-diagonal EEQ.  One block per SM takes molecules from a work queue
// (largest first, so the long factorisations start early) and solves each molecule's
// reduced system on its own:
//   * the matrix with the right-hand side appended as row nr is built from the geometry
//     straight into shared memory, packed by columns (column c holds rows c..nr), so
//     factoring it also yields z = L^-1 b in row nr;
//   * right-looking Cholesky with two block barriers per column: every thread computes
//     the pivot 1/sqrt(a_kk) itself, scales its share of column k, then the trailing
//     triangle is updated;
//   * back substitution L^T y = z by one warp.
// Molecules too large for shared memory use the same steps on a global-memory copy
// (column-major, lda = nr + 1).  info[m] = 1 when a pivot is not positive.
// ------------------------------------------------------------------------------------
struct EEQBatch {
    const int* roff;        // nmol+1 reduced-index offsets
    const long long* moff;  // nmol offsets of the global-memory copies (doubles)
    const int* order;       // molecules by decreasing size
    const int4* items;      // work items {first position in order, count, warp mode, 0}
    int nitems;
    int* next;              // work counter (zeroed before the launch)
    int smem_max;           // largest nr that fits the shared-memory path
    const int* red2atom;
    const int* anchor;
    const int* qlist;
    int nq;
    const double* q0;
    double* M;              // global copies for the large molecules
    double* y;              // solution (reduced index space)
    int* info;
    // mixed form: molecules with kWarpMaxRed < nr <= kTcMaxRed take the tensor-core
    // factorisation with FP64 refinement (k_eeq_tc.cuh); 0 in the FP64 form
    int tc;
    double* M64;            // FP64 lower tiles of those molecules
    const long long* m64off;
    double tol;             // refinement target ||b - M y||_inf
    int* refine;            // largest number of refinement corrections of the launch
};

__device__ void tc_solve(const View& V, const EEQBatch& P, int m, double* S);
constexpr int kTcMaxRedFwd = 304;   // kTcMaxRed of k_eeq_tc.cuh

// one molecule's atoms staged in shared memory: positions, alpha, EEQ diagonal, the
// reduced index maps (local atom indices) and the rhs row.  For a molecule of one
// fragment every reduced row has the same anchor a, and va[r] = A(k_r, a) is staged too,
// so that an entry of M costs one EEQ element instead of four (same value bit for bit:
// A is evaluated symmetrically and the terms are combined in the same order).
struct MolStage {
    double *x, *y, *z, *al, *ad, *rhs, *va;
    int *red, *anc;
    bool single;
};
constexpr int kStageAtoms = 320;                       // largest molecule of the batch path
constexpr int kStageDoubles = 7 * kStageAtoms;         // x y z al ad, rhs, va
constexpr int kStageInts = 2 * kStageAtoms;

__device__ __forceinline__ double eeq_a_s(const MolStage& M, int a, int b)
{
    if (a == b) return M.ad[a];
    const double dx = M.x[a] - M.x[b], dy = M.y[a] - M.y[b], dz = M.z[a] - M.z[b];
    const double d2 = dx * dx + dy * dy + dz * dz;
    const double s = M.al[a] + M.al[b];
    if (d2 >= 36.0 * s) return rsqrt(d2);
    const double r = sqrt(d2);
    return erf(r / sqrt(s)) / r;
}

// fills the staged arrays of M (x .. va, red, anc) for the molecule of reduced rows
// [r0, r0 + nr); `lane`/`nth` stride the work (block or warp), the caller synchronises
__device__ void fill_stage(const View& V, const EEQBatch& P, int r0, int nr, MolStage& M, int lane, int nth,
                           bool block)
{
    const int2 rg = V.jr[P.red2atom[r0]];
    for (int i = lane; i < rg.y - rg.x; i += nth) {
        const double4 p = V.pos[rg.x + i];
        M.x[i] = p.x; M.y[i] = p.y; M.z[i] = p.z;
        M.al[i] = V.alpeeq[rg.x + i];
        M.ad[i] = V.adiag[rg.x + i];
    }
    for (int r = lane; r < nr; r += nth) {
        const int k = P.red2atom[r0 + r], ak = P.anchor[k];
        M.red[r] = k - rg.x;
        M.anc[r] = ak - rg.x;
        M.rhs[r] = eeq_rhs_atom(V, k, P.qlist, P.nq, P.q0) - eeq_rhs_atom(V, ak, P.qlist, P.nq, P.q0);
    }
    M.single = P.anchor[P.red2atom[r0]] == P.anchor[P.red2atom[r0 + nr - 1]];
    if (block) __syncthreads(); else __syncwarp();
    if (M.single)
        for (int r = lane; r < nr; r += nth) M.va[r] = eeq_a_s(M, M.red[r], M.anc[r]);
}

__device__ MolStage stage_molecule(const View& V, const EEQBatch& P, int r0, int nr, double* base, int* ibase)
{
    MolStage M{base, base + kStageAtoms, base + 2 * kStageAtoms, base + 3 * kStageAtoms, base + 4 * kStageAtoms,
               base + 5 * kStageAtoms, base + 6 * kStageAtoms, ibase, ibase + kStageAtoms, false};
    fill_stage(V, P, r0, nr, M, threadIdx.x, blockDim.x, true);
    __syncthreads();
    return M;
}

// element (r, c) of [[M, .], [b^T, .]]; r == nr is the rhs row
__device__ __forceinline__ double eeq_aug(const MolStage& M, int nr, int r, int c)
{
    if (r == nr) return M.rhs[c];
    const int k = M.red[r], l = M.red[c];
    if (M.single) return ((eeq_a_s(M, k, l) - M.va[r]) - M.va[c]) + M.ad[M.anc[r]];
    const int ak = M.anc[r], al = M.anc[c];
    return eeq_a_s(M, k, l) - eeq_a_s(M, k, al) - eeq_a_s(M, ak, l) + eeq_a_s(M, ak, al);
}

// Rank-(k1 - k0) update of the trailing columns [k1, ccap) (rows c..nr) with the factored
// panel columns [k0, k1): a warp owns 4 columns x 32*RPL rows, each lane RPL rows x 4
// columns in registers; rows are read conflict-free along the packed columns, the column
// values as shared-memory broadcasts.
template <int RPL, class Off>
__device__ void chol_trailing(double* S, int nr, int ccap, int k0, int k1, Off co)
{
    constexpr int RB = 32 * RPL;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int m = ccap - k1;
    const int ncg = (m + 3) >> 2, nrb = (nr + 1 - k1 + RB - 1) / RB;
    for (int task = warp; task < ncg * nrb; task += nw) {
        const int cg = task / nrb, rb = task % nrb;
        const int c0 = k1 + 4 * cg, rbase = k1 + RB * rb;
        if (rbase + RB - 1 < c0) continue;
        double acc[RPL][4];
#pragma unroll
        for (int i = 0; i < RPL; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 4
        for (int p = k0; p < k1; ++p) {
            const double* cp = S + co(p) - p;   // element (r, p) at cp[r]
            double lr[RPL], lc[4];
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
                const int r = rbase + lane + 32 * i;
                lr[i] = r <= nr ? cp[r] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) lc[j] = c0 + j < ccap ? cp[c0 + j] : 0.0;
#pragma unroll
            for (int i = 0; i < RPL; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(lr[i], lc[j], acc[i][j]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = c0 + j;
            if (c >= ccap) break;
            double* cc = S + co(c) - c;
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
                const int r = rbase + lane + 32 * i;
                if (r >= c && r <= nr) cc[r] -= acc[i][j];
            }
        }
    }
}

// Blocked right-looking Cholesky of the first ccap columns of an augmented matrix with
// nr + 1 rows whose column c starts at S + co(c) (element (r, c) at S[co(c) + r - c]);
// updates reach columns < ccap only.  Per panel of kCholNB columns: warp 0 factors the
// panel's diagonal block in registers (lane i holds its row, pivots broadcast by
// shuffles) and leaves it with the inverse pivots in shared memory; after one barrier
// every thread solves its own rows of the panel against it (forward substitution along
// the row, no further barrier); after a second barrier the trailing columns take the
// panel's rank-kCholNB update (chol_trailing).  Returns false (uniformly) when a pivot
// is not positive.
constexpr int kCholNB = 8;
template <class Off>
__device__ bool chol_factor(double* S, int nr, int ccap, Off co)
{
    __shared__ double sL[kCholNB][kCholNB];   // diagonal block: L(i, j) for j < i, 1/L(j, j) at [j][j]
    __shared__ int sbad;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31;
    for (int k0 = 0; k0 < ccap; k0 += kCholNB) {
        const int kb = min(kCholNB, ccap - k0), k1 = k0 + kb;
        if (tid < 32) {
            double a[kCholNB];
#pragma unroll
            for (int j = 0; j < kCholNB; ++j)
                a[j] = (lane < kb && j <= lane) ? S[co(k0 + j) + lane - j] : 0.0;
            bool bad = false;
#pragma unroll
            for (int j = 0; j < kCholNB; ++j) {
                if (j >= kb) break;
                const double d = __shfl_sync(0xffffffffu, a[j], j);
                if (!(d > 0.0)) {
                    bad = true;
                    break;
                }
                const double is = rsqrt(d);   // 1/L(j, j); L(j, j) = d / sqrt(d)
                if (lane == j) a[j] = d * is;
                else if (lane > j) a[j] *= is;
                if (lane == j) sL[j][j] = is;
#pragma unroll
                for (int p = j + 1; p < kCholNB; ++p) {
                    const double lpj = __shfl_sync(0xffffffffu, a[j], p < kb ? p : 0);
                    if (p < kb && lane >= p) a[p] -= a[j] * lpj;
                }
            }
            if (lane < kb) {
#pragma unroll
                for (int j = 0; j < kCholNB; ++j)
                    if (j <= lane) {
                        S[co(k0 + j) + lane - j] = a[j];
                        if (j < lane) sL[lane][j] = a[j];
                    }
            }
            if (lane == 0) sbad = bad ? 1 : 0;
        }
        __syncthreads();
        if (sbad) return false;   // uniform: read after the barrier by every thread
        for (int r = k1 + tid; r <= nr; r += nt) {
            double v[kCholNB];
#pragma unroll
            for (int j = 0; j < kCholNB; ++j) v[j] = j < kb ? S[co(k0 + j) + r - k0 - j] : 0.0;
#pragma unroll
            for (int j = 0; j < kCholNB; ++j) {
                if (j >= kb) break;
                double x = v[j];
#pragma unroll
                for (int p = 0; p < j; ++p) x -= v[p] * sL[j][p];
                v[j] = x * sL[j][j];
            }
#pragma unroll
            for (int j = 0; j < kCholNB; ++j)
                if (j < kb) S[co(k0 + j) + r - k0 - j] = v[j];
        }
        __syncthreads();
        if (k1 >= ccap) continue;
        if (nr + 1 - k1 <= 96) chol_trailing<2>(S, nr, ccap, k0, k1, co);
        else chol_trailing<4>(S, nr, ccap, k0, k1, co);
        __syncthreads();
    }
    return true;
}

// L^T y = z for a factored augmented matrix (z_k = element (nr, k)), by 32-row blocks
// from the bottom: warp 0 solves the diagonal block (lane l holds row kb + l, each y_j
// broadcast with a shuffle), then every thread takes one row above the block and
// subtracts the block's contribution, a dot product along its packed column.
template <class Off>
__device__ void chol_back_subst(const double* S, int nr, Off co, double* y)
{
    for (int k = threadIdx.x; k < nr; k += blockDim.x) y[k] = S[co(k) + nr - k];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int kb = ((nr - 1) >> 5) << 5; kb >= 0; kb -= 32) {
        const int ke = min(kb + 32, nr);
        if (warp == 0) {
            const int r = kb + lane;
            double z = r < ke ? y[r] : 0.0;
            const double dinv = r < ke ? 1.0 / S[co(r)] : 0.0;
            double yr = 0.0;
            for (int j = ke - 1; j >= kb; --j) {
                const double yj = __shfl_sync(0xffffffffu, z * dinv, j - kb);
                if (r == j) yr = yj;
                if (r < j) z -= S[co(r) + j - r] * yj;   // L(j, r)
            }
            if (r < ke) y[r] = yr;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < kb; r += blockDim.x) {
            const double* cr = S + co(r) - r;   // element (j, r) at cr[j]
            double a = 0.0;
            for (int j = kb; j < ke; ++j) a += cr[j] * y[j];
            y[r] -= a;
        }
        __syncthreads();
    }
}

// Cholesky + back substitution L^T y = z of the augmented matrix (z_k = element (nr, k));
// y receives the solution.  Returns false when a pivot is not positive.
template <class Off>
__device__ bool chol_aug_solve(double* S, int nr, Off co, double* y, double* lk)
{
    (void)lk;
    const bool ok = chol_factor(S, nr, nr, co);
    __syncthreads();
    if (!ok) return false;
    chol_back_subst(S, nr, co, y);
    return true;
}

struct PackedCols {   // column c of an (nr+1) x nr packed lower matrix
    int n1;           // nr + 1
    __device__ __forceinline__ long long operator()(int c) const { return (long long)c * n1 - (long long)c * (c - 1) / 2; }
};
struct DenseCols {    // column c of a column-major matrix with leading dimension lda, from row c
    int lda;
    __device__ __forceinline__ long long operator()(int c) const { return (long long)c * lda + c; }
};

// Molecules beyond the shared-memory path, in two stages (s = nr - smem_max):
//  1. the first s columns (all rows and the rhs row) are built and factored in shared
//     memory (packed by columns) and copied to the molecule's global scratch G
//     (column-major, lda = nr + 1);
//  2. the trailing block, A22 - L21 L21^T with its rhs row, is written to G, read back
//     into shared memory, factored and back-substituted (y for rows s..nr-1);
//  3. y for rows 0..s-1: w = z1 - L21^T y2 (parallel), then L11^T y1 = w by one warp.
__device__ bool chol_two_stage(const EEQBatch& P, const MolStage& MS, int m, int nr, double* S, double* y)
{
    const int s = nr - P.smem_max;
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    double* G = P.M + P.moff[m];
    const int lda = nr + 1;
    // ---- stage 1: panel columns [0, s), rows c..nr, packed
    const PackedCols po{nr + 1};
    for (int c = warp; c < s; c += nw)
        for (int r = c + lane; r <= nr; r += 32) S[po(c) + r - c] = eeq_aug(MS, nr, r, c);
    __syncthreads();
    const bool ok1 = chol_factor(S, nr, s, po);
    __syncthreads();
    if (!ok1) return false;
    for (int c = warp; c < s; c += nw)   // a warp per column keeps many loads/stores in flight
        for (int r = c + lane; r <= nr; r += 32) G[(size_t)c * lda + r] = S[po(c) + r - c];
    // ---- stage 2: trailing block A22 - L21 L21^T (rows c..nr of columns c >= s) into G:
    // a warp owns 4 columns x 128 rows, the rank-s product in registers (as chol_trailing)
    {
        const int m2 = nr - s;
        const int ncg = (m2 + 3) >> 2, nrb = (nr + 1 - s + 127) >> 7;
        for (int task = warp; task < ncg * nrb; task += nw) {
            const int cg = task / nrb, rb = task % nrb;
            const int c0 = s + 4 * cg, rbase = s + 128 * rb;
            if (rbase + 127 < c0) continue;
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
#pragma unroll 4
            for (int p = 0; p < s; ++p) {
                const double* cp = S + po(p) - p;
                double lr[4], lc[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = rbase + lane + 32 * i;
                    lr[i] = r <= nr ? cp[r] : 0.0;
                }
#pragma unroll
                for (int j = 0; j < 4; ++j) lc[j] = c0 + j < nr ? cp[c0 + j] : 0.0;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(lr[i], lc[j], acc[i][j]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j;
                if (c >= nr) break;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = rbase + lane + 32 * i;
                    if (r >= c && r <= nr) G[(size_t)c * lda + r] = eeq_aug(MS, nr, r, c) - acc[i][j];
                }
            }
        }
    }
    __syncthreads();
    const int mt = nr - s;
    const PackedCols co{mt + 1};
    for (int c = warp; c < mt; c += nw)
        for (int r = c + lane; r <= mt; r += 32) S[co(c) + r - c] = G[(size_t)(s + c) * lda + s + r];
    __syncthreads();
    double* lk = S + co(mt);
    double* ys = lk + mt + 1;
    if (!chol_aug_solve(S, mt, co, ys, lk)) return false;
    for (int k = tid; k < mt; k += nt) y[s + k] = ys[k];
    // ---- stage 3: w_k = z_k - sum_{r >= s} L_rk y_r, then L11^T y1 = w with L11 and w
    // copied back into shared memory as a packed (s + 1) x s augmented matrix
    const PackedCols c1{s + 1};
    double* yt = S + c1(s);             // copy of y[s..nr) behind the packed L11
    double* y1 = yt + mt;
    for (int k = tid; k < mt; k += nt) yt[k] = ys[k];
    __syncthreads();
    for (int c = warp; c < s; c += nw)
        for (int r = c + lane; r < s; r += 32) S[c1(c) + r - c] = G[(size_t)c * lda + r];
    for (int k = warp; k < s; k += nw) {
        double a = 0.0;
        for (int r = s + lane; r < nr; r += 32) a += G[(size_t)k * lda + r] * yt[r - s];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) S[c1(k) + s - k] = G[(size_t)k * lda + nr] - a;
    }
    __syncthreads();
    chol_back_subst(S, s, c1, y1);
    for (int k = tid; k < s; k += nt) y[k] = y1[k];
    return true;
}

// ---- small molecules: one warp each, __syncwarp only --------------------------------
constexpr int kWarpMols = 8;          // molecules per warp-mode work item
constexpr int kWarpMaxRed = 70;       // largest reduced system of the warp path
constexpr int kWarpAtoms = kWarpMaxRed + 1;
constexpr int kWarpRegion = 8 * kWarpAtoms + kWarpMaxRed * (kWarpMaxRed + 3) / 2 + 2 * kWarpMaxRed + 2;

__device__ void warp_solve(const View& V, const EEQBatch& P, int m, double* R)
{
    const int lane = threadIdx.x & 31;
    const int r0 = P.roff[m], nr = P.roff[m + 1] - r0;
    if (nr == 0) {
        if (lane == 0) P.info[m] = 0;
        return;
    }
    MolStage M{R, R + kWarpAtoms, R + 2 * kWarpAtoms, R + 3 * kWarpAtoms, R + 4 * kWarpAtoms, R + 5 * kWarpAtoms,
               R + 6 * kWarpAtoms, reinterpret_cast<int*>(R + 7 * kWarpAtoms),
               reinterpret_cast<int*>(R + 7 * kWarpAtoms) + kWarpAtoms, false};
    fill_stage(V, P, r0, nr, M, lane, 32, false);
    __syncwarp();
    double* S = R + 8 * kWarpAtoms;
    const PackedCols co{nr + 1};
    double* lk = S + co(nr);
    double* ys = lk + nr + 1;
    for (int c = 0; c < nr; ++c)
        for (int r = c + lane; r <= nr; r += 32) S[co(c) + r - c] = eeq_aug(M, nr, r, c);
    __syncwarp();
    bool ok = true;
    for (int k = 0; k < nr; ++k) {
        const double d = S[co(k)];
        if (!(d > 0.0)) {
            ok = false;
            break;
        }
        const double inv = 1.0 / sqrt(d);
        double* ck = S + co(k);
        for (int r = k + 1 + lane; r <= nr; r += 32) {
            const double v = ck[r - k] * inv;
            ck[r - k] = v;
            lk[r] = v;
        }
        __syncwarp();
        if (lane == 0) ck[0] = d * inv;
        for (int c = k + 1; c < nr; ++c) {
            const double lc = lk[c];
            double* cc = S + co(c);
            for (int r = c + lane; r <= nr; r += 32) cc[r - c] -= lk[r] * lc;
        }
        __syncwarp();
    }
    if (ok) {
        for (int k = nr - 1; k >= 0; --k) {
            const double* ck = S + co(k);
            double sum = 0.0;
            for (int r = k + 1 + lane; r < nr; r += 32) sum += ck[r - k] * ys[r];
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) ys[k] = (ck[nr - k] - sum) / ck[0];
            __syncwarp();
        }
        for (int k = lane; k < nr; k += 32) P.y[r0 + k] = ys[k];
    }
    if (lane == 0) P.info[m] = ok ? 0 : 1;
    __syncwarp();
}

__global__ void __launch_bounds__(512) k_eeq_batch(View V, EEQBatch P)
{
    extern __shared__ __align__(16) double S[];
    __shared__ int4 item;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int w = atomicAdd(P.next, 1);
            item = w < P.nitems ? P.items[w] : make_int4(-1, 0, 0, 0);
        }
        __syncthreads();
        const int4 it = item;
        if (it.x < 0) return;
        if (it.z) {   // warp mode: warp w solves molecule order[first + w]
            const int w = threadIdx.x >> 5;
            if (w < it.y) warp_solve(V, P, P.order[it.x + w], S + (size_t)w * kWarpRegion);
            continue;
        }
        const int m = P.order[it.x];
        const int r0 = P.roff[m], nr = P.roff[m + 1] - r0;
        double* y = P.y + r0;
        if (nr == 0) {
            if (threadIdx.x == 0) P.info[m] = 0;
            continue;
        }
        if (P.tc && nr <= kTcMaxRedFwd) {
            tc_solve(V, P, m, S);
            continue;
        }
        bool ok;
        const MolStage MS = stage_molecule(V, P, r0, nr, S, reinterpret_cast<int*>(S + kStageDoubles));
        double* W = S + kStageDoubles + kStageInts / 2;   // matrix work area
        if (nr <= P.smem_max) {
            const PackedCols co{nr + 1};
            const long long tot = co(nr);   // all entries incl. the rhs row
            double* lk = W + tot;
            double* ys = lk + nr + 1;
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int c = warp; c < nr; c += nw)
                for (int r = c + lane; r <= nr; r += 32) W[co(c) + r - c] = eeq_aug(MS, nr, r, c);
            __syncthreads();
            ok = chol_aug_solve(W, nr, co, ys, lk);
            for (int k = threadIdx.x; k < nr; k += blockDim.x) y[k] = ys[k];
        } else {
            ok = chol_two_stage(P, MS, m, nr, W, y);
        }
        if (threadIdx.x == 0) P.info[m] = ok ? 0 : 1;
    }
}

}  // namespace
