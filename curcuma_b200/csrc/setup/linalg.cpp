#include "linalg.h"

#include <algorithm>
#include <cmath>
#include <utility>

namespace gfnff {
namespace linalg {

bool cholesky(double* A, int n)
{
    const int nb = 64;
    for (int k0 = 0; k0 < n; k0 += nb) {
        const int k1 = std::min(n, k0 + nb);
        // factor the diagonal panel (unblocked, left-looking inside the panel)
        for (int j = k0; j < k1; ++j) {
            double d = A[(size_t)j * n + j];
            for (int p = k0; p < j; ++p) d -= A[(size_t)j * n + p] * A[(size_t)j * n + p];
            if (!(d > 0.0)) return false;
            d = std::sqrt(d);
            A[(size_t)j * n + j] = d;
            const double inv = 1.0 / d;
            for (int i = j + 1; i < k1; ++i) {
                double s = A[(size_t)i * n + j];
                for (int p = k0; p < j; ++p) s -= A[(size_t)i * n + p] * A[(size_t)j * n + p];
                A[(size_t)i * n + j] = s * inv;
            }
        }
        // triangular solve for the panel below the diagonal block
#pragma omp parallel for schedule(static)
        for (int i = k1; i < n; ++i) {
            double* ri = A + (size_t)i * n;
            for (int j = k0; j < k1; ++j) {
                const double* rj = A + (size_t)j * n;
                double s = ri[j];
                for (int p = k0; p < j; ++p) s -= ri[p] * rj[p];
                ri[j] = s / rj[j];
            }
        }
        // trailing update of the lower triangle: A22 -= L21 L21^T
#pragma omp parallel for schedule(dynamic, 8)
        for (int i = k1; i < n; ++i) {
            double* ri = A + (size_t)i * n;
            for (int j = k1; j <= i; ++j) {
                const double* rj = A + (size_t)j * n;
                double s = 0.0;
                for (int p = k0; p < k1; ++p) s += ri[p] * rj[p];
                ri[j] -= s;
            }
        }
    }
    return true;
}

namespace {

// forward and backward substitution for columns [c0, c0 + W) of B (row-major, nrhs columns):
// rows of B are updated as contiguous segments, L is read by rows
template <int W>
void solve_columns(const double* L, int n, double* B, int nrhs, int c0, int w)
{
    double acc[W];
    for (int i = 0; i < n; ++i) {   // L y = b
        const double* li = L + (size_t)i * n;
        for (int c = 0; c < W; ++c) acc[c] = 0.0;
        for (int p = 0; p < i; ++p) {
            const double l = li[p];
            const double* bp = B + (size_t)p * nrhs + c0;
            if (w == W) {
                for (int c = 0; c < W; ++c) acc[c] += l * bp[c];
            } else {
                for (int c = 0; c < w; ++c) acc[c] += l * bp[c];
            }
        }
        double* bi = B + (size_t)i * nrhs + c0;
        for (int c = 0; c < w; ++c) bi[c] = (bi[c] - acc[c]) / li[i];
    }
    for (int i = n - 1; i >= 0; --i) {   // L^T x = y, row i final once the rows below are done
        const double* li = L + (size_t)i * n;
        double* bi = B + (size_t)i * nrhs + c0;
        for (int c = 0; c < w; ++c) bi[c] /= li[i];
        for (int p = 0; p < i; ++p) {
            const double l = li[p];
            if (l == 0.0) continue;
            double* bp = B + (size_t)p * nrhs + c0;
            if (w == W) {
                for (int c = 0; c < W; ++c) bp[c] -= l * bi[c];
            } else {
                for (int c = 0; c < w; ++c) bp[c] -= l * bi[c];
            }
        }
    }
}

}  // namespace

void cholesky_solve(const double* L, int n, double* B, int nrhs)
{
    // blocks of 16 right-hand sides per thread (the EEQ solve has one per fragment)
    constexpr int W = 16;
    const int nb = (nrhs + W - 1) / W;
#pragma omp parallel for schedule(dynamic, 1) if (nb > 1)
    for (int k = 0; k < nb; ++k) {
        const int c0 = k * W;
        solve_columns<W>(L, n, B, nrhs, c0, std::min(W, nrhs - c0));
    }
}

// ---- cache-blocked kernels for large systems (the oracle's per-geometry EEQ) ------------
// C[MR x NR] -= sum_p Ap[p][i] Bp[p][j] over packed K x MR and K x NR panels: the
// register-blocked inner kernel of both the Cholesky trailing update and the blocked
// triangular solves (AVX2 + FMA, a baseline of every x86-64 Xeon this code runs on).
namespace {

constexpr int kMR = 8, kNR = 4;

__attribute__((target("avx2,fma"))) void micro_kernel(int K, const double* __restrict__ Ap,
                                                      const double* __restrict__ Bp, double* C, int ldc,
                                                      int mr, int nr)
{
    double acc[kNR][kMR] = {};
    for (int p = 0; p < K; ++p) {
        const double* a = Ap + (size_t)p * kMR;
        const double* b = Bp + (size_t)p * kNR;
#pragma GCC unroll 4
        for (int j = 0; j < kNR; ++j)
#pragma omp simd
            for (int i = 0; i < kMR; ++i) acc[j][i] += a[i] * b[j];
    }
    for (int i = 0; i < mr; ++i)
        for (int j = 0; j < nr; ++j) C[(size_t)i * ldc + j] -= acc[j][i];
}

// packs rows [r0, r0 + m) x columns [c0, c0 + K) of a row-major matrix (leading dimension
// ld) into tiles of `w` rows: tile t holds element (r0 + t*w + i, c0 + p) at [t][p][i]
void pack_rows(const double* M, int ld, int r0, int m, int c0, int K, int w, double* out)
{
    const int nt = (m + w - 1) / w;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nt; ++t) {
        double* o = out + (size_t)t * K * w;
        for (int p = 0; p < K; ++p)
            for (int i = 0; i < w; ++i) {
                const int r = t * w + i;
                o[(size_t)p * w + i] = r < m ? M[(size_t)(r0 + r) * ld + c0 + p] : 0.0;
            }
    }
}

// packs rows [r0, r0 + K) x columns [c0, c0 + nc) into tiles of `w` columns: tile u holds
// element (r0 + p, c0 + u*w + j) at [u][p][j]
void pack_cols(const double* M, int ld, int r0, int K, int c0, int nc, int w, double* out)
{
    const int nt = (nc + w - 1) / w;
#pragma omp parallel for schedule(static)
    for (int u = 0; u < nt; ++u) {
        double* o = out + (size_t)u * K * w;
        for (int p = 0; p < K; ++p)
            for (int j = 0; j < w; ++j) {
                const int c = u * w + j;
                o[(size_t)p * w + j] = c < nc ? M[(size_t)(r0 + p) * ld + c0 + c] : 0.0;
            }
    }
}

}  // namespace

bool cholesky_blocked(double* A, int n)
{
    const int nb = 128, NC = 512;
    std::vector<double> Ap, Bp;
    for (int k0 = 0; k0 < n; k0 += nb) {
        const int k1 = std::min(n, k0 + nb), K = k1 - k0;
        // diagonal block (left-looking inside the block)
        for (int j = k0; j < k1; ++j) {
            double d = A[(size_t)j * n + j];
            for (int p = k0; p < j; ++p) d -= A[(size_t)j * n + p] * A[(size_t)j * n + p];
            if (!(d > 0.0)) return false;
            d = std::sqrt(d);
            A[(size_t)j * n + j] = d;
            const double inv = 1.0 / d;
            for (int i = j + 1; i < k1; ++i) {
                double s = A[(size_t)i * n + j];
                for (int p = k0; p < j; ++p) s -= A[(size_t)i * n + p] * A[(size_t)j * n + p];
                A[(size_t)i * n + j] = s * inv;
            }
        }
        // panel below: L21 = A21 L11^-T, row by row
#pragma omp parallel for schedule(static)
        for (int i = k1; i < n; ++i) {
            double* ri = A + (size_t)i * n;
            for (int j = k0; j < k1; ++j) {
                const double* rj = A + (size_t)j * n;
                double s = ri[j];
                for (int p = k0; p < j; ++p) s -= ri[p] * rj[p];
                ri[j] = s / rj[j];
            }
        }
        const int m = n - k1;
        if (m <= 0) break;
        // trailing lower triangle A22 -= L21 L21^T from packed copies of L21
        Ap.resize((size_t)((m + kMR - 1) / kMR) * kMR * K);
        Bp.resize((size_t)((m + kNR - 1) / kNR) * kNR * K);
        pack_rows(A, n, k1, m, k0, K, kMR, Ap.data());
        // L21^T as K x m: element (p, c) = L21(c, p), i.e. rows of L21 packed by columns
        {
            const int ntu = (m + kNR - 1) / kNR;
#pragma omp parallel for schedule(static)
            for (int u = 0; u < ntu; ++u) {
                double* o = Bp.data() + (size_t)u * K * kNR;
                for (int p = 0; p < K; ++p)
                    for (int j = 0; j < kNR; ++j) {
                        const int c = u * kNR + j;
                        o[(size_t)p * kNR + j] = c < m ? A[(size_t)(k1 + c) * n + k0 + p] : 0.0;
                    }
            }
        }
        for (int jc = 0; jc < m; jc += NC) {
            const int jc1 = std::min(m, jc + NC);
            const int t0 = jc / kMR, nt = (m + kMR - 1) / kMR;
#pragma omp parallel for schedule(dynamic, 4)
            for (int t = t0; t < nt; ++t) {
                const int i0 = t * kMR, mr = std::min(kMR, m - i0);
                const double* a = Ap.data() + (size_t)t * K * kMR;
                for (int j0 = jc; j0 < jc1 && j0 <= i0 + mr - 1; j0 += kNR) {
                    const int nr = std::min(kNR, jc1 - j0);
                    micro_kernel(K, a, Bp.data() + (size_t)(j0 / kNR) * K * kNR, A + (size_t)(k1 + i0) * n + k1 + j0,
                                 n, mr, nr);
                }
            }
        }
    }
    return true;
}

void cholesky_solve_blocked(const double* L, int n, double* B, int nrhs)
{
    // L Y = B then L^T X = Y, both by row blocks of nb: the block's rows take the GEMM
    // update from every solved block (packed panels, micro-kernel), then the small triangular
    // solve with the diagonal block.  Parallel over row tiles of the GEMM and over the
    // right-hand sides of the triangular solve.
    const int nb = 128;
    std::vector<double> Ap, Bp;
    for (int i0 = 0; i0 < n; i0 += nb) {
        const int i1 = std::min(n, i0 + nb), mb = i1 - i0;
        if (i0 > 0) {   // B[I] -= L[I, 0:i0] Y[0:i0]  (K = i0 in chunks)
            for (int k0 = 0; k0 < i0; k0 += 256) {
                const int K = std::min(256, i0 - k0);
                Ap.resize((size_t)((mb + kMR - 1) / kMR) * kMR * K);
                Bp.resize((size_t)((nrhs + kNR - 1) / kNR) * kNR * K);
                pack_rows(L, n, i0, mb, k0, K, kMR, Ap.data());
                pack_cols(B, nrhs, k0, K, 0, nrhs, kNR, Bp.data());
                const int ntr = (mb + kMR - 1) / kMR, ntc = (nrhs + kNR - 1) / kNR;
#pragma omp parallel for collapse(2) schedule(static)
                for (int t = 0; t < ntr; ++t)
                    for (int u = 0; u < ntc; ++u)
                        micro_kernel(K, Ap.data() + (size_t)t * K * kMR, Bp.data() + (size_t)u * K * kNR,
                                     B + (size_t)(i0 + t * kMR) * nrhs + u * kNR, nrhs,
                                     std::min(kMR, mb - t * kMR), std::min(kNR, nrhs - u * kNR));
            }
        }
#pragma omp parallel for schedule(static)
        for (int c = 0; c < nrhs; ++c)
            for (int i = i0; i < i1; ++i) {
                const double* li = L + (size_t)i * n;
                double s = B[(size_t)i * nrhs + c];
                for (int p = i0; p < i; ++p) s -= li[p] * B[(size_t)p * nrhs + c];
                B[(size_t)i * nrhs + c] = s / li[i];
            }
    }
    for (int i1 = n; i1 > 0; i1 -= nb) {
        const int i0 = std::max(0, i1 - nb), mb = i1 - i0;
        if (i1 < n) {   // B[I] -= L[i1:n, I]^T X[i1:n]  (K = n - i1 in chunks)
            for (int k0 = i1; k0 < n; k0 += 256) {
                const int K = std::min(256, n - k0);
                // A operand: rows I of L^T = columns I of L, packed K x MR from L(k0 + p, i0 + i)
                Ap.resize((size_t)((mb + kMR - 1) / kMR) * kMR * K);
                {
                    const int nt = (mb + kMR - 1) / kMR;
#pragma omp parallel for schedule(static)
                    for (int t = 0; t < nt; ++t) {
                        double* o = Ap.data() + (size_t)t * K * kMR;
                        for (int p = 0; p < K; ++p)
                            for (int i = 0; i < kMR; ++i) {
                                const int r = t * kMR + i;
                                o[(size_t)p * kMR + i] = r < mb ? L[(size_t)(k0 + p) * n + i0 + r] : 0.0;
                            }
                    }
                }
                Bp.resize((size_t)((nrhs + kNR - 1) / kNR) * kNR * K);
                pack_cols(B, nrhs, k0, K, 0, nrhs, kNR, Bp.data());
                const int ntr = (mb + kMR - 1) / kMR, ntc = (nrhs + kNR - 1) / kNR;
#pragma omp parallel for collapse(2) schedule(static)
                for (int t = 0; t < ntr; ++t)
                    for (int u = 0; u < ntc; ++u)
                        micro_kernel(K, Ap.data() + (size_t)t * K * kMR, Bp.data() + (size_t)u * K * kNR,
                                     B + (size_t)(i0 + t * kMR) * nrhs + u * kNR, nrhs,
                                     std::min(kMR, mb - t * kMR), std::min(kNR, nrhs - u * kNR));
            }
        }
#pragma omp parallel for schedule(static)
        for (int c = 0; c < nrhs; ++c)
            for (int i = i1 - 1; i >= i0; --i) {
                double s = B[(size_t)i * nrhs + c];
                for (int p = i + 1; p < i1; ++p) s -= L[(size_t)p * n + i] * B[(size_t)p * nrhs + c];
                B[(size_t)i * nrhs + c] = s / L[(size_t)i * n + i];
            }
    }
}

bool lu_solve(double* A, int n, double* b)
{
    for (int k = 0; k < n; ++k) {
        int piv = k;
        double best = std::fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double v = std::fabs(A[(size_t)i * n + k]);
            if (v > best) { best = v; piv = i; }
        }
        if (best == 0.0) return false;
        if (piv != k) {
            for (int j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)piv * n + j]);
            std::swap(b[k], b[piv]);
        }
        const double inv = 1.0 / A[(size_t)k * n + k];
#pragma omp parallel for schedule(static) if (n - k > 256)
        for (int i = k + 1; i < n; ++i) {
            double f = A[(size_t)i * n + k] * inv;
            if (f == 0.0) continue;
            A[(size_t)i * n + k] = f;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
            b[i] -= f * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < n; ++j) s -= A[(size_t)i * n + j] * b[j];
        b[i] = s / A[(size_t)i * n + i];
    }
    return true;
}

bool eeq_schur_solve(double* A, int n, const double* x, const int* frag, int nfrag,
                     const double* qf, double* q, bool blocked)
{
    std::vector<double> Acopy;
    const bool keep = true;
    if (keep) Acopy.assign(A, A + (size_t)n * n);
    if (blocked ? cholesky_blocked(A, n) : cholesky(A, n)) {
        // right-hand sides: column 0 = x, columns 1..nfrag = C^T
        const int nr = 1 + nfrag;
        std::vector<double> B((size_t)n * nr, 0.0);
        for (int i = 0; i < n; ++i) {
            B[(size_t)i * nr] = x[i];
            B[(size_t)i * nr + 1 + frag[i]] = 1.0;
        }
        if (blocked) cholesky_solve_blocked(A, n, B.data(), nr);
        else cholesky_solve(A, n, B.data(), nr);
        // S = C Z2 (nfrag x nfrag), r = C z1 - qf
        std::vector<double> S((size_t)nfrag * nfrag, 0.0), r(nfrag, 0.0);
        for (int i = 0; i < n; ++i) {
            const int f = frag[i];
            r[f] += B[(size_t)i * nr];
            for (int g = 0; g < nfrag; ++g) S[(size_t)f * nfrag + g] += B[(size_t)i * nr + 1 + g];
        }
        for (int f = 0; f < nfrag; ++f) r[f] -= qf[f];
        std::vector<double> Sf = S;
        bool ok = cholesky(Sf.data(), nfrag);
        if (ok) {
            cholesky_solve(Sf.data(), nfrag, r.data(), 1);
        } else {
            ok = lu_solve(S.data(), nfrag, r.data());
        }
        if (ok) {
            for (int i = 0; i < n; ++i) {
                double s = B[(size_t)i * nr];
                for (int g = 0; g < nfrag; ++g) s -= B[(size_t)i * nr + 1 + g] * r[g];
                q[i] = s;
            }
            return true;
        }
    }
    // fallback: LU of the augmented (n + nfrag) system
    const int m = n + nfrag;
    std::vector<double> M((size_t)m * m, 0.0), rhs(m, 0.0);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) M[(size_t)i * m + j] = Acopy[(size_t)i * n + j];
        M[(size_t)i * m + n + frag[i]] = 1.0;
        M[(size_t)(n + frag[i]) * m + i] = 1.0;
        rhs[i] = x[i];
    }
    for (int f = 0; f < nfrag; ++f) rhs[n + f] = qf[f];
    if (!lu_solve(M.data(), m, rhs.data())) return false;
    for (int i = 0; i < n; ++i) q[i] = rhs[i];
    return true;
}

void sym_eig(const std::vector<double>& Ain, int n, std::vector<double>& eval,
             std::vector<double>& evec)
{
    std::vector<double> A = Ain;
    evec.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) evec[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n; ++p)
            for (int r = p + 1; r < n; ++r) off += A[(size_t)p * n + r] * A[(size_t)p * n + r];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p) {
            for (int r = p + 1; r < n; ++r) {
                const double apr = A[(size_t)p * n + r];
                if (std::fabs(apr) < 1e-300) continue;
                const double app = A[(size_t)p * n + p], arr = A[(size_t)r * n + r];
                const double theta = (arr - app) / (2.0 * apr);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                                 (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akr = A[(size_t)k * n + r];
                    A[(size_t)k * n + p] = c * akp - s * akr;
                    A[(size_t)k * n + r] = s * akp + c * akr;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], ark = A[(size_t)r * n + k];
                    A[(size_t)p * n + k] = c * apk - s * ark;
                    A[(size_t)r * n + k] = s * apk + c * ark;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = evec[(size_t)k * n + p], vkr = evec[(size_t)k * n + r];
                    evec[(size_t)k * n + p] = c * vkp - s * vkr;
                    evec[(size_t)k * n + r] = s * vkp + c * vkr;
                }
            }
        }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(),
              [&](int a, int b) { return A[(size_t)a * n + a] < A[(size_t)b * n + b]; });
    eval.resize(n);
    std::vector<double> V((size_t)n * n);
    for (int k = 0; k < n; ++k) {
        eval[k] = A[(size_t)idx[k] * n + idx[k]];
        for (int i = 0; i < n; ++i) V[(size_t)i * n + k] = evec[(size_t)i * n + idx[k]];
    }
    evec.swap(V);
}

}  // namespace linalg
}  // namespace gfnff
