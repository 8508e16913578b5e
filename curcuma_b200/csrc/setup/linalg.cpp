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
                     const double* qf, double* q)
{
    std::vector<double> Acopy;
    const bool keep = true;
    if (keep) Acopy.assign(A, A + (size_t)n * n);
    if (cholesky(A, n)) {
        // right-hand sides: column 0 = x, columns 1..nfrag = C^T
        const int nr = 1 + nfrag;
        std::vector<double> B((size_t)n * nr, 0.0);
        for (int i = 0; i < n; ++i) {
            B[(size_t)i * nr] = x[i];
            B[(size_t)i * nr + 1 + frag[i]] = 1.0;
        }
        cholesky_solve(A, n, B.data(), nr);
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
