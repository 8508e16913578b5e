// TEST INFRASTRUCTURE ONLY.  CPU restatement of curcuma's ALPB solvation per geometry
// (ff_methods/alpb_solvation.cpp), used by the oracle as the parity checker of the device
// kernels.  Pinned against curcuma's xtb 6.7.1 references (gfnff_alpb_xtb.ref.json).
#include "alpb_oracle.h"

#include <cmath>

namespace gfnff {
namespace {

using namespace alpb;

// contributions of one pair (i > j) to psi_i and psi_j and their derivatives along d = r_i - r_j
// (alpb_solvation.cpp:502-649): per side the non-overlapping or the
// overlapping form, by whether r is below rvdw_self + rho_other
struct PsiPair {
    double gi = 0.0, gj = 0.0;    // psi_i, psi_j contributions
    double di = 0.0, dj = 0.0;    // d psi_i / d r_i = di * d; d psi_j / d r_j = dj * d
};

static void no_overlap(double r, double rho, double sign, double& g, double& dv)
{
    const double r1 = 1.0 / r, ap = r + rho, am = r - rho, ab = ap * am;
    const double rhab = rho / ab, lnab = 0.5 * std::log(am / ap) * r1;
    g += rhab + lnab;
    dv += sign * (-2.0 * rhab / ab + (rhab - lnab) * r1 * r1);
}

static void overlap(double r, double rho, double rvdw, double sign, double& g, double& dv)
{
    if (r + rho <= rvdw) return;   // completely inside
    const double r1 = 1.0 / r, r12 = 0.5 * r1, r24 = r12 * r12;
    const double ap = r + rho, am = r - rho, rh1 = 1.0 / rvdw, rhr1 = 1.0 / ap, aprh1 = ap * rh1;
    const double lnab = std::log(aprh1);
    g += rh1 - rhr1 + r12 * (0.5 * am * (rhr1 - rh1 * aprh1) - lnab);
    double dgi = rhr1 * rhr1 * (1.0 - 0.25 * am * r1 * (1.0 + aprh1 * aprh1)) + rho * r24 * (rhr1 - rh1 * aprh1) +
                 r12 * (r1 * lnab - rhr1);
    dv += sign * dgi * r1;
}

static PsiPair psi_pair(const AlpbModel& A, int i, int j, double r)
{
    PsiPair p;
    const double rhoi = A.rho[i], rhoj = A.rho[j], rvi = A.vdwr[i], rvj = A.vdwr[j];
    const bool ovij = r < rvi + rhoj, ovji = r < rhoi + rvj;
    if (!ovij && !ovji && std::fabs(rhoi - rhoj) < 1e-8) {
        // equal radii: the form of rho_j on both sides
        double g = 0.0, d = 0.0;
        no_overlap(r, rhoj, 1.0, g, d);
        p.gi = p.gj = g;
        p.di = d;
        p.dj = -d;
        return p;
    }
    if (ovij) overlap(r, rhoj, rvi, 1.0, p.gi, p.di);
    else no_overlap(r, rhoj, 1.0, p.gi, p.di);
    if (ovji) overlap(r, rhoi, rvj, -1.0, p.gj, p.dj);
    else no_overlap(r, rhoi, -1.0, p.gj, p.dj);
    return p;
}

static double d2(const double* x, int i, int j, double d[3])
{
    d[0] = x[3 * i] - x[3 * j];
    d[1] = x[3 * i + 1] - x[3 * j + 1];
    d[2] = x[3 * i + 2] - x[3 * j + 2];
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
}

// surface area of atom i (alpb_solvation.cpp:696-805); with weight != 0 the
// derivative w * d sasa_i / d r is added into grad
static double sasa_atom(const AlpbModel& A, const double* x, int n, int i, double weight, double* grad)
{
    std::vector<int> nb;
    const double src2 = A.srcut * A.srcut, lr2 = kLrCut * kLrCut;
    for (int j = 0; j < n; ++j) {
        if (j == i) continue;
        double d[3];
        const double r2 = d2(x, i, j, d);
        if (r2 < lr2 && r2 < src2) nb.push_back(j);
    }
    std::vector<double> gr(3 * nb.size());
    std::vector<int> gi(nb.size());
    double s = 0.0;
    for (int p = 0; p < kNang; ++p) {
        const double px = x[3 * i] + A.vdwsa[i] * A.grid[3 * p], py = x[3 * i + 1] + A.vdwsa[i] * A.grid[3 * p + 1],
                     pz = x[3 * i + 2] + A.vdwsa[i] * A.grid[3 * p + 2];
        double sp = 1.0;
        int nn = 0;
        for (int j : nb) {
            const double t0 = px - x[3 * j], t1 = py - x[3 * j + 1], t2 = pz - x[3 * j + 2];
            const double tj2 = t0 * t0 + t1 * t1 + t2 * t2;
            if (tj2 >= A.trj2_hi[j]) continue;
            if (tj2 <= A.trj2_lo[j]) {
                sp = 0.0;
                break;
            }
            const double sq = std::sqrt(tj2), uj = sq - A.vdwsa[j], ah3uj2 = kAh3 * uj * uj;
            double ds = kAh1 + 3.0 * ah3uj2;
            const double sij = kAh0 + (kAh1 + ah3uj2) * uj;
            sp *= sij;
            ds = ds / (sij * sq);
            gi[nn] = j;
            gr[3 * nn] = ds * t0;
            gr[3 * nn + 1] = ds * t1;
            gr[3 * nn + 2] = ds * t2;
            ++nn;
        }
        if (sp > kTolSesp) {
            const double wsa = A.weight[p] * A.wrp[i] * sp;
            s += wsa;
            if (weight != 0.0)
                for (int k = 0; k < nn; ++k)
                    for (int c = 0; c < 3; ++c) {
                        const double dr = weight * wsa * gr[3 * k + c];
                        grad[3 * i + c] += dr;
                        grad[3 * gi[k] + c] -= dr;
                    }
        }
    }
    return s;
}

// inertia-like shape tensor of the vdW spheres (alpb_solvation.cpp:908-938): adet, and for the
// gradient the tensor, the centre and the total r^3
struct Shape {
    double I[3][3] = {{0}}, c[3] = {0, 0, 0}, tot3 = 0.0, adet = 0.0;
};

static Shape shape(const AlpbModel& A, const double* x, int n)
{
    constexpr double tof = 2.0 / 5.0;
    Shape s;
    for (int i = 0; i < n; ++i) {
        const double r3 = A.vdwr[i] * A.vdwr[i] * A.vdwr[i];
        s.tot3 += r3;
        for (int d = 0; d < 3; ++d) s.c[d] += x[3 * i + d] * r3;
    }
    for (int d = 0; d < 3; ++d) s.c[d] /= s.tot3;
    for (int i = 0; i < n; ++i) {
        const double r2a = A.vdwr[i] * A.vdwr[i], r3 = r2a * A.vdwr[i];
        double v[3];
        for (int d = 0; d < 3; ++d) v[d] = x[3 * i + d] - s.c[d];
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) s.I[a][b] += r3 * ((a == b ? r2 + tof * r2a : 0.0) - v[a] * v[b]);
    }
    const double det = s.I[0][0] * (s.I[1][1] * s.I[2][2] - s.I[1][2] * s.I[2][1]) -
                       s.I[0][1] * (s.I[1][0] * s.I[2][2] - s.I[1][2] * s.I[2][0]) +
                       s.I[0][2] * (s.I[1][0] * s.I[2][1] - s.I[1][1] * s.I[2][0]);
    s.adet = std::sqrt(std::pow(det, 1.0 / 3.0) / (tof * s.tot3));
    return s;
}

}  // namespace

void alpb_prepare(const AlpbModel& A, const double* x, int n, AlpbGeom& g, double* Aeeq)
{
    g.psi.assign(n, 0.0);
    // ---- Born radii (alpb_solvation.cpp:502-694)
    const double lr2 = kLrCut * kLrCut;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) {
            double d[3];
            const double r2 = d2(x, i, j, d);
            if (r2 >= lr2) continue;
            const PsiPair p = psi_pair(A, i, j, std::sqrt(r2));
            g.psi[i] += p.gi;
            g.psi[j] += p.gj;
        }
    g.brad.resize(n);
    g.dpsi.resize(n);
    for (int i = 0; i < n; ++i) {
        const double s1 = 1.0 / A.svdw[i], v1 = 1.0 / A.vdwr[i], s2 = 0.5 * A.svdw[i];
        const double br = g.psi[i] * s2;
        double arg2 = br * (kObcGamma * br - kObcBeta);
        const double arg = br * (kObcAlpha + arg2);
        arg2 = 2.0 * arg2 + kObcAlpha + kObcGamma * br * br;
        const double th = std::tanh(arg), ch = std::cosh(arg);
        g.brad[i] = A.born_scale / (s1 - v1 * th);
        double dp = ch * (s1 - v1 * th);
        dp = s2 * v1 * arg2 / (dp * dp);
        g.dpsi[i] = A.born_scale * dp;
    }
    // ---- surface areas, HB weights (alpb_solvation.cpp:873-881), shape
    g.sasa.resize(n);
    g.hbw.assign(n, 0.0);
    g.dhbdw.assign(n, 0.0);
    g.gsasa = 0.0;
    for (int i = 0; i < n; ++i) {
        g.sasa[i] = sasa_atom(A, x, n, i, 0.0, nullptr);
        g.gsasa += g.sasa[i] * A.gamsasa[i];
        if (A.lhb) {
            const double smaxd = 1.0 / (A.vdwsa[i] * A.vdwsa[i]);
            g.hbw[i] = A.hbmag[i] * g.sasa[i] * smaxd;
            g.dhbdw[i] = A.hbmag[i] * smaxd;
        }
    }
    g.adet = shape(A, x, n).adet;
    // ---- Born matrix into the EEQ matrix (eeq_solver.cpp:3781-3784: A += B)
    if (!Aeeq) return;
    const double corr = A.keps * A.alpbet / g.adet;
    for (int i = 0; i < n; ++i) {
        Aeeq[(size_t)i * n + i] += A.keps / g.brad[i] + 2.0 * g.hbw[i] + corr;
        for (int j = 0; j < i; ++j) {
            double d[3];
            const double r = std::sqrt(d2(x, i, j, d));
            const double ab = std::sqrt(g.brad[i] * g.brad[j]);
            double a = ab / (ab + kZetaP16o16 * r);
            a *= a; a *= a; a *= a; a *= a;
            const double b = A.keps / (r + ab * a) + corr;
            Aeeq[(size_t)i * n + j] += b;
            Aeeq[(size_t)j * n + i] += b;
        }
    }
}

double alpb_energy_gradient(const AlpbModel& A, const double* x, int n, const AlpbGeom& g, const double* q, double* grad)
{
    // ---- Born energy and its direct and Born-radius gradient (alpb_solvation.cpp:1139-1203)
    std::vector<double> dEdbr(n, 0.0);
    double egb = 0.0, qt = 0.0;
    for (int i = 0; i < n; ++i) {
        qt += q[i];
        for (int j = 0; j < i; ++j) {
            double d[3];
            const double r = std::sqrt(d2(x, i, j, d));
            const double qq = q[i] * q[j];
            const double ab = std::sqrt(g.brad[i] * g.brad[j]);
            const double a1 = ab / (ab + kZetaP16o16 * r);
            double a16 = a1 * a1;
            a16 *= a16; a16 *= a16; a16 *= a16;
            const double fgb = r + ab * a16, dfgb = 1.0 / fgb, dfgb2 = dfgb * dfgb;
            egb += qq * A.keps * dfgb;
            const double ap = (1.0 - kZetaP16 * a1 * a16) * dfgb2;
            for (int c = 0; c < 3; ++c) {
                const double dG = ap * d[c] * A.keps / r * qq;
                grad[3 * i + c] -= dG;
                grad[3 * j + c] += dG;
            }
            const double bp = -0.5 * (r * kZetaP16 / ab * a1 + 1.0) / ab * a16 * dfgb2;
            dEdbr[i] += g.brad[j] * bp * A.keps * qq;
            dEdbr[j] += g.brad[i] * bp * A.keps * qq;
        }
    }
    for (int i = 0; i < n; ++i) {
        const double bp = 1.0 / g.brad[i], qb = q[i] * bp;
        egb += 0.5 * q[i] * qb * A.keps;
        dEdbr[i] += -0.5 * A.keps * qb * bp * q[i];
    }
    // d brad_i / d r through psi: per pair, psi_i along d = r_i - r_j (and psi_j)
    const double lr2 = kLrCut * kLrCut;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) {
            double d[3];
            const double r2 = d2(x, i, j, d);
            if (r2 >= lr2) continue;
            const PsiPair p = psi_pair(A, i, j, std::sqrt(r2));
            const double wi = dEdbr[i] * g.dpsi[i] * p.di, wj = dEdbr[j] * g.dpsi[j] * p.dj;
            for (int c = 0; c < 3; ++c) {
                grad[3 * i + c] += wi * d[c];
                grad[3 * j + c] -= wi * d[c];
                grad[3 * j + c] += wj * d[c];
                grad[3 * i + c] -= wj * d[c];
            }
        }
    // ---- HB term (kept in the Born matrix diagonal) and the surface gradient
    double ghb = 0.0;
    for (int i = 0; i < n; ++i) ghb += g.hbw[i] * q[i] * q[i];
    for (int i = 0; i < n; ++i) {
        const double w = A.gamsasa[i] + g.dhbdw[i] * q[i] * q[i];
        if (w != 0.0) sasa_atom(A, x, n, i, w, grad);
    }
    // ---- ALPB shape term (alpb_solvation.cpp:940-1003)
    double eshape = 0.0;
    if (A.alpbet > 0.0) {
        const Shape s = shape(A, x, n);
        eshape = 0.5 * qt * qt * A.alpbet / s.adet * A.keps;
        const double (&I)[3][3] = s.I;
        double D[3][3];
        D[0][0] = I[0][0] * (I[1][1] + I[2][2]) - I[0][1] * I[0][1] - I[0][2] * I[0][2];
        D[0][1] = I[0][1] * I[2][2] - I[0][2] * I[1][2];
        D[0][2] = I[0][2] * I[1][1] - I[0][1] * I[2][1];
        D[1][0] = D[0][1];
        D[1][1] = I[1][1] * (I[0][0] + I[2][2]) - I[0][1] * I[0][1] - I[1][2] * I[1][2];
        D[1][2] = I[0][0] * I[1][2] - I[0][1] * I[0][2];
        D[2][0] = D[0][2];
        D[2][1] = D[1][2];
        D[2][2] = I[2][2] * (I[0][0] + I[1][1]) - I[0][2] * I[0][2] - I[1][2] * I[1][2];
        const double ke = A.keps * A.alpbet;
        const double scale = (250.0 / (48.0 * s.tot3 * s.tot3 * s.tot3 * std::pow(s.adet, 5.0))) *
                             (-0.5 * ke * qt * qt / (s.adet * s.adet));
        for (int i = 0; i < n; ++i) {
            const double r3 = A.vdwr[i] * A.vdwr[i] * A.vdwr[i];
            double v[3];
            for (int c = 0; c < 3; ++c) v[c] = x[3 * i + c] - s.c[c];
            for (int a = 0; a < 3; ++a)
                grad[3 * i + a] += r3 * scale * (D[a][0] * v[0] + D[a][1] * v[1] + D[a][2] * v[2]);
        }
    }
    // gborn (with the shape term) + ghb + gsasa + gshift
    return egb + eshape + ghb + g.gsasa + A.gshift;
}

}  // namespace gfnff
