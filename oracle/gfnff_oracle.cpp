// TEST INFRASTRUCTURE ONLY: the CPU oracle for the per-geometry GFN-FF energy and
// gradient.  Every block restates the curcuma routine named beside it (paths relative
// to src/core/energy_calculators/ff_methods/ unless noted).  The product library never
// links this file; tests and bench.py's CPU baseline use it as the checker.
#include "gfnff_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../curcuma_b200/csrc/setup/linalg.h"
#include "alpb_oracle.h"
#include "../curcuma_b200/csrc/setup/model.h"
#include "../curcuma_b200/csrc/tables/gfnff_tables.inc"

using namespace gfnff;

namespace {

thread_local std::string g_err;

struct V3 {
    double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }

// Periodic cell, minimum-image convention of curcuma's CUDA kernels
// (cuda/gfnff_kernels.cu:92-119): h holds the lattice vectors as columns, h[3*col + row]
// (bohr), hi its inverse; d -> h (f - rint(f)) with f = hi d.
struct OCell {
    double h[9] = {0}, hi[9] = {0};
    bool on = false;
    V3 operator()(V3 d) const
    {
        if (!on) return d;
        double f[3];
        for (int r = 0; r < 3; ++r) {
            f[r] = hi[r] * d.x + hi[3 + r] * d.y + hi[6 + r] * d.z;
            f[r] -= std::rint(f[r]);
        }
        return {h[0] * f[0] + h[3] * f[1] + h[6] * f[2], h[1] * f[0] + h[4] * f[1] + h[7] * f[2],
                h[2] * f[0] + h[5] * f[1] + h[8] * f[2]};
    }
};

struct Grad {
    std::vector<double> g;
    explicit Grad(int n) : g(3 * (size_t)n, 0.0) {}
    void add(int i, V3 v) { g[3 * i] += v.x; g[3 * i + 1] += v.y; g[3 * i + 2] += v.z; }
};

}  // namespace

struct oracle_handle {
    Model m;
    AlpbModel solv;   // ALPB implicit solvation (off: gas phase)
    OCell cell;       // periodic cell (off: isolated system)
};

// ---------------------------------------------------------------------------------
// Geometry helpers: forcefieldfunctions.h:35-83 (BondStretching, AngleBending),
// gfnff_geometry.h:66-160 (calculateDihedralAngle), :207-265 (calculateOutOfPlaneAngle)
// ---------------------------------------------------------------------------------
static double angle_cos(V3 i, V3 j, V3 k, V3 d[3])
{
    V3 rij = i - j, rkj = k - j;
    double a = norm(rij), b = norm(rkj);
    d[0] = d[1] = d[2] = {0, 0, 0};
    if (a < 1e-10 || b < 1e-10) return 1.0;
    V3 nij = (1.0 / a) * rij, nkj = (1.0 / b) * rkj;
    double c = dot(rij, rkj) / (a * b);
    c = std::max(-1.0, std::min(1.0, c));
    double s = std::sqrt(std::max(0.0, 1.0 - c * c));
    if (s < 1e-14) return c;
    double f = 1.0 / s;
    d[0] = (-f / a) * (nkj - c * nij);
    d[2] = (-f / b) * (nij - c * nkj);
    d[1] = -1.0 * (d[0] + d[2]);
    return c;
}

static double dihedral(V3 ri, V3 rj, V3 rk, V3 rl, V3 g[4])
{
    for (int a = 0; a < 4; ++a) g[a] = {0, 0, 0};
    V3 v1 = rj - ri, v2 = rk - rj, v3 = rl - rk;
    V3 n1 = cross(v1, v2), n2 = cross(v2, v3);
    double n1n = norm(n1), n2n = norm(n2), v2n = norm(v2);
    if (n1n < 1e-10 || n2n < 1e-10 || v2n < 1e-10) return 0.0;
    V3 h1 = (1.0 / n1n) * n1, h2 = (1.0 / n2n) * n2;
    double cphi = dot(h1, h2);
    double sphi = (v2n * dot(h1, v3)) / n2n;
    sphi = std::max(-1.0, std::min(1.0, sphi));
    double phi = std::atan2(sphi, cphi);
    double nen = n1n * n2n * std::sin(phi);
    if (std::fabs(nen) < 1e-14) return phi;
    double o = 1.0 / nen;
    V3 rab = cross(n1, v2), rbb = cross(n2, v2), rac = cross(n1, v3), rbc = cross(n2, v3);
    V3 rba = cross(n2, v1), raa = cross(n1, v1);
    V3 rapb = v1 + v2, rbpc = v2 + v3;
    V3 rapba = cross(rapb, n1), rapbb = cross(rapb, n2), rbpca = cross(rbpc, n1), rbpcb = cross(rbpc, n2);
    g[0] = o * ((cphi * n2n / n1n) * rab - rbb);
    g[1] = o * (cphi * ((n2n / n1n) * rapba + (n1n / n2n) * rbc) - (rac + rapbb));
    g[2] = o * (cphi * ((n2n / n1n) * raa + (n1n / n2n) * rbpcb) - (rba + rbpca));
    g[3] = o * ((cphi * n1n / n2n) * rbb - rab);
    return phi;
}

static double oop(V3 ri, V3 rj, V3 rk, V3 rl, V3 g[4])
{
    for (int a = 0; a < 4; ++a) g[a] = {0, 0, 0};
    V3 re = ri - rj, rd = rk - rj, rv = rl - ri;
    V3 rn = cross(re, rd);
    double rnn = norm(rn), rvn = norm(rv);
    if (rnn < 1e-10 || rvn < 1e-10) return 0.0;
    double so = dot((1.0 / rnn) * rn, (1.0 / rvn) * rv);
    so = std::max(-1.0, std::min(1.0, so));
    double om = std::asin(so);
    double nen = rnn * rvn * std::cos(om);
    if (std::fabs(nen) < 1e-14) return om;
    double o = 1.0 / nen, s = std::sin(om);
    V3 rdme = rd - re, rve = cross(rv, re), rne = cross(rn, re), rdv = cross(rd, rv), rdn = cross(rd, rn);
    V3 rvdme = cross(rv, rdme), rndme = cross(rn, rdme);
    g[0] = o * (rdv - rn - s * ((rvn / rnn) * rdn - (rnn / rvn) * rv));
    g[1] = o * (rvdme - (s * rvn / rnn) * rndme);
    g[2] = o * (rve - (s * rvn / rnn) * rne);
    g[3] = o * (rn - (s * rnn / rvn) * rv);
    return om;
}

// With a periodic cell (mic.on) the displacement vectors of the terms curcuma's CUDA kernels
// treat with the minimum image take it (CN and its chain rule, HB coordination numbers,
// bonds, angles, the A-H, H-B and A-B vectors of HB and XB terms, repulsion, Coulomb and D4
// pairs); torsions, inversions, ATM, BATM, the EEQ matrix and the set-up lists (D4 pairs by
// set-up distance) use plain differences.
static int engrad(const Model& m, const AlpbModel& solv, const OCell& mic, const double* xb, double* T, double* gout,
                  double* qout, double* cnout)
{
    const int n = m.n;
    AlpbGeom sg;   // ALPB state of this geometry (gfnff_method.cpp:1128-1140, 1805-1853)
    auto X = [&](int i) { return V3{xb[3 * i], xb[3 * i + 1], xb[3 * i + 2]}; };
    auto D = [&](int a, int b) { return mic(X(b) - X(a)); };   // x_b - x_a, minimum image
    for (int t = 0; t < ORC_NTERMS; ++t) T[t] = 0.0;
    Grad G(n);
    std::vector<double> dEdcn(n, 0.0);

    // ---- CN with the 6 bohr neighbour list: cn_calculator.cpp:367-428 -------------
    const double kn = -7.5, cnmax = 4.4;
    std::vector<std::vector<int>> nbr(n);
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            V3 d = D(j, i);
            if (d.x * d.x + d.y * d.y + d.z * d.z < 36.0) { nbr[i].push_back(j); nbr[j].push_back(i); }
        }
    std::vector<double> cnraw(n, 0.0), cn(n, 0.0);
    for (int i = 0; i < n; ++i) {
        std::sort(nbr[i].begin(), nbr[i].end());
        double s = 0.0;
        for (int j : nbr[i]) {
            const double r = norm(D(j, i));
            const double rc = m.rcov_cn[i] + m.rcov_cn[j];
            s += 0.5 * (1.0 + std::erf(kn * ((r - rc) / rc)));
        }
        cnraw[i] = s;
        cn[i] = std::log(1.0 + std::exp(cnmax)) - std::log(1.0 + std::exp(cnmax - s));
    }
    if (cnout) std::copy(cn.begin(), cn.end(), cnout);

    // ---- D4 weights + dC6/dCN at the step CN: d4param_generator.cpp:1079-1930 ------
    const int K = (int)m.present_Z.size();
    std::vector<double> w((size_t)n * kMaxRef), dw((size_t)n * kMaxRef);
    for (int i = 0; i < n; ++i) d4_weights(m, i, cn[i], &w[(size_t)i * kMaxRef], &dw[(size_t)i * kMaxRef]);
    std::vector<double> hg((size_t)n * K * kMaxRef, 0.0), hdg((size_t)n * K * kMaxRef, 0.0);
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < K; ++s) {
            const double* C = &m.c6ref[(((size_t)m.slot[i] * K + s) * kMaxRef) * kMaxRef];
            for (int b = 0; b < kMaxRef; ++b) {
                double g = 0.0, dg = 0.0;
                for (int a = 0; a < m.nref[i]; ++a) {
                    g += w[(size_t)i * kMaxRef + a] * C[a * kMaxRef + b];
                    dg += dw[(size_t)i * kMaxRef + a] * C[a * kMaxRef + b];
                }
                hg[((size_t)i * K + s) * kMaxRef + b] = g;
                hdg[((size_t)i * K + s) * kMaxRef + b] = dg;
            }
        }

    // ---- EEQ Phase 2: eeq_solver.cpp:3201-3700 + Schur Cholesky :2087-2256 ---------
    std::vector<double> q(n, 0.0);
    {
        const double TSQRT2PI = 0.797884560802866;
        std::vector<double> A((size_t)n * n), x(n);
#pragma omp parallel for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            A[(size_t)i * n + i] = m.gam[i] + TSQRT2PI / std::sqrt(m.alpeeq[i]);
            for (int j = 0; j < i; ++j) {
                const double dx = xb[3 * i] - xb[3 * j], dy = xb[3 * i + 1] - xb[3 * j + 1],
                             dz = xb[3 * i + 2] - xb[3 * j + 2];
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                const double g = 1.0 / std::sqrt(m.alpeeq[i] + m.alpeeq[j]);
                const double v = std::erf(g * r) / r;
                A[(size_t)i * n + j] = v;
                A[(size_t)j * n + i] = v;
            }
        }
        for (int i = 0; i < n; ++i) x[i] = m.chi_base[i] + m.cnf[i] * std::sqrt(cn[i]);
        // implicit solvation: the solvent's reaction field enters the solve, A += B
        if (solv.on) alpb_prepare(solv, xb, n, sg, A.data());
        if (!linalg::eeq_schur_solve(A.data(), n, x.data(), m.frag.data(), m.nfrag, m.qfrag.data(), q.data(),
                                     n >= 1024)) {
            g_err = "EEQ solve failed";
            return 3;
        }
    }
    if (qout) std::copy(q.begin(), q.end(), qout);

    // ---- HB coordination numbers: ff_workspace_gfnff.cpp:46-99 --------------------
    struct HBG { int H, B; V3 dH, dB; };
    std::vector<HBG> hbg;
    std::unordered_map<int, double> hbcn;
    {
        const double kn2 = 27.5, inv_sqrt_pi = 0.5641895835477563;
        for (const auto& e : m.bond_hb) {
            const int H = e.h;
            for (int B : e.b_atoms) {
                V3 d = D(H, B);
                const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                if (r2 > 900.0) continue;
                const double r = std::sqrt(r2);
                const double rc = 1.78 * (4.0 / 3.0) * (m.rcov_d3[H] + m.rcov_d3[B]);
                const double arg = -kn2 * (r - rc) / rc;
                hbcn[H] += 0.5 * (1.0 + std::erf(arg));
                const double dcn = inv_sqrt_pi * (-kn2 / rc) * std::exp(-arg * arg) / r;
                hbg.push_back({H, B, (-dcn) * d, dcn * d});
            }
        }
    }

    // ---- bonds: ff_workspace_gfnff.cpp:104-182 ------------------------------------
    for (const auto& b : m.bonds) {
        V3 ij = D(b.j, b.i);
        const double r = norm(ij);
        V3 d0 = (1.0 / r) * ij;
        const double r0 = (b.r0_base_i + b.cnfak_i * cn[b.i] + b.r0_base_j + b.cnfak_j * cn[b.j] + b.rabshift) * b.ff;
        const double dr = r - r0;
        double alpha = b.alpha;
        double hcn = 0.0;
        if (b.nr_hb >= 1) {
            auto it = hbcn.find(b.hb_h);
            hcn = it == hbcn.end() ? 0.0 : it->second;
            alpha = (-(1.0 - 0.9) * hcn + 1.0) * b.alpha;
        }
        const double e = b.fc * std::exp(-alpha * dr * dr);
        T[ORC_BOND] += e;
        const double dEdr = -2.0 * alpha * dr * e;
        G.add(b.i, dEdr * d0);
        G.add(b.j, (-dEdr) * d0);
        if (b.nr_hb >= 1) {
            const double zz = 0.1 * b.alpha * dr * dr * e;
            for (const auto& h : hbg) {
                if (h.H != b.hb_h) continue;
                G.add(h.H, zz * h.dH);
                G.add(h.B, zz * h.dB);
            }
        }
        const double yy = -dEdr;
        dEdcn[b.i] += yy * b.ff * b.cnfak_i;
        dEdcn[b.j] += yy * b.ff * b.cnfak_j;
    }

    // ---- angles: :187-280 ----------------------------------------------------------
    {
        const double atcuta = 0.595;
        for (const auto& a : m.angles) {
            V3 pi = D(a.j, a.i), pj{0, 0, 0}, pk = D(a.j, a.k), d[3];   // the apex as the origin
            double c = angle_cos(pi, pj, pk, d);
            c = std::max(-1.0, std::min(1.0, c));
            const double th = std::acos(c);
            double e, dedth;
            if (std::fabs(M_PI - a.theta0) < 1e-6) {
                const double dt = th - a.theta0;
                e = a.fc * dt * dt;
                dedth = 2.0 * a.fc * dt;
            } else {
                const double c0 = std::cos(a.theta0), dc = c - c0;
                e = a.fc * dc * dc;
                dedth = 2.0 * a.fc * std::sin(th) * (c0 - c);
            }
            const double rij2 = dot(pi - pj, pi - pj), rjk2 = dot(pk - pj, pk - pj);
            const double ri = m.rcov_d3[a.i] * (4.0 / 3.0), rj = m.rcov_d3[a.j] * (4.0 / 3.0),
                         rk = m.rcov_d3[a.k] * (4.0 / 3.0);
            const double cij = atcuta * (ri + rj) * (ri + rj), cjk = atcuta * (rj + rk) * (rj + rk);
            double rrij = rij2 / cij; rrij = rrij * rrij;
            double rrjk = rjk2 / cjk; rrjk = rrjk * rrjk;
            const double dij = 1.0 / (1.0 + rrij), djk = 1.0 / (1.0 + rrjk), damp = dij * djk;
            const double d2ij = rij2 > 1e-8 ? -2.0 * 2.0 * rrij / (rij2 * (1.0 + rrij) * (1.0 + rrij)) : 0.0;
            const double d2jk = rjk2 > 1e-8 ? -2.0 * 2.0 * rrjk / (rjk2 * (1.0 + rrjk) * (1.0 + rrjk)) : 0.0;
            T[ORC_ANGLE] += e * damp;
            V3 t1 = (e * d2ij * djk) * (pi - pj), t2 = (e * d2jk * dij) * (pk - pj);
            G.add(a.i, (dedth * damp) * d[0] + t1);
            G.add(a.j, (dedth * damp) * d[1] - t1 - t2);
            G.add(a.k, (dedth * damp) * d[2] + t2);
        }
    }

    // ---- torsions (primary + extra): :282-487 ---------------------------------------
    for (size_t t = 0; t < m.torsions.size(); ++t) {
        const auto& d = m.torsions[t];
        const bool extra = (int)t >= m.n_primary_torsions;
        V3 ri = X(d.i), rj = X(d.j), rk = X(d.k), rl = X(d.l), g[4];
        const double phi = dihedral(ri, rj, rk, rl, g);
        const double c1 = d.n * (phi - d.phi0) + M_PI;
        const double e = d.V * (1.0 + std::cos(c1));
        const double atc = (!extra && d.nci) ? 0.305 : 0.505;
        auto rc = [&](int a) { return m.rcov_d3[a] * (4.0 / 3.0); };
        const double rij2 = dot(ri - rj, ri - rj), rjk2 = dot(rj - rk, rj - rk), rkl2 = dot(rk - rl, rk - rl);
        const double cij = atc * (rc(d.i) + rc(d.j)) * (rc(d.i) + rc(d.j));
        const double cjk = atc * (rc(d.j) + rc(d.k)) * (rc(d.j) + rc(d.k));
        const double ckl = atc * (rc(d.k) + rc(d.l)) * (rc(d.k) + rc(d.l));
        double a1 = rij2 / cij; a1 *= a1;
        double a2 = rjk2 / cjk; a2 *= a2;
        double a3 = rkl2 / ckl; a3 *= a3;
        const double dij = 1.0 / (1.0 + a1), djk = 1.0 / (1.0 + a2), dkl = 1.0 / (1.0 + a3);
        const double damp = dij * djk * dkl;
        T[ORC_TORSION] += e * damp;
        const double dEdphi = -d.V * d.n * std::sin(c1) * damp;
        G.add(d.i, dEdphi * g[0]);
        G.add(d.j, dEdphi * g[1]);
        G.add(d.k, dEdphi * g[2]);
        G.add(d.l, dEdphi * g[3]);
        const double e2ij = rij2 > 1e-8 ? -4.0 * a1 / (rij2 * (1.0 + a1) * (1.0 + a1)) : 0.0;
        const double e2jk = rjk2 > 1e-8 ? -4.0 * a2 / (rjk2 * (1.0 + a2) * (1.0 + a2)) : 0.0;
        const double e2kl = rkl2 > 1e-8 ? -4.0 * a3 / (rkl2 * (1.0 + a3) * (1.0 + a3)) : 0.0;
        V3 t1 = (e * e2ij * djk * dkl) * (ri - rj), t2 = (e * dij * e2jk * dkl) * (rj - rk),
           t3 = (e * dij * djk * e2kl) * (rk - rl);
        G.add(d.i, t1);
        G.add(d.j, t2 - t1);
        G.add(d.k, t3 - t2);
        G.add(d.l, -1.0 * t3);
    }

    // ---- inversions: :489-609 ------------------------------------------------------
    for (const auto& v : m.inversions) {
        V3 rc = X(v.i), r1 = X(v.j), r2 = X(v.k), r3 = X(v.l), g[4];
        const double om = oop(rc, r1, r2, r3, g);
        auto rcv = [&](int a) { return m.rcov_d3[a] * (4.0 / 3.0); };
        auto damp = [](double rsq, double a, double b) {
            const double cut = 0.505 * (a + b) * (a + b);
            const double rr = (rsq / cut) * (rsq / cut);
            return 1.0 / (1.0 + rr);
        };
        auto ddamp = [](double r2, double a, double b) {
            if (r2 < 1e-8) return 0.0;
            const double cut = 0.505 * (a + b) * (a + b);
            const double rr = (r2 / cut) * (r2 / cut);
            return -4.0 * rr / (r2 * (1.0 + rr) * (1.0 + rr));
        };
        const double rij2 = dot(r1 - rc, r1 - rc), rjk2 = dot(r1 - r2, r1 - r2), rjl2 = dot(r1 - r3, r1 - r3);
        const double ci = rcv(v.i), c1 = rcv(v.j), c2 = rcv(v.k), c3 = rcv(v.l);
        const double dij = damp(rij2, ci, c1), djk = damp(rjk2, c2, c1), djl = damp(rjl2, c1, c3);
        const double dmp = dij * djk * djl;
        double et, dEdom;
        if (v.type == 0) {
            et = v.fc * (1.0 - std::cos(om));
            dEdom = v.fc * std::sin(om) * dmp;
        } else {
            const double df = std::cos(om) - std::cos(v.omega0);
            et = v.fc * df * df;
            dEdom = -2.0 * v.fc * std::sin(om) * df * dmp;
        }
        T[ORC_INVERSION] += et * dmp;
        G.add(v.i, dEdom * g[0]);
        G.add(v.j, dEdom * g[1]);
        G.add(v.k, dEdom * g[2]);
        G.add(v.l, dEdom * g[3]);
        const double e1 = ddamp(rij2, ci, c1), e2 = ddamp(rjk2, c2, c1), e3 = ddamp(rjl2, c1, c3);
        V3 t1 = (et * e1 * djk * djl) * (r1 - rc), t2 = (et * e2 * dij * djl) * (r1 - r2),
           t3 = (et * e3 * dij * djk) * (r1 - r3);
        G.add(v.i, -1.0 * t1);
        G.add(v.j, t1 + t2 + t3);
        G.add(v.k, -1.0 * t2);
        G.add(v.l, -1.0 * t3);
    }

    // ---- D4 dispersion: :715-772 ---------------------------------------------------
    for (const auto& d : m.disp) {
        V3 rv = D(d.j, d.i);
        const double r = norm(rv);
        if (r > 50.0 || r < 1e-10) continue;
        const double r2 = r * r, r6 = r2 * r2 * r2, r06 = d.r0sq * d.r0sq * d.r0sq;
        const double t6 = 1.0 / (r6 + r06);
        const double r8 = r6 * r2, r08 = r06 * d.r0sq;
        const double t8 = 1.0 / (r8 + r08);
        const double sum = t6 + 2.0 * d.r4r2 * t8;
        T[ORC_DISPERSION] += -d.c6 * sum * d.zetac6;
        const double d6 = -6.0 * r2 * r2 * t6 * t6, d8 = -8.0 * r2 * r2 * r2 * t8 * t8;
        const double dEdr = -d.c6 * d.zetac6 * (d6 + 2.0 * d.r4r2 * d8) * r;
        V3 g = (dEdr / r) * rv;
        G.add(d.i, g);
        G.add(d.j, -1.0 * g);
        const double val = sum * d.zetac6;
        const int sj = m.slot[d.j], si = m.slot[d.i];
        double dci = 0.0, dcj = 0.0;
        for (int b = 0; b < m.nref[d.j]; ++b) {
            dci += hdg[((size_t)d.i * K + sj) * kMaxRef + b] * w[(size_t)d.j * kMaxRef + b];
            dcj += hg[((size_t)d.i * K + sj) * kMaxRef + b] * dw[(size_t)d.j * kMaxRef + b];
        }
        (void)si;
        dEdcn[d.i] -= dci * val;
        dEdcn[d.j] -= dcj * val;
    }

    // ---- repulsion: :774-848 -------------------------------------------------------
    auto rep = [&](const RepPair& p, int slot) {
        V3 rv = D(p.j, p.i);
        const double r = norm(rv);
        if (r > 20.0 || r < 1e-8) return;
        const double e = p.repab * std::exp(-p.alpha * (r * std::sqrt(r))) / r;
        T[slot] += e;
        const double dEdr = -e / r - 1.5 * p.alpha * std::sqrt(r) * e;
        V3 g = (dEdr / r) * rv;
        G.add(p.i, g);
        G.add(p.j, -1.0 * g);
    };
    for (const auto& p : m.rep_bonded) rep(p, ORC_BONDED_REP);
    for (const auto& p : m.rep_nonbonded) rep(p, ORC_NONBONDED_REP);

    // ---- Coulomb pairs (r <= 100 bohr): :850-900 -----------------------------------
    {
        double ec = 0.0;
        std::vector<double> gc(3 * (size_t)n, 0.0);
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : ec)
        for (int i = 0; i < n; ++i) {
            double gx = 0.0, gy = 0.0, gz = 0.0;
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                V3 rv = D(j, i);
                const double r = norm(rv);
                if (r > 100.0 || r < 1e-10) continue;
                const double gam = 1.0 / std::sqrt(m.alpeeq[i] + m.alpeeq[j]);
                const double gr = gam * r;
                const double ef = std::erf(gr);
                if (j > i) ec += q[i] * q[j] * ef / r;
                const double dfr = gam * std::exp(-gr * gr) * (2.0 / 1.772453850905516);
                const double dEdr = q[i] * q[j] * (dfr / r - ef / (r * r));
                gx += dEdr * rv.x / r;
                gy += dEdr * rv.y / r;
                gz += dEdr * rv.z / r;
            }
            gc[3 * i] = gx; gc[3 * i + 1] = gy; gc[3 * i + 2] = gz;
        }
        T[ORC_COULOMB] += ec;
        for (size_t k = 0; k < gc.size(); ++k) G.g[k] += gc[k];
    }

    // ---- hydrogen bonds: :938-1409 -------------------------------------------------
    {
        const double HB_BACUT = 49.0, HB_SCUT = 22.0, HB_ALP = 6.0, HB_LONGCUT = 85.0, HB_ST = 15.0,
                     HB_SF = 1.0, HB_NBCUT = 11.20, TORS_HB = 0.94, BEND_HB = 0.20, XHACI_GLOBABH = 0.268,
                     XHACI_COH = 0.350, HBLPCUT = 56.0;
        auto qs = [&](double qq) { const double e = std::exp(HB_ST * qq); return e / (e + HB_SF); };
        for (const auto& hb : m.hbonds) {
            V3 pA = X(hb.a), pB = X(hb.b);
            // A-H, H-B, A-B: minimum image; the neighbour, lone-pair and carbonyl vectors: plain
            const V3 vAH = D(hb.a, hb.h), vHB = D(hb.h, hb.b), vAB = D(hb.a, hb.b);
            const double rAH = norm(vAH), rHB = norm(vHB), rAB = norm(vAB);
            if (rAB > 50.0) continue;
            const double rAH4 = rAH * rAH * rAH * rAH, rHB4 = rHB * rHB * rHB * rHB;
            const double den = 1.0 / (rAH4 + rHB4);
            const double QH = qs(hb.q_h), QA = qs(-hb.q_a), QB = qs(-hb.q_b);
            const double bas = (QA * hb.bas_a * rAH4 + QB * hb.bas_b * rHB4) * den;
            const double aci = (hb.aci_b * rAH4 + hb.aci_a * rHB4) * den;
            const double rv = m.rvdw[hb.a] + m.rvdw[hb.b];
            const double dsh = 1.0 / (1.0 + std::pow(HB_SCUT * rv / (rAB * rAB), HB_ALP));
            const double dlg = 1.0 / (1.0 + std::pow(rAB * rAB / HB_LONGCUT, HB_ALP));
            const double denv = dsh * dlg;
            double doutl;
            {
                const double ex = (HB_BACUT / rv) * ((rAH + rHB) / rAB - 1.0);
                doutl = ex > 15.0 ? 0.0 : 2.0 / (1.0 + std::exp(ex));
            }
            const int zB = m.Z[hb.b];
            double onb = 1.0;
            if (hb.case_type >= 2) {
                const double cut = (zB == 7 && hb.nb_b.size() == 1) ? 2.0 : HB_NBCUT;
                for (int nb : hb.nb_b) {
                    const double ra = norm(X(nb) - pA), rb = norm(X(nb) - pB);
                    const double ex = (cut / rv) * ((ra + rb) / rAB - 1.0);
                    onb *= (2.0 / (1.0 + std::exp(-ex)) - 1.0);
                }
            }
            const double rdamp = hb.case_type >= 2
                                     ? denv * (1.8 / (rHB * rHB * rHB) - 0.8 / (rAB * rAB * rAB))
                                     : denv / (rAB * rAB * rAB);
            double olp = 1.0, lpd = 0.0;
            int nlp = 0;
            V3 lpv{0, 0, 0}, lpp = pB;
            if (hb.case_type == 4) {
                lpd = 0.50 - 0.018 * ((zB >= 1 && zB <= 86) ? gfnff_tables::repz[zB - 1] : 1.0);
                nlp = (int)hb.nb_b.size();
                for (int nb : hb.nb_b) lpv = lpv + (X(nb) - pB);
                const double vn = norm(lpv);
                if (vn > 1e-10 && nlp > 0) {
                    lpp = pB + (-lpd) * ((1.0 / vn) * lpv);
                    const double ral = norm(pA - lpp);
                    const double ex = (HBLPCUT / rv) * ((ral + lpd + 1e-12) / rAB - 1.0);
                    olp = 2.0 / (1.0 + std::exp(ex));
                } else {
                    nlp = 0;
                    olp = 1.0;
                }
            }
            const double qhoutl = QH * doutl * onb * olp;
            double eangl = 1.0, etors = 1.0;
            struct TG { double e; V3 g[4]; int D; };
            std::vector<TG> tg;
            V3 ga3[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            int jj = -1, kk = -1, ll = -1;
            if (hb.case_type == 3 && hb.parent_c != -1) {
                const int Bi = hb.b, Ci = hb.parent_c, Hi = hb.h;
                jj = Bi; kk = Ci; ll = Hi;
                {
                    const double c0 = 120.0 * M_PI / 180.0;
                    const double fc = 1.0 - BEND_HB;
                    const double kijk = fc / ((std::cos(0.0) - std::cos(c0)) * (std::cos(0.0) - std::cos(c0)));
                    V3 va = X(Ci), vb = X(Bi), vc = X(Hi);
                    V3 vab = va - vb, vcb = vc - vb;
                    const double rab2 = dot(vab, vab), rcb2 = dot(vcb, vcb);
                    V3 vp = cross(vcb, vab);
                    const double rp = norm(vp) + 1e-14;
                    double ca = dot(vab, vcb) / (std::sqrt(rab2) * std::sqrt(rcb2) + 1e-14);
                    ca = std::max(-1.0, std::min(1.0, ca));
                    const double th = std::acos(ca);
                    double ea, deddt;
                    if (M_PI - c0 < 1e-6) {
                        const double dt = th - c0;
                        ea = kijk * dt * dt;
                        deddt = 2.0 * kijk * dt;
                    } else {
                        ea = kijk * (ca - std::cos(c0)) * (ca - std::cos(c0));
                        deddt = 2.0 * kijk * std::sin(th) * (std::cos(c0) - ca);
                    }
                    eangl = 1.0 - ea;
                    V3 deda = (-deddt / (rab2 * rp)) * cross(vab, vp);
                    V3 dedc = (deddt / (rcb2 * rp)) * cross(vcb, vp);
                    ga3[0] = deda + dedc;
                    ga3[1] = -1.0 * deda;
                    ga3[2] = -1.0 * dedc;
                }
                for (int D : hb.nb_c) {
                    if (D == Bi) continue;
                    V3 g[4];
                    const double phi = dihedral(X(D), X(Bi), X(Ci), X(Hi), g);
                    const double fct = (1.0 - TORS_HB) / 2.0;
                    const double c1 = 2 * (phi - M_PI / 2.0) + M_PI;
                    const double et = (1.0 + std::cos(c1)) * fct + TORS_HB;
                    const double dij = -2 * std::sin(c1) * fct;
                    TG t;
                    t.e = et;
                    t.D = D;
                    for (int a = 0; a < 4; ++a) t.g[a] = dij * g[a];
                    tg.push_back(t);
                }
                etors = 1.0;
                for (auto& t : tg) etors *= t.e;
            }
            double gs = 1.0;
            if (hb.case_type == 2 || hb.case_type == 4) gs = XHACI_GLOBABH;
            else if (hb.case_type == 3) gs = XHACI_COH;
            double E;
            const double cst = hb.aci_a * hb.bas_b * QA * QB * gs;
            if (hb.case_type >= 2) E = -rdamp * qhoutl * cst * eangl * etors;
            else E = -bas * aci * rdamp * qhoutl;
            T[ORC_HBOND] += E;

            V3 drab = -1.0 * vAB, drah = -1.0 * vAH, drbh = vHB;
            const double rab2 = rAB * rAB, rbh2 = rHB * rHB, rah2 = rAH * rAH;
            const double rahprbh = rAH + rHB + 1e-12;
            const double ratio1 = std::pow(rab2 / HB_LONGCUT, HB_ALP);
            const double ratio3 = std::pow(HB_SCUT * rv / rab2, HB_ALP);
            const double ddamp = (-2.0 * HB_ALP * ratio1 / (1.0 + ratio1)) + (2.0 * HB_ALP * ratio3 / (1.0 + ratio3));
            const double expo = (HB_BACUT / rv) * (rahprbh / rAB - 1.0);
            if (expo > 15.0) continue;
            const double ratio2 = std::exp(expo);
            V3 ga{0, 0, 0}, gb{0, 0, 0}, gh{0, 0, 0};
            if (hb.case_type >= 2) {
                const double rbhdamp = denv * 1.8 / (rbh2 * rHB);
                const double rabdamp = denv * (-0.8) / (rab2 * rAB);
                const double dterm = -qhoutl * eangl * etors * cst;
                const double aterm = -rdamp * QH * onb * olp * eangl * etors * cst;
                const double nbterm = -rdamp * QH * doutl * olp * eangl * etors * cst;
                double gi = ((rabdamp + rbhdamp) * ddamp - 3.0 * rabdamp) / rab2;
                gi *= dterm;
                V3 dg = gi * drab;
                ga = dg;
                gb = -1.0 * dg;
                gi = -3.0 * rbhdamp / rbh2;
                gi *= dterm;
                dg = gi * drbh;
                gb = gb + dg;
                gh = -1.0 * dg;
                const double tmp1 = -2.0 * aterm * ratio2 * expo / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB);
                gi = -tmp1 * rahprbh / rab2;
                dg = gi * drab;
                ga = ga + dg;
                gb = gb - dg;
                V3 dgao = (tmp1 / rAH) * drah;
                ga = ga + dgao;
                V3 dgbo = (tmp1 / rHB) * drbh;
                gb = gb + dgbo;
                gh = gh - dgao - dgbo;
                const double cutg = (zB == 7 && hb.nb_b.size() == 1) ? 2.0 : HB_NBCUT;
                for (int nb : hb.nb_b) {
                    V3 pn = X(nb);
                    V3 dranb = pA - pn, drbnb = pB - pn;
                    const double ranb = norm(dranb), rbnb = norm(drbnb);
                    const double sum = ranb + rbnb + 1e-12;
                    const double ex = (cutg / rv) * (sum / rAB - 1.0);
                    const double r2n = std::exp(-ex);
                    const double oi = 2.0 / (1.0 + r2n) - 1.0;
                    double others = 1.0;
                    if (std::fabs(oi) > 1e-12) others = onb / oi;
                    const double tmp2 = 2.0 * nbterm * others * r2n * ex / ((1.0 + r2n) * (1.0 + r2n)) / (sum - rAB);
                    double gn = -tmp2 * sum / rab2;
                    dg = gn * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    V3 dgan = (tmp2 / ranb) * dranb, dgbn = (tmp2 / rbnb) * drbnb;
                    ga = ga + dgan;
                    gb = gb + dgbn;
                    G.add(nb, -1.0 * dgan - dgbn);
                }
                if (hb.case_type == 4 && nlp > 0) {
                    const double lpterm = -rdamp * QH * doutl * onb * cst;
                    const double ral = norm(pA - lpp);
                    const double sum = ral + lpd + 1e-12;
                    const double ex = (HBLPCUT / rv) * (sum / rAB - 1.0);
                    const double r2l = std::exp(ex);
                    const double tmp3 = -2.0 * lpterm * r2l * ex / ((1.0 + r2l) * (1.0 + r2l)) / (sum - rAB);
                    double gl = -tmp3 * sum / rab2;
                    V3 dgl = gl * drab;
                    ga = ga + dgl;
                    gb = gb - dgl;
                    V3 dral = pA - lpp;
                    gl = tmp3 / (ral + 1e-12);
                    V3 dgal = gl * dral;
                    ga = ga + dgal;
                    gb = gb - dgal;
                    V3 glp = -1.0 * dgal;
                    const double vn = norm(lpv);
                    if (vn > 1e-10) {
                        // gii(:,col) = -lpd*nlp*(e_col*(-1)/vn + lpv*lpv(col)/vn^3), gnb = gii*glp
                        double lv[3] = {lpv.x, lpv.y, lpv.z}, gl3[3] = {glp.x, glp.y, glp.z}, out[3] = {0, 0, 0};
                        const double vn3 = std::pow(vn, 3.0);
                        for (int col = 0; col < 3; ++col)
                            for (int row = 0; row < 3; ++row) {
                                const double unit = (row == col) ? -1.0 : 0.0;
                                const double gii = -lpd * (double)nlp * (unit / vn + lv[row] * lv[col] / vn3);
                                out[row] += gii * gl3[col];
                            }
                        V3 gnb{out[0], out[1], out[2]};
                        gb = gb + gnb;
                        V3 share = (1.0 / (double)nlp) * gnb;
                        for (int nb : hb.nb_b) G.add(nb, -1.0 * share);
                    }
                }
                if (hb.case_type == 3 && jj >= 0) {
                    const double bterm = -rdamp * qhoutl * etors * cst;
                    const double tterm = -rdamp * qhoutl * eangl * cst;
                    G.add(jj, bterm * ga3[0]);
                    G.add(kk, bterm * ga3[1]);
                    G.add(ll, bterm * ga3[2]);
                    for (auto& t : tg) {
                        const double fk = std::fabs(t.e) > 1e-12 ? etors / t.e : 0.0;
                        const double tk = fk * tterm;
                        G.add(t.D, tk * t.g[0]);
                        G.add(jj, tk * t.g[1]);
                        G.add(kk, tk * t.g[2]);
                        G.add(ll, tk * t.g[3]);
                    }
                }
            } else {
                const double caa = QA * hb.bas_a, cbb = QB * hb.bas_b;
                const double rterm = -aci * rdamp * qhoutl, dterm = -aci * bas * qhoutl;
                const double sterm = -rdamp * bas * qhoutl, aterm = -aci * bas * rdamp * QH;
                const double dv = 1.0 / (rAH4 + rHB4);
                const double tmp = dv * dv * 4.0;
                const double dd24a = rah2 * rHB4 * tmp, dd24b = rbh2 * rAH4 * tmp;
                double gi = (caa - cbb) * dd24a * rterm;
                ga = gi * drah;
                gi = (cbb - caa) * dd24b * rterm;
                gb = gi * drbh;
                gh = -1.0 * ga - gb;
                gi = (hb.aci_b - hb.aci_a) * dd24a;
                V3 dga = (gi * sterm) * drah;
                ga = ga + dga;
                gi = (hb.aci_a - hb.aci_b) * dd24b;
                V3 dgb = (gi * sterm) * drbh;
                gb = gb + dgb;
                gh = gh - dga - dgb;
                gi = rdamp * (ddamp - 3.0) / rab2;
                V3 dg = (gi * dterm) * drab;
                ga = ga + dg;
                gb = gb - dg;
                gi = aterm * 2.0 * ratio2 * expo * rahprbh / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB) / rab2;
                dg = gi * drab;
                ga = ga + dg;
                gb = gb - dg;
                const double to = -2.0 * aterm * ratio2 * expo / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB);
                V3 dgao = (to / rAH) * drah, dgbo = (to / rHB) * drbh;
                ga = ga + dgao;
                gb = gb + dgbo;
                gh = gh - dgao - dgbo;
            }
            G.add(hb.a, ga);
            G.add(hb.b, gb);
            G.add(hb.h, gh);
        }
    }

    // ---- halogen bonds: :1411-1524 --------------------------------------------------
    {
        const double XB_BACUT = 70.0, XB_SCUT = 5.0, HB_ALP = 6.0, LC = 70.0, XB_ST = 15.0, XB_SF = 0.03;
        auto qs = [&](double qq) { const double e = std::exp(XB_ST * qq); return e / (e + XB_SF); };
        for (const auto& xbd : m.xbonds) {
            V3 vAX = D(xbd.a, xbd.x), vXB = D(xbd.x, xbd.b), vAB = D(xbd.a, xbd.b);
            const double rAX = norm(vAX), rXB = norm(vXB), rAB = norm(vAB);
            if (rXB > 20.0) continue;
            const double rv = m.rvdw[xbd.a] + m.rvdw[xbd.b];
            const double dsh = 1.0 / (1.0 + std::pow(XB_SCUT * rv / (rXB * rXB), HB_ALP));
            const double dlg = 1.0 / (1.0 + std::pow(rXB * rXB / LC, HB_ALP));
            const double ex = XB_BACUT * ((rAX + rXB) / rAB - 1.0);
            if (ex > 15.0) continue;
            const double dol = 2.0 / (1.0 + std::exp(ex));
            const double QX = qs(xbd.q_x), QB = qs(-xbd.q_b);
            const double R = dsh * dlg * dol / (rXB * rXB * rXB);
            T[ORC_XBOND] += -R * QB * xbd.aci_x * QX;
            const double rs = XB_SCUT * rv / (rXB * rXB);
            const double st = std::pow(rs, HB_ALP);
            const double dds = -2.0 * HB_ALP * dsh * st / (rXB * (1.0 + st));
            const double rl = (rXB * rXB) / LC;
            const double lt = std::pow(rl, HB_ALP);
            const double ddl = -2.0 * HB_ALP * rXB * dlg * lt / (LC * (1.0 + lt));
            const double et = std::exp(ex), de = 1.0 + et;
            const double do_ax = -2.0 * et * XB_BACUT / (rAB * de * de);
            const double do_xb = do_ax;
            const double do_ab = 2.0 * et * XB_BACUT * (rAX + rXB) / (rAB * rAB * de * de);
            const double r3 = rXB * rXB * rXB;
            const double dR_xb = (dds * dlg * dol + dsh * ddl * dol + dsh * dlg * do_xb) / r3 - 3.0 * R / rXB;
            const double dR_ax = dsh * dlg * do_ax / r3, dR_ab = dsh * dlg * do_ab / r3;
            const double pre = -QB * xbd.aci_x * QX;
            const double eXB = pre * dR_xb, eAX = pre * dR_ax, eAB = pre * dR_ab;
            V3 uAX = (1.0 / (rAX + 1e-14)) * vAX, uXB = (1.0 / (rXB + 1e-14)) * vXB, uAB = (1.0 / (rAB + 1e-14)) * vAB;
            G.add(xbd.a, -eAX * uAX - eAB * uAB);
            G.add(xbd.x, eAX * uAX - eXB * uXB);
            G.add(xbd.b, eXB * uXB + eAB * uAB);
        }
    }

    // ---- ATM: :1526-1663 ------------------------------------------------------------
    for (const auto& t : m.atm) {
        V3 pi = X(t.i), pj = X(t.j), pk = X(t.k);
        V3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double rij = norm(vij), rik = norm(vik), rjk = norm(vjk);
        const double r2ij = rij * rij, r2ik = rik * rik, r2jk = rjk * rjk;
        const double c9 = std::sqrt(std::fabs(t.c6ij * t.c6ik * t.c6jk));
        auto rc = [&](int a) { return m.rcov_d3[a]; };
        const double r0ij = 0.58 * std::sqrt(3.0 * rc(t.i) * rc(t.j)) + 4.80;
        const double r0ik = 0.58 * std::sqrt(3.0 * rc(t.i) * rc(t.k)) + 4.80;
        const double r0jk = 0.58 * std::sqrt(3.0 * rc(t.j) * rc(t.k)) + 4.80;
        const double rijk = rij * rik * rjk, r2ijk = r2ij * r2ik * r2jk, r3ijk = rijk * r2ijk;
        const double tmp = std::pow(r0ij * r0ik * r0jk / rijk, 14.0 / 3.0);
        const double fdmp = 1.0 / (1.0 + 6.0 * tmp);
        const double A = r2ij + r2jk - r2ik, B = r2ij + r2ik - r2jk, C = r2ik + r2jk - r2ij;
        const double ang = (0.375 * A * B * C / r2ijk + 1.0) / r3ijk;
        T[ORC_ATM] += ang * fdmp * c9 / 3.0 * t.scale;
        const double r5ijk = r2ijk * r3ijk;
        const double dfdmp = -2.0 * 14.0 * tmp * fdmp * fdmp;
        auto P3 = [](double v) { return std::pow(v, 3); };
        auto P2 = [](double v) { return std::pow(v, 2); };
        const double dij = -0.375 * (P3(r2ij) + P2(r2ij) * (r2jk + r2ik) + r2ij * (3.0 * P2(r2jk) + 2.0 * r2jk * r2ik + 3.0 * P2(r2ik)) - 5.0 * P2(r2jk - r2ik) * (r2jk + r2ik)) / r5ijk;
        const double dik = -0.375 * (P3(r2ik) + P2(r2ik) * (r2jk + r2ij) + r2ik * (3.0 * P2(r2jk) + 2.0 * r2jk * r2ij + 3.0 * P2(r2ij)) - 5.0 * P2(r2jk - r2ij) * (r2jk + r2ij)) / r5ijk;
        const double djk = -0.375 * (P3(r2jk) + P2(r2jk) * (r2ik + r2ij) + r2jk * (3.0 * P2(r2ik) + 2.0 * r2ik * r2ij + 3.0 * P2(r2ij)) - 5.0 * P2(r2ik - r2ij) * (r2ik + r2ij)) / r5ijk;
        const double pre = -c9 * t.scale / 3.0;
        V3 gij = (pre * (-dij * fdmp + ang * dfdmp) / r2ij) * vij;
        V3 gik = (pre * (-dik * fdmp + ang * dfdmp) / r2ik) * vik;
        V3 gjk = (pre * (-djk * fdmp + ang * dfdmp) / r2jk) * vjk;
        G.add(t.i, -1.0 * (gij + gik));
        G.add(t.j, gij - gjk);
        G.add(t.k, gik + gjk);
    }

    // ---- BATM: :1665-1739 -----------------------------------------------------------
    for (const auto& b : m.batm) {
        V3 pi = X(b.i), pj = X(b.j), pk = X(b.k);
        V3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double r2ij = dot(vij, vij), r2jk = dot(vjk, vjk), r2ik = dot(vik, vik);
        const double rij = std::sqrt(r2ij), rjk = std::sqrt(r2jk), rik = std::sqrt(r2ik);
        const double rijk3 = r2ij * r2jk * r2ik;
        const double mijk = -r2ij + r2jk + r2ik, imjk = r2ij - r2jk + r2ik, ijmk = r2ij + r2jk - r2ik;
        const double ang = 0.375 * ijmk * imjk * mijk / rijk3;
        const double rav3 = std::pow(rijk3, 1.5);
        const double angr9 = (ang + 1.0) / rav3;
        auto fq = [&](int a) { return std::min(std::max(1.0 - 3.0 * m.qa[a], -4.0), 4.0); };
        const double c9 = fq(b.i) * fq(b.j) * fq(b.k) * b.zi * b.zj * b.zk;
        T[ORC_BATM] += c9 * angr9;
        auto P3 = [](double v) { return std::pow(v, 3); };
        auto P2 = [](double v) { return std::pow(v, 2); };
        const double dij = -0.375 * (P3(r2ij) + P2(r2ij) * (r2jk + r2ik) + r2ij * (3.0 * P2(r2jk) + 2.0 * r2jk * r2ik + 3.0 * P2(r2ik)) - 5.0 * P2(r2jk - r2ik) * (r2jk + r2ik)) / (rij * rijk3 * rav3);
        const double djk = -0.375 * (P3(r2jk) + P2(r2jk) * (r2ik + r2ij) + r2jk * (3.0 * P2(r2ik) + 2.0 * r2ik * r2ij + 3.0 * P2(r2ij)) - 5.0 * P2(r2ik - r2ij) * (r2ik + r2ij)) / (rjk * rijk3 * rav3);
        const double dik = -0.375 * (P3(r2ik) + P2(r2ik) * (r2jk + r2ij) + r2ik * (3.0 * P2(r2jk) + 2.0 * r2jk * r2ij + 3.0 * P2(r2ij)) - 5.0 * P2(r2jk - r2ij) * (r2jk + r2ij)) / (rik * rijk3 * rav3);
        V3 gij = (-dij * c9 / rij) * vij, gjk = (-djk * c9 / rjk) * vjk, gik = (-dik * c9 / rik) * vik;
        G.add(b.j, gjk - gij);
        G.add(b.k, -1.0 * gik - gjk);
        G.add(b.i, gij + gik);
    }

    // ---- triple-bond torsions: :611-653 ---------------------------------------------
    for (const auto& s : m.storsions) {
        V3 g[4];
        const double phi = dihedral(X(s.i), X(s.j), X(s.k), X(s.l), g);
        T[ORC_STORSION] += -s.erefhalf * std::cos(2.0 * phi) + s.erefhalf;
        const double dEdphi = 2.0 * s.erefhalf * std::sin(2.0 * phi);
        G.add(s.i, dEdphi * g[0]);
        G.add(s.j, dEdphi * g[1]);
        G.add(s.k, dEdphi * g[2]);
        G.add(s.l, dEdphi * g[3]);
    }

    // ---- post-process: ff_workspace.cpp:415-536 ------------------------------------
    if (n >= 2) {
        const double s2p = 0.797884560802865;
        double een = 0.0, eself = 0.0;
        for (int i = 0; i < n; ++i) {
            if (m.alpeeq[i] <= 0.0) continue;
            double chi = (m.cnf[i] != 0.0) ? m.chi_base[i] + m.cnf[i] * std::sqrt(std::max(cn[i], 0.0))
                                           : m.chi_base[i] + m.cnf[i] * std::sqrt(m.cn_setup[i]);
            een -= q[i] * chi;
            eself += 0.5 * q[i] * q[i] * (m.gam[i] + s2p / std::sqrt(m.alpeeq[i]));
        }
        T[ORC_COULOMB] += een + eself;
    }
    {
        std::vector<double> v(n);
        for (int i = 0; i < n; ++i) {
            const double qt = q[i] * m.cnf[i] / (2.0 * std::sqrt(std::max(cn[i], 0.0)) + 1e-16);
            v[i] = dEdcn[i] - qt;
        }
        const double sqrtpi = 1.77245385091;
        std::vector<double> dlog(n);
        for (int i = 0; i < n; ++i) dlog[i] = std::exp(cnmax) / (std::exp(cnmax) + std::exp(cnraw[i]));
        for (int i = 0; i < n; ++i)
            for (int j : nbr[i]) {
                if (j >= i) continue;
                V3 rv = D(i, j);
                const double r = std::sqrt(dot(rv, rv));
                const double rs = m.rcov_cn[i] + m.rcov_cn[j];
                const double dr = (r - rs) / rs;
                const double de = (kn / sqrtpi) * std::exp(-kn * kn * dr * dr) / rs;
                V3 comp = (de / r) * rv;
                // diag(i) -= dlog_i comp; diag(j) += dlog_j comp; pairs (i,j) -dlog_j comp,
                // (j,i) +dlog_i comp -- applied against v
                G.add(i, (-dlog[i] * v[i]) * comp);
                G.add(j, (dlog[j] * v[j]) * comp);
                G.add(i, (-dlog[j] * v[j]) * comp);
                G.add(j, (dlog[i] * v[i]) * comp);
            }
    }
    if (solv.on) T[ORC_SOLVATION] = alpb_energy_gradient(solv, xb, n, sg, q.data(), G.g.data());
    double tot = m.e0;
    for (int t = 0; t < ORC_TOTAL; ++t) tot += T[t];
    T[ORC_TOTAL] = tot;
    if (gout) std::copy(G.g.begin(), G.g.end(), gout);
    return 0;
}

extern "C" {

oracle_handle* oracle_create(int n, const int* Z, const double* xyz_ang, int charge)
{
    try {
        auto* h = new oracle_handle;
        h->m = build_model(n, Z, xyz_ang, charge);
        return h;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// a set-up that consults a topology cache file (<geometry>.topo.json) before Phase 1
oracle_handle* oracle_create_cached(int n, const int* Z, const double* xyz_ang, int charge, const char* topo_json)
{
    try {
        auto* h = new oracle_handle;
        h->m = build_model(n, Z, xyz_ang, charge, SetupOptions(), BuildLists(), topo_json);
        return h;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

int oracle_topo_cache_hit(oracle_handle* h) { return h && h->m.topo_cache_hit ? 1 : 0; }

// periodic cell: cell_ang[3*k + d] = component d of lattice vector k (Angstrom); NULL: none
int oracle_set_cell(oracle_handle* h, const double* cell_ang)
{
    if (!h) return 1;
    h->cell = OCell();
    if (!cell_ang) return 0;
    double* c = h->cell.h;
    for (int k = 0; k < 9; ++k) c[k] = cell_ang[k] * kAngToBohr;
    auto H = [&](int r, int col) { return c[3 * col + r]; };
    const double det = H(0, 0) * (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) - H(0, 1) * (H(1, 0) * H(2, 2) - H(1, 2) * H(2, 0)) +
                       H(0, 2) * (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0));
    if (!(std::fabs(det) > 1e-6)) {
        g_err = "singular cell";
        return 1;
    }
    // inverse = adjugate / det (cyclic cofactors), stored in the same column layout
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) {
            const int r1 = (col + 1) % 3, r2 = (col + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
            h->cell.hi[3 * col + r] = (H(r1, c1) * H(r2, c2) - H(r1, c2) * H(r2, c1)) / det;
        }
    h->cell.on = true;
    return 0;
}

// the model read from a parameter file (the product's set-up cache) instead of a fresh set-up
oracle_handle* oracle_create_from_parameters(const char* path)
{
    try {
        auto* h = new oracle_handle;
        h->m = load_parameters(path);
        return h;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void oracle_destroy(oracle_handle* h) { delete h; }

int oracle_set_solvent(oracle_handle* h, const char* solvent)
{
    if (!h) return 1;
    if (!alpb_setup(h->solv, h->m.Z, solvent ? solvent : "")) {
        g_err = std::string("unknown solvent: ") + (solvent ? solvent : "");
        return 1;
    }
    return 0;
}
const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_engrad(oracle_handle* h, const double* xyz_ang, double* terms, double* grad, double* q,
                  double* cn, int nthreads)
{
    if (!h || !xyz_ang || !terms) return 1;
#ifdef _OPENMP
    const int old = omp_get_max_threads();
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    std::vector<double> xb(3 * (size_t)h->m.n);
    for (size_t k = 0; k < xb.size(); ++k) xb[k] = xyz_ang[k] * kAngToBohr;
    int rc;
    try {
        rc = engrad(h->m, h->solv, h->cell, xb.data(), terms, grad, q, cn);
    } catch (const std::exception& e) {
        g_err = e.what();
        rc = 2;
    }
#ifdef _OPENMP
    omp_set_num_threads(old);
#endif
    return rc;
}

int oracle_refresh_topology(oracle_handle* h, const double* xyz_ang)
{
    if (!h) return -1;
    std::vector<double> xb(3 * (size_t)h->m.n);
    for (size_t k = 0; k < xb.size(); ++k) xb[k] = xyz_ang[k] * kAngToBohr;
    return refresh_topology(h->m, xb.data()) ? 1 : 0;
}

int oracle_redetect_hbxb(oracle_handle* h, const double* xyz_ang)
{
    if (!h) return 1;
    std::vector<double> xb(3 * (size_t)h->m.n);
    for (size_t k = 0; k < xb.size(); ++k) xb[k] = xyz_ang[k] * kAngToBohr;
    redetect_hbxb(h->m, xb.data());
    return 0;
}

long oracle_list(oracle_handle* h, int kind, int* out, long cap)
{
    if (!h) return -1;
    const Model& m = h->m;
    std::vector<int> v;
    long cnt = 0;
    switch (kind) {
        case 0: for (auto& b : m.bonds) { v.push_back(b.i); v.push_back(b.j); } cnt = m.bonds.size(); break;
        case 1: for (auto& a : m.angles) { v.insert(v.end(), {a.i, a.j, a.k}); } cnt = m.angles.size(); break;
        case 2: for (auto& t : m.torsions) { v.insert(v.end(), {t.i, t.j, t.k, t.l}); } cnt = m.torsions.size(); break;
        case 3: for (auto& t : m.inversions) { v.insert(v.end(), {t.i, t.j, t.k, t.l}); } cnt = m.inversions.size(); break;
        case 4: for (auto& d : m.disp) { v.push_back(d.i); v.push_back(d.j); } cnt = m.disp.size(); break;
        case 5: for (auto& r : m.rep_nonbonded) { v.push_back(r.i); v.push_back(r.j); } cnt = m.rep_nonbonded.size(); break;
        case 6: for (auto& hb : m.hbonds) { v.insert(v.end(), {hb.a, hb.h, hb.b, hb.case_type}); } cnt = m.hbonds.size(); break;
        case 7: for (auto& x : m.xbonds) { v.insert(v.end(), {x.a, x.x, x.b}); } cnt = m.xbonds.size(); break;
        case 8: v = m.hyb; cnt = m.n; break;
        case 9: v = m.frag; cnt = m.n; break;
        case 10: v = m.pi_frag; cnt = m.n; break;
        case 11: for (auto& r : m.rep_bonded) { v.push_back(r.i); v.push_back(r.j); } cnt = m.rep_bonded.size(); break;
        case 12: for (auto& t : m.atm) { v.insert(v.end(), {t.i, t.j, t.k}); } cnt = m.atm.size(); break;
        case 13: for (auto& t : m.batm) { v.insert(v.end(), {t.i, t.j, t.k}); } cnt = m.batm.size(); break;
        default: return -1;
    }
    if (out) std::copy(v.begin(), v.begin() + std::min<long>((long)v.size(), cap), out);
    return cnt;
}

int oracle_atom_data(oracle_handle* h, int which, double* out)
{
    if (!h || !out) return 1;
    const Model& m = h->m;
    const std::vector<double>* src = nullptr;
    switch (which) {
        case 0: src = &m.qa; break;
        case 1: src = &m.cn_setup; break;
        case 2: src = &m.alpeeq; break;
        case 3: src = &m.gam; break;
        case 4: src = &m.chi_base; break;
        case 5: src = &m.cnf; break;
        case 6:   // target charge of the atom's fragment
            for (int i = 0; i < m.n; ++i) out[i] = m.qfrag[m.frag[i]];
            return 0;
        default: return 1;
    }
    std::copy(src->begin(), src->end(), out);
    return 0;
}

int oracle_nfrag(oracle_handle* h) { return h ? h->m.nfrag : -1; }

long oracle_term_params(oracle_handle* h, int kind, double* out, long cap)
{
    if (!h) return -1;
    const Model& m = h->m;
    std::vector<double> v;
    if (kind == 0) {
        for (const auto& b : m.bonds) v.insert(v.end(), {(double)b.i, (double)b.j, b.fc, b.alpha, b.r0_setup, b.rabshift, b.ff});
    } else if (kind == 1) {
        for (const auto& a : m.angles) v.insert(v.end(), {(double)a.i, (double)a.j, (double)a.k, a.fc, a.theta0});
    } else if (kind == 2) {
        for (int t = 0; t < (int)m.torsions.size(); ++t) {
            const auto& q = m.torsions[t];
            v.insert(v.end(), {(double)q.i, (double)q.j, (double)q.k, (double)q.l, q.V, q.n, q.phi0,
                               t < m.n_primary_torsions ? 1.0 : 0.0});
        }
    } else if (kind == 3) {
        for (const auto& q : m.inversions) v.insert(v.end(), {(double)q.i, (double)q.j, (double)q.k, (double)q.l, q.fc, q.omega0, (double)q.type});
    } else {
        return -1;
    }
    const int width = kind == 0 ? 7 : (kind == 1 ? 5 : (kind == 2 ? 8 : 7));
    if (out) std::copy(v.begin(), v.begin() + std::min<long>(cap, (long)v.size()), out);
    return (long)v.size() / width;
}

}  // extern "C"
