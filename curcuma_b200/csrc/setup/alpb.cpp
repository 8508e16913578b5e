// ALPB set-up: solvent parameters, per-atom radii and surface data, Lebedev grid.
#include "alpb.h"

#include <algorithm>
#include <cctype>
#include <cmath>

#include "../tables/alpb_tables.inc"

namespace gfnff {

// Points of one octahedral orbit of the Lebedev-Laikov construction (Lebedev & Laikov,
// Doklady Math. 59 (1999) 477): type 1 the six vertices (+-1, 0, 0); type 3 the eight
// (+-a, +-a, +-a) with a = 1/sqrt 3; type 4 the 24 permutations of (+-a, +-a, +-b) with
// b = sqrt(1 - 2a^2); type 5 the 24 of (+-a, +-b, 0) with b = sqrt(1 - a^2); type 6 the 48 of
// (+-a, +-b, +-c) with c = sqrt(1 - a^2 - b^2).  Every point carries the orbit's weight v.
static void orbit(int type, double a, double b, double v, std::vector<double>& x, std::vector<double>& w)
{
    auto put = [&](double p, double q, double r) {
        x.push_back(p);
        x.push_back(q);
        x.push_back(r);
        w.push_back(v);
    };
    const double sg[2] = {1.0, -1.0};
    switch (type) {
        case 1:
            for (int d = 0; d < 3; ++d)
                for (double s : sg) put(d == 0 ? s : 0.0, d == 1 ? s : 0.0, d == 2 ? s : 0.0);
            break;
        case 3: {
            const double c = std::sqrt(1.0 / 3.0);
            for (double s0 : sg)
                for (double s1 : sg)
                    for (double s2 : sg) put(s0 * c, s1 * c, s2 * c);
            break;
        }
        case 4: {
            const double c = std::sqrt(1.0 - 2.0 * a * a);
            const double t[3][3] = {{a, a, c}, {a, c, a}, {c, a, a}};
            for (const auto& p : t)
                for (double s0 : sg)
                    for (double s1 : sg)
                        for (double s2 : sg) put(s0 * p[0], s1 * p[1], s2 * p[2]);
            break;
        }
        case 5: {
            const double c = std::sqrt(1.0 - a * a);
            const double t[6][3] = {{a, c, 0}, {c, a, 0}, {a, 0, c}, {c, 0, a}, {0, a, c}, {0, c, a}};
            for (const auto& p : t)
                for (double s0 : sg)
                    for (double s1 : sg) {
                        double q[3] = {p[0], p[1], p[2]};
                        int k = 0;
                        for (int d = 0; d < 3; ++d)
                            if (q[d] != 0.0) q[d] *= (k++ == 0 ? s0 : s1);
                        put(q[0], q[1], q[2]);
                    }
            break;
        }
        case 6: {
            const double c = std::sqrt(1.0 - a * a - b * b);
            const double t[6][3] = {{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a}, {c, a, b}, {c, b, a}};
            for (const auto& p : t)
                for (double s0 : sg)
                    for (double s1 : sg)
                        for (double s2 : sg) put(s0 * p[0], s1 * p[1], s2 * p[2]);
            break;
        }
        default:
            break;
    }
}

void lebedev230(std::vector<double>& xyz, std::vector<double>& w)
{
    xyz.clear();
    w.clear();
    for (const auto& o : alpb_tables::lebedev230) orbit(o.type, o.a, o.b, o.v, xyz, w);
}

static int find_solvent(const std::string& name)
{
    std::string s = name;
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    for (const auto& a : alpb_tables::aliases)
        if (s == a.name) return a.solvent;
    return -1;
}

// alpb_solvation.cpp:196-396 (init, loadSolventParameters for GFN-FF, setupRadii)
bool alpb_setup(AlpbModel& m, const std::vector<int>& Z, const std::string& solvent)
{
    m = AlpbModel();
    if (solvent.empty() || solvent == "none") return true;
    const int si = find_solvent(solvent);
    if (si < 0) return false;
    const auto& p = alpb_tables::solvents[si];
    using namespace alpb;
    m.on = true;
    m.solvent = p.name;
    m.epsv = p.epsv;
    m.gshift = p.gshift * kKcalToAu;
    m.born_scale = p.c1;
    m.born_offset = p.soset * 0.1 * kAngToAu;
    m.probe = p.rprobe * kAngToAu;
    m.alpbet = kAlpbFactor / p.epsv;   // GFN-FF always uses the ALPB shape term
    m.keps = (1.0 / p.epsv - 1.0) / (1.0 + m.alpbet);
    const int n = (int)Z.size();
    m.vdwr.resize(n); m.rho.resize(n); m.svdw.resize(n); m.vdwsa.resize(n);
    m.trj2_lo.resize(n); m.trj2_hi.resize(n); m.wrp.resize(n); m.gamsasa.resize(n); m.hbmag.resize(n);
    double vmax = 0.0;
    for (int i = 0; i < n; ++i) {
        const int z = Z[i];
        const bool known = z >= 1 && z <= 94;
        m.vdwr[i] = known ? alpb_tables::vdw_rad_d3_ang[z - 1] * kAngToAu : 2.0 * kAngToAu;
        m.rho[i] = m.vdwr[i] * (known ? p.sx[z - 1] : 0.8);
        m.svdw[i] = m.vdwr[i] - m.born_offset;
        m.vdwsa[i] = m.vdwr[i] + m.probe;
        m.trj2_lo[i] = (m.vdwsa[i] - kWSmooth) * (m.vdwsa[i] - kWSmooth);
        m.trj2_hi[i] = (m.vdwsa[i] + kWSmooth) * (m.vdwsa[i] + kWSmooth);
        // radial weight of the smoothed surface (alpb_solvation.cpp:378-386)
        double r = m.vdwsa[i] + kWSmooth;
        const double w1 = (0.25 / kWSmooth + 3.0 * kAh3 * (0.2 * r * r - 0.5 * r * m.vdwsa[i] +
                                                           m.vdwsa[i] * m.vdwsa[i] / 3.0)) * r * r * r;
        r = m.vdwsa[i] - kWSmooth;
        const double w2 = (0.25 / kWSmooth + 3.0 * kAh3 * (0.2 * r * r - 0.5 * r * m.vdwsa[i] +
                                                           m.vdwsa[i] * m.vdwsa[i] / 3.0)) * r * r * r;
        m.wrp[i] = w1 - w2;
        m.gamsasa[i] = known ? p.gamscale[z - 1] * 4.0 * kPi * kSurfaceTension : 0.0;
        const double t = known ? p.tmp[z - 1] : 0.0;
        m.hbmag[i] = std::fabs(t) > 1.0e-3 ? -(t * t) * kKcalToAu : 0.0;
        if (m.hbmag[i] < 0.0) m.lhb = true;
        vmax = std::max(vmax, m.vdwsa[i]);
    }
    m.srcut = 2.0 * (kWSmooth + vmax) + kROffset;
    lebedev230(m.grid, m.weight);
    return true;
}

}  // namespace gfnff
