// GFN-FF setup, part 2: the parameter generators for every energy term and the HB/XB
// detection.  Each generator cites the curcuma routine it restates (paths relative to
// src/core/energy_calculators/).
#include "setup_internal.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <set>
#include <stdexcept>
#include <tuple>

namespace gfnff {
namespace detail {

using namespace gfnff_tables;

static int table_row(int z)
{
    if (z <= 0) return 0;
    if (z <= 2) return 1;
    if (z <= 10) return 2;
    if (z <= 18) return 3;
    if (z <= 36) return 4;
    if (z <= 54) return 5;
    return 6;
}

// ---------------------------------------------------------------------------------
// Bonds: ff_methods/gfnff_method.cpp:7557-7608 (generateBondsNative) and
// :4184-5082 (getGFNFFBondParameters)
// ---------------------------------------------------------------------------------
static BondTerm make_bond_term(const Ctx& c, int a1, int a2, const std::vector<int>& nb20)
{
    const Model& m = c.m;
    const int z1 = c.Z[a1], z2 = c.Z[a2];
    const double bp1 = bond_params[z1 - 1], bp2 = bond_params[z2 - 1];
    const double cn1 = m.cn_setup[a1], cn2 = m.cn_setup[a2];
    const double r01 = r0_gfnff[z1 - 1], r02 = r0_gfnff[z2 - 1];
    const double ck1 = cnfak_gfnff[z1 - 1], ck2 = cnfak_gfnff[z2 - 1];
    const double ra = r01 + ck1 * cn1, rb = r02 + ck2 * cn2;
    const double en1 = en_rab_gfnff[z1 - 1], en2 = en_rab_gfnff[z2 - 1];
    const int row1 = table_row(z1), row2 = table_row(z2);
    const double k1 = 0.005 * (p_enpoly[(row1 - 1) * 2] + p_enpoly[(row2 - 1) * 2]);
    const double k2 = 0.005 * (p_enpoly[(row1 - 1) * 2 + 1] + p_enpoly[(row2 - 1) * 2 + 1]);
    const double den = std::fabs(en1 - en2);
    const double ff = 1.0 - k1 * den - k2 * den * den;

    const double gen_rabshift = -0.110, gen_rabshifth = -0.050, hyper_shift = 0.030;
    const double hshift3 = -0.110, hshift4 = -0.110, hshift5 = -0.060;
    double shift = 0.0;
    const int h1v = m.hyb[a1], h2v = m.hyb[a2];
    const int mh1 = (h1v < 1 || h1v > 3) ? 3 : h1v;
    const int mh2 = (h2v < 1 || h2v > 3) ? 3 : h2v;
    int hybi = std::max(mh1, mh2), hybj = std::min(mh1, mh2);
    int bbtyp = 1;
    if (hybi == 5 || hybj == 5) bbtyp = 4;
    else if (hybi == 1 || hybj == 1) bbtyp = 3;
    else if (hybi == 2 && hybj == 2) bbtyp = 2;
    else if (hybi == 3 && hybj == 2 && (z1 == 7 || z2 == 7)) bbtyp = 2;
    if (bbtyp == 4) shift = hyper_shift;
    else if (z1 == 1 || z2 == 1) shift = gen_rabshifth;
    if (z1 == 9 && z2 == 9) shift += 0.22;
    if ((h1v == 3 && h2v == 0) || (h1v == 0 && h2v == 3)) shift -= 0.022;
    if ((h1v == 1 && h2v == 0) || (h1v == 0 && h2v == 1)) shift += 0.14;
    if (z1 > 10 && z2 > 10) {
        shift += hshift3;
        if (z1 > 18) shift += hshift4;
        if (z2 > 18) shift += hshift4;
        if (z1 > 36) shift += hshift5;
        if (z2 > 36) shift += hshift5;
    }
    const double rabshift = gen_rabshift + shift;

    const int hyb1 = m.hyb[a1], hyb2 = m.hyb[a2];
    const int mi = (hyb1 < 1 || hyb1 > 3) ? 3 : hyb1;
    const int mj = (hyb2 < 1 || hyb2 > 3) ? 3 : hyb2;
    hybi = std::max(mi, mj);
    hybj = std::min(mi, mj);
    double bstrength;
    if (z1 == 1 && z2 == 1) bstrength = bstren[1];
    else if (hybi == 5 || hybj == 5) bstrength = bstren[4];
    else bstrength = bsmat[hybi * 4 + hybj];
    if (hybi == 3 && hybj == 2 && (z1 == 7 || z2 == 7)) bstrength = bstren[2] * 1.04;
    if (bbtyp == 3 && ((z1 == 6 && z2 == 8) || (z1 == 8 && z2 == 6))) bstrength = bstren[3] * 0.90;
    if (bbtyp == 3) {
        if (hyb1 == 0 || hyb2 == 0) bbtyp = 1;
        else if (hyb1 == 3 || hyb2 == 3) bbtyp = 1;
        else if (hyb1 == 2 || hyb2 == 2) bbtyp = 2;
    }
    {
        const int g1 = periodic_group[z1 - 1], g2 = periodic_group[z2 - 1];
        bool bridge = false;
        if ((g1 == 7 || z1 == 1) && h1v == 1) { bbtyp = 3; bridge = true; }
        if ((g2 == 7 || z2 == 1) && h2v == 1) { bbtyp = 3; bridge = true; }
        if (bridge) {
            if (g1 == 7) bstrength = bstren[1] * 0.50;
            if (g2 == 7) bstrength = bstren[1] * 0.50;
            if (z1 == 1 || z1 == 9) bstrength = bstren[1] * 0.30;
            if (z2 == 1 || z2 == 9) bstrength = bstren[1] * 0.30;
        }
    }
    const double qa1 = m.qa[a1], qa2 = m.qa[a2];
    const double qafac = qa1 * qa2 * 70.0;
    const double ex = std::exp(-15.0 * qafac);
    const double fqq = 1.0 + 0.047 * ex / (1.0 + ex);
    double ringf = 1.0;
    {
        const int rs = same_ring_size(c, a1, a2);
        if (rs > 0) ringf = 1.0 + 0.020 * std::pow(6.0 - rs, 2);
    }
    double fxh = 1.0;
    if (z1 == 1 || z2 == 1) {
        const int heavy = (z1 == 1) ? z2 : z1;
        const int hidx = (z1 == 1) ? a2 : a1;
        bool ring3 = (heavy == 6 && m.ring_size[hidx] == 3);
        bool ald = false;
        if (heavy == 6 && m.pi_frag[hidx] > 0) {
            int npo = 0;
            for (int nb : m.adj[hidx]) if (c.Z[nb] == 8 && m.pi_frag[nb] > 0) ++npo;
            ald = (npo == 1);
        }
        if (heavy == 6 && ring3) fxh = 1.05;
        else if (heavy == 6 && ald) fxh = 0.95;
        else if (heavy == 5) fxh = 1.10;
        else if (heavy == 7) fxh = 1.06;
        else if (heavy == 8) fxh = 0.93;
    }
    double fcn = 1.0;
    const int n20a = nb20.empty() ? 0 : nb20[a1], n20b = nb20.empty() ? 0 : nb20[a2];
    if (z1 > 10 && z2 > 10) {
        fcn /= (1.0 + 0.007 * n20a * n20a);
        fcn /= (1.0 + 0.007 * n20b * n20b);
    }
    double fheavy = 1.0, fpi = 1.0, metal_shift = 0.0, pi_shift = 0.0;
    const double pibo = pibo_of(c, a1, a2);
    if (pibo > 0.0) {
        pi_shift = 0.340 * (0.370 - pibo);
        fpi = 1.0 - 1.00 * (0.315 - pibo);
        if (bbtyp != 3 && pibo > 0.1) bbtyp = 2;
    }
    const int im1 = metal_type[z1 - 1], im2 = metal_type[z2 - 1];
    const int g1 = periodic_group[z1 - 1], g2 = periodic_group[z2 - 1];
    int mt1 = 0, mt2 = 0;
    if (z1 > 1 && g1 == 1) mt1 = 1;
    else if (z1 > 1 && g1 == 2) mt1 = 2;
    else if (g1 > 2 && im1 == 1) mt1 = 3;
    else if (im1 == 2) mt1 = 4;
    if (z2 > 1 && g2 == 1) mt2 = 1;
    else if (z2 > 1 && g2 == 2) mt2 = 2;
    else if (g2 > 2 && im2 == 1) mt2 = 3;
    else if (im2 == 2) mt2 = 4;
    if (mt1 == 4 || mt2 == 4) {
        if (im1 == 2 && z2 > 10) fheavy = 0.65;
        if (im2 == 2 && z1 > 10) fheavy = 0.65;
        if (im1 == 2 && z2 == 15) fheavy = 1.60;
        if (im2 == 2 && z1 == 15) fheavy = 1.60;
        if (im1 == 2 && g2 == 6) fheavy = 0.85;
        if (im2 == 2 && g1 == 6) fheavy = 0.85;
        if (im1 == 2 && g2 == 7) fheavy = 1.30;
        if (im2 == 2 && g1 == 7) fheavy = 1.30;
        if (im2 == 2 && hyb1 == 1) {
            if (z1 == 6) { fpi = 1.5; metal_shift = -0.45; }
            if (z1 == 7 && n20a != 1) { fpi = 0.4; metal_shift = 0.47; }
        }
        if (im1 == 2 && hyb2 == 1) {
            if (z2 == 6) { fpi = 1.5; metal_shift = -0.45; }
            if (z2 == 7 && n20b != 1) { fpi = 0.4; metal_shift = 0.47; }
        }
        if (im1 == 2 && z2 == 1) fxh = (row1 <= 5) ? 0.80 : 1.00;
        if (im2 == 2 && z1 == 1) fxh = (row2 <= 5) ? 0.80 : 1.00;
    }
    if ((im1 == 1 && z2 == 1) || (im2 == 1 && z1 == 1)) fxh = 1.20;
    if (im1 == 2) metal_shift += 0.15;
    if (im2 == 2) metal_shift += 0.15;
    if (im1 == 1 && g1 <= 2) metal_shift += 0.2;
    if (im2 == 1 && g2 <= 2) metal_shift += 0.2;
    if (mt1 == 3) metal_shift += 0.05;
    if (mt2 == 3) metal_shift += 0.05;
    const double total_shift = rabshift + pi_shift + metal_shift;

    BondTerm b;
    b.i = a1;
    b.j = a2;
    b.r0_setup = (ra + rb + total_shift) * ff;
    b.rabshift = total_shift;
    b.fc = -(bp1 * bp2 * bstrength * fqq * ringf * fheavy * fpi * fxh * fcn);
    const double srb1 = 0.3731, srb2 = 0.3171, srb3 = 0.2538;
    double fsrb2;
    if (mt1 == 4 || mt2 == 4) fsrb2 = -srb2 * 0.22;
    else if (mt1 > 0 || mt2 > 0) fsrb2 = srb2 * 0.28;
    else fsrb2 = srb2;
    const double dena = std::fabs(en_gfnff[z1 - 1] - en_gfnff[z2 - 1]);
    const double t1 = fsrb2 * dena * dena;
    const double t2 = srb3 * bstrength;
    b.alpha = srb1 * (1.0 + t1 + t2);
    b.r0_base_i = r01;
    b.r0_base_j = r02;
    b.cnfak_i = ck1;
    b.cnfak_j = ck2;
    b.ff = ff;
    return b;
}

static void generate_bonds(Ctx& c)
{
    const int n = c.n;
    std::vector<double> rc(n);
    double rmax = 0.0;
    bool heavy = false;
    for (int i = 0; i < n; ++i) {
        rc[i] = covalent_radii[c.Z[i] - 1] * kAngToBohr;
        rmax = std::max(rmax, rc[i]);
        heavy |= c.Z[i] > 10;
    }
    // neighbour counts within 20 bohr (gfnff_method.cpp:7320-7349), only consulted for
    // bonds between two heavy atoms or transition-metal bonds
    std::vector<int> nb20;
    if (heavy) {
        nb20.assign(n, 0);
        pairs_within(c, 20.0, true, [&](int i, int j, double) { ++nb20[i]; ++nb20[j]; });
    }
    std::vector<std::pair<int, int>> pl;
    pairs_within(c, 1.3 * 2.0 * rmax + 1e-6, false, [&](int i, int j, double) {
        const double d = dist_bohr(c, i, j);
        if (d < 1.3 * (rc[i] + rc[j])) pl.push_back({i, j});
    });
    std::sort(pl.begin(), pl.end());
    c.m.bonds.clear();
    for (auto& p : pl) c.m.bonds.push_back(make_bond_term(c, p.first, p.second, nb20));
}

// ---------------------------------------------------------------------------------
// Angles: gfnff_method.cpp:7658-7744 (generateAnglesNative), :5083-5786
// (getGFNFFAngleParameters)
// ---------------------------------------------------------------------------------
static bool fg_carbonyl_on(const Ctx& c, int carbon)
{
    int cnt = 0;
    for (int nb : c.m.adj[carbon])
        if (c.Z[nb] == 8 && c.m.pi_frag[nb] != 0 && c.m.adj[nb].size() == 1) ++cnt;
    return cnt >= 1;
}

// functional_groups.cpp:112-139 (isAmideNitrogen)
static bool fg_amide_n(const Ctx& c, int a)
{
    if (c.Z[a] != 7 || c.m.hyb[a] != 3 || c.m.pi_frag[a] == 0) return false;
    if (c.m.adj[a].empty()) return false;
    int pic = 0, co = 0;
    for (int nb : c.m.adj[a])
        if (c.Z[nb] == 6 && c.m.pi_frag[nb] != 0) {
            ++pic;
            if (fg_carbonyl_on(c, nb)) ++co;
        }
    return pic == 1 && co == 1;
}

// functional_groups.cpp:141-166 (isAmideHydrogen)
static bool fg_amide_h(const Ctx& c, int a)
{
    if (c.Z[a] != 1 || c.m.adj[a].size() != 1) return false;
    const int nn = c.m.adj[a][0];
    if (!fg_amide_n(c, nn)) return false;
    int sp3 = 0;
    for (int nb : c.m.adj[nn]) if (c.Z[nb] == 6 && c.m.hyb[nb] == 3) ++sp3;
    return sp3 == 1;
}

static bool angle_term_params(const Ctx& c, int ai, int aj, int ak, double ang, double& fc, double& th0)
{
    const Model& m = c.m;
    const int zc = c.Z[aj], zi = c.Z[ai], zk = c.Z[ak];
    const int hyb_c = m.hyb[aj];
    const double fijk = angle_params[zc - 1] * angl2_neighbors[zi - 1] * angl2_neighbors[zk - 1];
    double fqq = 1.0;
    {
        const double qc = m.qa[aj], qi = m.qa[ai], qk = m.qa[ak];
        if (std::fabs(qc) < 1.0 && std::fabs(qi) < 1.0 && std::fabs(qk) < 1.0) {
            const double cp = qc * qi + qc * qk;
            const bool met = c.is_metal[ai] || c.is_metal[aj] || c.is_metal[ak];
            fqq = 1.0 - cp * (-0.54) * (met ? 2.5 : 1.0);
        }
    }
    double f2 = 1.0;
    int nh = 0, no = 0, nc = 0, nnn = 0, nsi = 0, nmet = 0, npi = 0;
    for (int a : {ai, ak}) {
        const int z = c.Z[a];
        if (z == 1) ++nh;
        if (z == 6) ++nc;
        if (z == 7) ++nnn;
        if (z == 8) ++no;
        if (z == 14) ++nsi;
        if (c.is_metal[a]) ++nmet;
        if (m.pi_frag[a] != 0) ++npi;
    }
    const int hyb = hyb_c;
    const int nn_c = (int)m.adj[aj].size();
    double nn = std::max(1.0, (double)nn_c);
    double fn = std::max(0.05, 1.0 - 2.36 / (nn * nn));
    double feta = 1.0;
    if (metal_type[zc - 1] == 2) {
        const int hi = m.hyb[ai], hk = m.hyb[ak];
        if (hi == 1 || hi == 2) feta *= 0.3;
        if (hk == 1 || hk == 2) feta *= 0.3;
    }
    double r0 = 100.0;
    switch (hyb_c) {
        case 1: r0 = 180.0; break;
        case 2: r0 = 120.0; break;
        case 3: r0 = 109.5; break;
        case 5: r0 = 90.0; break;
        default: r0 = 100.0;
    }
    const int gc = periodic_group[zc - 1];
    const double adeg = ang * 180.0 / M_PI;
    if (hyb_c == 3 && zc > 10) {
        if (nn_c <= 3) r0 = 89.0;
        if (nn_c >= 4) r0 = 100.0;
        if (nn_c == 4 && gc == 5) r0 = 109.5;
        if (nn_c == 4 && gc == 4 && zc > 49) r0 = 109.5;
        if (gc == 4) r0 = r0 - nh * 5.0;
        if (gc == 5) r0 = r0 - nh * 5.0;
        if (gc == 6) r0 = r0 - nh * 5.0;
    }
    bool co2 = false;
    if (hyb == 5) {
        f2 = 0.11;
        if (adeg > 160.0) r0 = 180.0;
    } else if (zc == 5) {
        if (hyb == 3 || hyb == 2) r0 = 115.0;
    } else if (zc == 6) {
        if (hyb == 3) {
            if (nh == 2) r0 = 108.6;
            if (no == 1) r0 = 108.5;
            if (nn_c > 4 && adeg > 160.0) r0 = 180.0;
        } else if (hyb == 2) {
            if (no == 2) r0 = 122.0;
            if (no == 1) f2 = 0.7;
        } else if (hyb == 1) {
            if (no == 2) { co2 = true; f2 = 2.0; }
        }
    } else if (zc == 7) {
        const int rc = smallest_ring_bend(c, aj, ai, ak);
        if (nn_c == 2) {
            f2 = 1.4;
            r0 = 115.0;
            if (rc != 0) r0 = 105.0;
            if (no >= 1) r0 = 103.0;
            int nf = (zi == 9) + (zk == 9);
            if (nf >= 1) r0 = 102.0;
            if (hyb == 1) r0 = 180.0;
            bool tmn = (c.is_metal[ai] && metal_type[zi - 1] == 2) ||
                       (c.is_metal[ak] && metal_type[zk - 1] == 2);
            if (tmn && hyb == 1 && nnn >= 1) r0 = 135.0;
        } else if (hyb == 3) {
            const int hi = m.hyb[ai], hk = m.hyb[ak];
            const bool sp2n = (hi == 1 || hi == 2 || hk == 1 || hk == 2);
            if (npi > 0 || sp2n) {
                if (fg_amide_n(c, aj)) {
                    r0 = 115.0;
                    f2 = 1.2;
                } else {
                    r0 = 113.0;
                    f2 = 1.0 - (pibo_of(c, aj, ai) + pibo_of(c, aj, ak)) * 0.7;
                }
            } else {
                r0 = 104.0;
                f2 = 0.40;
                f2 += nh * 0.19;
                f2 += no * 0.25;
                f2 += nc * 0.01;
            }
        }
    }
    const int rc = smallest_ring_bend(c, aj, ai, ak);
    if (rc == 3) r0 = 82.0;
    else if (rc == 4) r0 = 96.0;
    else if (rc == 5 && zc == 6) r0 = 109.0;
    if (rc == 0 && m.ring_size[aj] == 3) {
        const int ri = m.ring_size[ai], rk = m.ring_size[ak];
        if ((ri == 3 && rk == 0) || (ri == 0 && rk == 3)) r0 += 4.0;
    }
    const bool triple = !co2 && (hyb == 1 || m.hyb[ai] == 1 || m.hyb[ak] == 1);
    if (triple) {
        f2 = 0.60;
        if (nnn >= 1) f2 = 1.00;
        const int imi = metal_type[zi - 1], imk = metal_type[zk - 1];
        if ((imi == 2 || imk == 2) && adeg > 160.0) {
            if (zc == 6 && zi == 6) f2 = 3.0;
            if (zc == 6 && zk == 6) f2 = 3.0;
            if (zc == 6 && zi == 7) f2 = 3.0;
            if (zc == 6 && zk == 7) f2 = 3.0;
            const int gi = periodic_group[zi - 1], gk = periodic_group[zk - 1];
            if (zc == 6 && gi == 6) f2 = 14.0;
            if (zc == 6 && gk == 6) f2 = 14.0;
            if (zc == 7 && zi == 7) f2 = 10.0;
            if (zc == 7 && zi == 6) f2 = 10.0;
            if (zc == 7 && zk == 6) f2 = 10.0;
            if (zc == 7 && zi == 8) { r0 = 180.0; f2 = 12.0; }
            if (zc == 7 && zk == 8) { r0 = 180.0; f2 = 12.0; }
        }
    }
    if (gc == 6 && nn_c == 4 && no >= 1) r0 = 115.0;
    if (gc == 7 && hyb == 1) {
        r0 = 90.0;
        if (zc > 9 && adeg > 160.0) r0 = 180.0;
        f2 = 0.6 / std::pow((double)zc, 0.15);
    }
    if (hyb == 3 && gc == 4 && zc > 32) {
        if (m.qa[aj] > 0.4) {
            if (adeg > 140.0) r0 = 180.0;
            if (adeg < 100.0) r0 = 90.0;
            f2 = 1.0;
        }
    }
    if (metal_type[zc - 1] > 0) {
        if (hyb == 0) { r0 = 90.0; f2 = 1.35; }
        if (hyb == 1) r0 = 180.0;
        if (hyb == 2) r0 = 120.0;
        if (hyb == 3) r0 = 109.5;
        if (adeg > 160.0) r0 = 180.0;
    }
    if (zc == 8 && m.adj[aj].size() == 2) {
        r0 = 104.5;
        if (nh == 2) { r0 = 100.0; f2 = 1.20; }
        r0 = r0 + 7.0 * nsi;
        r0 = r0 + 14.0 * nmet;
        if (npi == 2) r0 = 109.0;
        if (nmet > 0 && adeg > 160.0) { r0 = 180.0; f2 = 0.3; }
    }
    th0 = r0 * M_PI / 180.0;
    const double fbsmall = 1.0 - 0.50 * std::exp(-0.64 * (th0 - M_PI) * (th0 - M_PI));
    if (fijk < 0.001) fc = 0.0;
    else fc = fijk * fqq * f2 * fn * fbsmall * feta;
    return true;
}

static void generate_angles(Ctx& c)
{
    std::vector<AngleTerm> out;
    for (int j = 0; j < c.n; ++j) {
        const auto& nb = c.m.adj[j];
        if (nb.size() <= 1 || nb.size() > 6) continue;
        for (size_t a = 0; a < nb.size(); ++a)
            for (size_t b = a + 1; b < nb.size(); ++b) {
                const int i = nb[a], k = nb[b];
                double v1[3], v2[3];
                for (int d = 0; d < 3; ++d) {
                    v1[d] = c.xb[3 * i + d] - c.xb[3 * j + d];
                    v2[d] = c.xb[3 * k + d] - c.xb[3 * j + d];
                }
                const double n1 = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
                const double n2 = std::sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
                if (n1 < 1e-10 || n2 < 1e-10) continue;
                double ca = (v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2]) / (n1 * n2);
                ca = std::max(-1.0, std::min(1.0, ca));
                const double ang = std::acos(ca);
                double fc, th0;
                angle_term_params(c, i, j, k, ang, fc, th0);
                if (fc < 1e-10) continue;
                const int zc = c.Z[j];
                if (metal_type[zc - 1] > 0 && ang * 180.0 / M_PI < 60.0) continue;
                out.push_back({i, j, k, fc, th0});
            }
    }
    std::sort(out.begin(), out.end(), [](const AngleTerm& a, const AngleTerm& b) {
        if (a.j != b.j) return a.j < b.j;
        if (a.i != b.i) return a.i < b.i;
        return a.k < b.k;
    });
    c.m.angles = out;
}

// ---------------------------------------------------------------------------------
// Torsions: ff_methods/gfnff_torsions.cpp:1561-2049 (generateTorsionsNative) and
// :510-1234 (getGFNFFTorsionParameters)
// ---------------------------------------------------------------------------------
static double dihedral_ang(const Ctx& c, int i, int j, int k, int l)
{   // gfnff_torsions.cpp:108-173 (Angstrom geometry)
    const double* x = c.xa.data();
    double v1[3], v2[3], v3[3];
    for (int d = 0; d < 3; ++d) {
        v1[d] = x[3 * j + d] - x[3 * i + d];
        v2[d] = x[3 * k + d] - x[3 * j + d];
        v3[d] = x[3 * l + d] - x[3 * k + d];
    }
    double n1[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
    double n2[3] = {v2[1] * v3[2] - v2[2] * v3[1], v2[2] * v3[0] - v2[0] * v3[2], v2[0] * v3[1] - v2[1] * v3[0]};
    const double a = std::sqrt(n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]);
    const double b = std::sqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
    const double v = std::sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
    if (a < 1e-10 || b < 1e-10 || v < 1e-10) return 0.0;
    for (int d = 0; d < 3; ++d) { n1[d] /= a; n2[d] /= b; }
    const double cphi = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    const double sphi = v * (n1[0] * v3[0] + n1[1] * v3[1] + n1[2] * v3[2]);
    return std::atan2(sphi, cphi);
}

static bool tors_terminal_co(const Ctx& c, int cc)
{   // gfnff_torsions.cpp:339-357
    int no = 0;
    for (int j : c.m.adj[cc])
        if (c.Z[j] == 8 && c.m.pi_frag[j] != 0 && c.m.adj[j].size() == 1) ++no;
    return no == 1;
}
static bool tors_alpha_co(const Ctx& c, int a, int b)
{   // :364-383
    auto pi = [&](int x) { return c.m.pi_frag[x] != 0; };
    if (pi(a) && c.m.hyb[b] == 3 && c.Z[a] == 6 && c.Z[b] == 6 && tors_terminal_co(c, a)) return true;
    if (pi(b) && c.m.hyb[a] == 3 && c.Z[b] == 6 && c.Z[a] == 6 && tors_terminal_co(c, b)) return true;
    return false;
}
static bool tors_amide(const Ctx& c, int a)
{   // :425-454
    if (c.m.pi_frag[a] == 0 || c.m.hyb[a] != 3 || c.Z[a] != 7) return false;
    int nc = 0, ic = -1;
    for (int j : c.m.adj[a])
        if (c.Z[j] == 6 && c.m.pi_frag[j] != 0) { ++nc; ic = j; }
    return nc == 1 && tors_terminal_co(c, ic);
}

struct TorsParams { double V = 0.0, fij = 0.0, fkl = 0.0, fqq = 1.0; int n = 1; double phi0 = M_PI; };

static TorsParams torsion_params(const Ctx& c, int ia, int ja, int ka, int la, int btyp,
                                 bool in_ring, int ring_size)
{
    const Model& m = c.m;
    TorsParams p;
    const int zi = c.Z[ia], zj = c.Z[ja], zk = c.Z[ka], zl = c.Z[la];
    const int hyb_j = m.hyb[ja], hyb_k = m.hyb[ka];
    const double qa_j = m.qa[ja], qa_k = m.qa[ka];
    const double cn_i = (double)m.adj[ia].size(), cn_l = (double)m.adj[la].size();
    const bool jpi = m.pi_frag[ja] > 0, kpi = m.pi_frag[ka] > 0;
    if (jpi && kpi) { p.n = 2; p.phi0 = M_PI; }
    else if (hyb_j == 3 && hyb_k == 3) { p.n = 3; p.phi0 = M_PI; }
    else if (hyb_j == 2 && hyb_k == 2) { p.n = 2; p.phi0 = M_PI; }
    else if ((hyb_j == 2 && hyb_k == 3) || (hyb_j == 3 && hyb_k == 2)) { p.n = 3; p.phi0 = M_PI; }
    else { p.n = 1; p.phi0 = M_PI; }
    const double fcthr = 1.0e-3;
    double fij = tors_angewChem2020[zj - 1] * tors_angewChem2020[zk - 1];
    if (fij < fcthr || tors_angewChem2020[zj - 1] < 0.0 || tors_angewChem2020[zk - 1] < 0.0) return p;
    const double fkl_base = tors2_angewChem2020[zi - 1] * tors2_angewChem2020[zl - 1];
    double fkl = fkl_base;
    const int hyb_i = m.hyb[ia], hyb_l = m.hyb[la];
    auto n_not_pi = [&](int a, int z) {
        if (z != 7) return false;
        for (int nb : m.adj[a]) if (pibo_of(c, a, nb) > 0.1) return false;
        for (int nb : m.adj[a]) if (m.hyb[nb] == 1 || m.hyb[nb] == 2) return false;
        return true;
    };
    if (n_not_pi(ia, zi)) fkl = fkl_base * 0.5;
    if (n_not_pi(la, zl)) fkl = fkl_base * 0.5;
    if (fkl < fcthr || tors_angewChem2020[zi - 1] < 0.0 || tors_angewChem2020[zl - 1] < 0.0) return p;
    const double cnp = cn_i * cn_l;
    if (cnp > 0.01) fkl *= std::pow(cnp, -0.14);
    if (hyb_i == 5 || hyb_l == 5) fkl *= 1.5;
    double f1 = 1.0;
    int eh_j = hyb_j, eh_k = hyb_k;
    if (jpi && eh_j == 3) eh_j = 2;
    if (kpi && eh_k == 3) eh_k = 2;
    if (eh_j == 3 && eh_k == 3) {
        const int gj = (zj == 7 || zj == 15) ? 5 : (zj == 8 || zj == 16) ? 6 : 0;
        const int gk = (zk == 7 || zk == 15) ? 5 : (zk == 8 || zk == 16) ? 6 : 0;
        if (gj == 6 && gk == 6) {
            f1 = 5.0; p.n = 2; p.phi0 = 90.0 * M_PI / 180.0;
            if (zj >= 16 && zk >= 16) f1 = 25.0;
        } else if (gj == 5 && gk == 5) {
            f1 = 3.0; p.n = 3; p.phi0 = 60.0 * M_PI / 180.0;
        } else if ((gj == 5 && gk == 6) || (gj == 6 && gk == 5)) {
            f1 = 1.0; p.n = 2; p.phi0 = 90.0 * M_PI / 180.0;
            if (zj >= 15 && zk >= 15) f1 = 20.0;
        }
    } else if (!in_ring && ((eh_j == 2 && eh_k == 3) || (eh_j == 3 && eh_k == 2))) {
        f1 = 0.5;
        if (zj == 7 || zk == 7) f1 = 0.2;
    } else if (eh_j == 2 && eh_k == 2) {
        f1 = 1.0;
    }
    double f2 = 0.0, cpibo = 0.0;
    {
        const double pb = pibo_of(c, ja, ka);
        cpibo = pb;
        if (pb > 0.0) {
            const double diff = 1.24 - pb;
            f2 = pb * std::exp(-2.5 * std::pow(diff, 14));
            if (zi > 10 && m.pi_frag[ia] <= 0) f2 *= 1.3;
            if (zl > 10 && m.pi_frag[la] <= 0) f2 *= 1.3;
            f1 *= 0.55;
        }
    }
    int nhi = 1, nhj = 1;
    for (int nb : m.adj[ja]) if (c.Z[nb] == 1) ++nhi;
    for (int nb : m.adj[ka]) if (c.Z[nb] == 1) ++nhj;
    fij *= std::pow((double)(nhi * nhj), 0.07);
    if (tors_alpha_co(c, ja, ka)) fij *= 1.3;
    if (tors_amide(c, ja) && zk == 6 && hyb_k == 3) fij *= 1.3;
    if (tors_amide(c, ka) && zj == 6 && hyb_j == 3) fij *= 1.3;
    if (c.is_metal[ja] && m.adj[ja].size() > 4) return p;
    if (c.is_metal[ka] && m.adj[ka].size() > 4) return p;
    if (in_ring) {
        p.n = 1;
        p.phi0 = 0.0;
        if (btyp == 2) p.n = 2;
        int rings4 = 0, ringl = 0;
        if (ring_size == 3) rings4 = 3;
        else if (ring_size > 3) rings4 = smallest_ring_all(c, ia, ja, ka, la);
        const bool notpicon = !(m.pi_frag[ia] > 0 || m.pi_frag[la] > 0);
        if (rings4 > 0 && btyp == 1) {
            if (rings4 >= 4) ringl = largest_ring_all(c, ia, ja, ka, la);
            if (rings4 == 3 && notpicon) { p.n = 1; p.phi0 = 0.0; f1 = 0.3; }
            if (rings4 == 4 && ringl == rings4 && notpicon) { p.n = 6; p.phi0 = 30.0 * M_PI / 180.0; f1 = 1.0; }
            if (rings4 == 5 && ringl == rings4 && notpicon) { p.n = 6; p.phi0 = 30.0 * M_PI / 180.0; f1 = 1.5; }
            if (rings4 == 6 && ringl == rings4 && notpicon) { p.n = 3; p.phi0 = 60.0 * M_PI / 180.0; f1 = 5.7; }
        }
        if (rings4 == 0 && btyp == 1 && (int)cn_i == 1 && (int)cn_l == 1) {
            p.n = 6; p.phi0 = 30.0 * M_PI / 180.0; f1 = 0.30;
        }
        if (btyp == 2 && ring_size == 5 && zj * zk == 42) {
            if (tors_amide(c, ja) || tors_amide(c, ka)) {
                f1 = 5.0;
                if (cpibo > 0.0) f1 *= 0.55;
            }
        }
    }
    if (!in_ring && jpi && !kpi && hyb_k == 3) {
        f1 = 0.5;
        if (zj == 7) f1 = 0.2;
        p.phi0 = M_PI;
        p.n = 3;
    } else if (!in_ring && kpi && !jpi && hyb_j == 3) {
        f1 = 0.5;
        if (zk == 7) f1 = 0.2;
        p.phi0 = M_PI;
        p.n = 3;
    }
    const double fqq = 1.0 + std::fabs(qa_j * qa_k) * 12.0;
    const double fctot = (f1 + 10.0 * 1.18 * f2) * fqq * fij * fkl;
    if (fctot < fcthr) return p;
    p.V = fctot;
    p.fij = fij;
    p.fkl = fkl;
    p.fqq = fqq;
    return p;
}

static void generate_torsions(Ctx& c)
{
    const Model& m = c.m;
    std::vector<TorsionTerm> prim, extra;
    std::set<std::array<int, 4>> seen;
    auto angle_at = [&](int a, int b, int d) {
        const double* x = c.xa.data();
        double u[3], v[3];
        for (int q = 0; q < 3; ++q) { u[q] = x[3 * a + q] - x[3 * b + q]; v[q] = x[3 * d + q] - x[3 * b + q]; }
        const double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        const double nv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int q = 0; q < 3; ++q) { u[q] /= nu; v[q] /= nv; }
        return std::acos(std::max(-1.0, std::min(1.0, u[0] * v[0] + u[1] * v[1] + u[2] * v[2])));
    };
    const double thr = 170.0 * M_PI / 180.0;
    for (size_t bi = 0; bi < m.topo_bonds.size(); ++bi) {
        const int j = m.topo_bonds[bi].first, k = m.topo_bonds[bi].second;
        if (j >= k) continue;
        if (m.adj[j].size() < 2 || m.adj[k].size() < 2) continue;
        const int bt = m.bond_type[bi];
        if (bt == 3 || bt == 6) continue;
        for (int i : m.adj[j]) {
            if (i == k) continue;
            for (int l : m.adj[k]) {
                if (l == j || i == l) continue;
                std::array<int, 4> f = {i, j, k, l}, r = {l, k, j, i};
                auto kk = f < r ? f : r;
                if (seen.count(kk)) continue;
                seen.insert(kk);
                if (angle_at(i, j, k) > thr || angle_at(j, k, l) > thr) continue;
                const int rs = same_ring_size(c, j, k);
                const bool in_ring = rs > 0;
                TorsParams p = torsion_params(c, i, j, k, l, bt, in_ring, rs);
                if (std::fabs(p.V) >= 1.0e-3) prim.push_back({l, j, k, i, p.V, (double)p.n, p.phi0, 0});
                const bool sp3c = m.hyb[j] == 3 && m.hyb[k] == 3;
                const bool sp3o = m.hyb[i] == 3 && m.hyb[l] == 3;
                if (sp3c && sp3o && !in_ring && bt < 5 && p.fij > 0.0 && p.fkl > 0.0) {
                    double ff = -0.90;
                    if (c.Z[j] == 7 || c.Z[k] == 7) ff = 0.70;
                    if (c.Z[j] == 8 || c.Z[k] == 8) ff = -2.00;
                    const double eb = ff * p.fij * p.fkl * p.fqq;
                    if (std::isfinite(eb)) extra.push_back({l, j, k, i, eb, 1.0, M_PI, 0});
                }
            }
        }
    }
    c.m.n_primary_torsions = (int)prim.size();
    c.m.torsions = prim;
    c.m.torsions.insert(c.m.torsions.end(), extra.begin(), extra.end());
}

// ---------------------------------------------------------------------------------
// Inversions: gfnff_inversions.cpp:749-871; triple-bond torsions:
// gfnff_torsions.cpp:2070-2161
// ---------------------------------------------------------------------------------
static void generate_inversions(Ctx& c)
{
    const Model& m = c.m;
    c.m.inversions.clear();
    for (int i = 0; i < c.n; ++i) {
        if (m.adj[i].size() != 3) continue;
        const int Zi = c.Z[i];
        const bool has_pi = m.pi_frag[i] > 0;
        const bool satN = !has_pi && Zi == 7;
        if (!has_pi && !satN) continue;
        std::vector<int> nb = m.adj[i];
        {
            const int nn = (int)nb.size();
            std::vector<double> sd(nn);
            for (int q = 0; q < nn; ++q) {
                const double* x = c.xa.data();
                const double dx = x[3 * i] - x[3 * nb[q]], dy = x[3 * i + 1] - x[3 * nb[q] + 1],
                             dz = x[3 * i + 2] - x[3 * nb[q] + 2];
                sd[q] = std::sqrt(dx * dx + dy * dy + dz * dz);
            }
            for (int ii = 1; ii < nn; ++ii) {
                const int idx = ii - 1;
                int k = idx;
                double pp = sd[idx];
                for (int jj = ii; jj < nn; ++jj) {
                    if (sd[jj] > pp) break;
                    k = jj;
                    pp = sd[jj];
                }
                if (k == idx) break;
                sd[k] = sd[idx];
                sd[idx] = pp;
                std::swap(nb[idx], nb[k]);
            }
        }
        InversionTerm t;
        t.i = i; t.j = nb[0]; t.k = nb[1]; t.l = nb[2];
        if (satN) {
            double V = 0.0;
            for (int q = 0; q < 3; ++q) V += 0.60 * std::sqrt(repz[c.Z[nb[q]] - 1]);
            t.fc = V;
            t.omega0 = 80.0 * M_PI / 180.0;
            t.type = -1;
        } else {
            int ncarbo = 0, nf = 0;
            for (int q = 0; q < 3; ++q) {
                const int z = c.Z[nb[q]];
                if (z == 8 || z == 16) ++ncarbo;
                if (z == 9 || z == 17 || z == 35 || z == 53) ++nf;
            }
            const double fqq = 1.0 + m.qa[i] * 5.0;
            const double sp = pibo_of(c, i, nb[0]) + pibo_of(c, i, nb[1]) + pibo_of(c, i, nb[2]);
            const double f2 = 1.0 - sp * 0.50;
            double V = 1.05 * f2 * fqq;
            if (Zi == 5 && ncarbo > 0) V *= 38.0;
            if (Zi == 6 && ncarbo > 0) V *= 38.0;
            if (Zi == 6 && nf > 0 && ncarbo == 0) V *= 10.0;
            if (Zi == 7 && ncarbo > 0) V *= 10.0 / f2;
            t.fc = V;
            t.omega0 = 0.0;
            t.type = 0;
        }
        c.m.inversions.push_back(t);
    }
}

static void generate_storsions(Ctx& c)
{
    const Model& m = c.m;
    c.m.storsions.clear();
    for (int i = 0; i < c.n; ++i) {
        if (c.Z[i] != 6 || m.adj[i].size() != 2) continue;
        for (int nbi : m.adj[i]) {
            if (nbi <= i) continue;
            if (c.Z[nbi] != 6 || m.adj[nbi].size() != 2) continue;
            if (dist_bohr(c, i, nbi) > 2.37) continue;
            int jj = -1, kk = -1;
            for (int x : m.adj[i]) if (x != nbi && c.Z[x] == 6) jj = x;
            for (int x : m.adj[nbi]) if (x != i && c.Z[x] == 6) kk = x;
            if (jj == -1 || kk == -1) continue;
            if (!(m.hyb[jj] == 2 && m.hyb[kk] == 2)) continue;
            int ii = -1, ll = -1;
            for (int x : m.adj[jj])
                if (x != i && m.hyb[x] == 2 && c.Z[x] == 6 && m.adj[x].size() == 3 && x > ii) ii = x;
            for (int x : m.adj[kk])
                if (x != nbi && m.hyb[x] == 2 && c.Z[x] == 6 && m.adj[x].size() == 3 && x > ll) ll = x;
            if (ii != -1 && ll != -1) c.m.storsions.push_back({ii, jj, kk, ll, 3.75e-4});
        }
    }
}

// ---------------------------------------------------------------------------------
// Repulsion pairs: gfnff_method.cpp:9749-9889 (generateRepulsionPairsNative)
// ---------------------------------------------------------------------------------
static void generate_repulsion(Ctx& c)
{
    const Model& m = c.m;
    const double REPSCALB = 1.7583, REPSCALN = 0.4270, QREPSCAL = 0.3480, NREPSCAL = -0.1270;
    const double HHFAC = 0.6290, HH13REP = 1.4580, HH14REP = 0.7080;
    c.m.rep_bonded.clear();
    c.m.rep_nonbonded.clear();
    for (auto& b : m.topo_bonds) {
        const int zi = c.Z[b.first] - 1, zj = c.Z[b.second] - 1;
        RepPair r;
        r.i = b.first;
        r.j = b.second;
        r.alpha = std::sqrt(repa_angewChem2020[zi] * repa_angewChem2020[zj]);
        r.repab = repz[zi] * repz[zj] * REPSCALB;
        c.m.rep_bonded.push_back(r);
    }
    auto make = [&](int ii, int jj, std::vector<RepPair>& out) {
        const int i = std::min(ii, jj), j = std::max(ii, jj);
        if (i == j || c.bonded(i, j)) return;
        const int zi = c.Z[i] - 1, zj = c.Z[j] - 1;
        const double cni = (double)m.adj[i].size(), cnj = (double)m.adj[j].size();
        const double fni = 1.0 + NREPSCAL / (1.0 + cni * cni);
        const double fnj = 1.0 + NREPSCAL / (1.0 + cnj * cnj);
        const double d1 = repan_angewChem2020[zi] * (1.0 + m.qa[i] * QREPSCAL) * fni;
        const double d2 = repan_angewChem2020[zj] * (1.0 + m.qa[j] * QREPSCAL) * fnj;
        double ff = 1.0;
        const int Zi = zi + 1, Zj = zj + 1;
        if (Zi == 1 && Zj == 1) {
            ff = HHFAC;
            const int td = topo_dist(c, i, j);
            if (td == 2) ff *= HH13REP;
            else if (td == 3) ff *= HH14REP;
        } else if ((Zi == 1 && metal_type[Zj - 1] > 0) || (Zj == 1 && metal_type[Zi - 1] > 0)) {
            ff = 0.85;
        } else if ((Zi == 1 && Zj == 6) || (Zj == 1 && Zi == 6)) {
            ff = 0.91;
        } else if ((Zi == 1 && Zj == 8) || (Zj == 1 && Zi == 8)) {
            ff = 1.04;
        }
        RepPair r;
        r.i = i;
        r.j = j;
        r.alpha = std::sqrt(d1 * d2) * ff;
        r.repab = repz[zi] * repz[zj] * REPSCALN;
        out.push_back(r);
    };
    const bool cell = (m.opt.cell_list_min_atoms == 0 || c.n >= m.opt.cell_list_min_atoms);
    c.m.nonbonded_rep_all_pairs = !cell;
    auto by_pair = [](const RepPair& a, const RepPair& b) { return a.i != b.i ? a.i < b.i : a.j < b.j; };
    if (cell) {
        // rows in parallel, one list per thread; a thread's rows are a contiguous ascending
        // range, so its list sorted by (i, j) and the lists joined in thread order are the
        // whole list sorted by (i, j), the same list as a serial pass
        std::vector<std::vector<RepPair>> part(setup_threads());
        pairs_within_rows(c, 20.0, false, [&](int t, int i, int j, double) { make(i, j, part[t]); });
#pragma omp parallel for schedule(dynamic, 1)
        for (int t = 0; t < (int)part.size(); ++t) std::sort(part[t].begin(), part[t].end(), by_pair);
        size_t tot = 0;
        for (auto& p : part) tot += p.size();
        c.m.rep_nonbonded.reserve(tot);
        for (auto& p : part) c.m.rep_nonbonded.insert(c.m.rep_nonbonded.end(), p.begin(), p.end());
    } else {
        for (int i = 0; i < c.n; ++i)
            for (int j = i + 1; j < c.n; ++j) make(i, j, c.m.rep_nonbonded);
        std::sort(c.m.rep_nonbonded.begin(), c.m.rep_nonbonded.end(), by_pair);
    }
}

// ---------------------------------------------------------------------------------
// D4 dispersion: dispersion/d4param_generator.cpp:881-1080 (C6 reference integration),
// :1079-1165 (Gaussian weights, wf = 4), :1235-1290 (half contraction), :1959-2092
// (pair list, 60 bohr), gfnff_method.cpp:9915-10049 (ATM triples).
// ---------------------------------------------------------------------------------
static const double kFreq[kNumFreq] = {0.000001, 0.050000, 0.100000, 0.200000, 0.300000, 0.400000,
                                       0.500000, 0.600000, 0.700000, 0.800000, 0.900000, 1.000000,
                                       1.200000, 1.400000, 1.600000, 1.800000, 2.000000, 2.500000,
                                       3.000000, 4.000000, 5.000000, 7.500000, 10.000000};

static double c6_reference(int ei, int ej, int ri, int rj)
{
    const double* ai = &d4_alpha_corr[((size_t)ei * kMaxRef + ri) * kNumFreq];
    const double* aj = &d4_alpha_corr[((size_t)ej * kMaxRef + rj) * kNumFreq];
    double c6 = 0.0;
    for (int w = 0; w < kNumFreq - 1; ++w) {
        const double p0 = ai[w] * aj[w];
        const double p1 = ai[w + 1] * aj[w + 1];
        c6 += 0.5 * (p0 + p1) * (kFreq[w + 1] - kFreq[w]);
    }
    return c6 * (3.0 / M_PI);
}

static double zeta_scale(int Z, double q)
{   // gfnff_par.h:941-962
    if (Z < 1 || Z > 86) return 1.0;
    const double zeff = zeta_zeff[Z - 1], cc = zeta_c[Z - 1];
    const double qmod = zeff + q;
    if (qmod < 0.0) return std::exp(3.0);
    return std::exp(3.0 * (1.0 - std::exp(cc * (1.0 - zeff / qmod))));
}

// half contraction at the setup weights: g[i][s][b] = sum_a w_i[a] C6ref[a][b]
static std::vector<double> half_contraction(const Model& m)
{
    const int n = m.n, K = (int)m.present_Z.size();
    std::vector<double> g((size_t)n * K * kMaxRef, 0.0);
    for (int i = 0; i < n; ++i) {
        const double* wi = &m.w_setup[(size_t)i * kMaxRef];
        for (int s = 0; s < K; ++s) {
            const int ne = std::min(d4_refn[m.present_Z[s] - 1], kMaxRef);
            const double* C = &m.c6ref[(((size_t)m.slot[i] * K + s) * kMaxRef) * kMaxRef];
            for (int b = 0; b < ne; ++b) {
                double v = 0.0;
                for (int a = 0; a < m.nref[i]; ++a) v += wi[a] * C[(size_t)a * kMaxRef + b];
                g[((size_t)i * K + s) * kMaxRef + b] = v;
            }
        }
    }
    return g;
}

static double setup_c6(const Model& m, const std::vector<double>& g, int i, int j)
{
    const int K = (int)m.present_Z.size();
    const double* gi = &g[((size_t)i * K + m.slot[j]) * kMaxRef];
    const double* wj = &m.w_setup[(size_t)j * kMaxRef];
    double v = 0.0;
    for (int b = 0; b < m.nref[j]; ++b) v += gi[b] * wj[b];
    return v;
}

// the D4 pair list at the setup geometry (pairs within 60 bohr, rows by i, j ascending)
static void disp_list(Ctx& c, const std::vector<double>& g)
{
    Model& m = c.m;
    const int n = c.n;
    const double a1 = 0.58, a2 = 4.80;
    std::vector<std::vector<DispPair>> rows(n);
    pairs_within(c, 60.0, false, [&](int i, int j, double) {
        DispPair d;
        d.i = i;
        d.j = j;
        d.c6 = setup_c6(m, g, i, j);
        d.r4r2 = 3.0 * m.sqrt_zr4r2[i] * m.sqrt_zr4r2[j];
        d.r0sq = std::pow(a1 * std::sqrt(d.r4r2) + a2, 2);
        d.zetac6 = m.zeta[i] * m.zeta[j];
        rows[i].push_back(d);
    });
    m.disp.clear();
    for (auto& r : rows) {
        std::sort(r.begin(), r.end(), [](const DispPair& a, const DispPair& b) { return a.j < b.j; });
        m.disp.insert(m.disp.end(), r.begin(), r.end());
    }
}

static void setup_d4(Ctx& c)
{
    Model& m = c.m;
    const int n = c.n;
    m.present_Z.clear();
    m.slot.assign(n, -1);
    std::vector<int> sl(119, -1);
    for (int i = 0; i < n; ++i) {
        const int z = c.Z[i];
        if (sl[z] < 0) { sl[z] = (int)m.present_Z.size(); m.present_Z.push_back(z); }
        m.slot[i] = sl[z];
    }
    const int K = (int)m.present_Z.size();
    m.c6ref.assign((size_t)K * K * kMaxRef * kMaxRef, 0.0);
    for (int a = 0; a < K; ++a)
        for (int b = 0; b < K; ++b) {
            const int ea = m.present_Z[a] - 1, eb = m.present_Z[b] - 1;
            for (int ra = 0; ra < d4_refn[ea]; ++ra)
                for (int rb = 0; rb < d4_refn[eb]; ++rb)
                    m.c6ref[(((size_t)a * K + b) * kMaxRef + ra) * kMaxRef + rb] = c6_reference(ea, eb, ra, rb);
        }
    m.nref.resize(n);
    m.refcn.assign((size_t)n * kMaxRef, 0.0);
    m.w_setup.assign((size_t)n * kMaxRef, 0.0);
    m.zeta.resize(n);
    m.sqrt_zr4r2.resize(n);
    for (int i = 0; i < n; ++i) {
        const int e = c.Z[i] - 1;
        m.nref[i] = std::min(d4_refn[e], kMaxRef);
        for (int r = 0; r < kMaxRef; ++r) m.refcn[(size_t)i * kMaxRef + r] = d4_refcn[(size_t)e * kMaxRef + r];
        const double r4 = (e < 36) ? d4_r4_over_r2[e] : 10.0;
        m.sqrt_zr4r2[i] = std::sqrt(0.5 * r4 * std::sqrt((double)(e + 1)));
        m.zeta[i] = zeta_scale(c.Z[i], m.qa[i]);
        d4_weights(m, i, m.cn_setup[i], &m.w_setup[(size_t)i * kMaxRef], nullptr);
    }
    const std::vector<double> g = half_contraction(m);
    auto c6_of = [&](int i, int j) { return setup_c6(m, g, i, j); };
    m.disp.clear();
    if (m.opt.dispersion && !m.disp_on_device) disp_list(c, g);
    // ATM triples over bonded triplets (s9 = 1)
    m.atm.clear();
    if (m.opt.dispersion) {
        std::set<std::array<int, 3>> tri;
        for (int i = 0; i < n; ++i)
            for (int j : m.adj[i]) {
                if (j <= i) continue;
                for (int k : m.adj[i])
                    if (k != j) { std::array<int, 3> t = {i, j, k}; std::sort(t.begin(), t.end()); tri.insert(t); }
                for (int k : m.adj[j])
                    if (k != i) { std::array<int, 3> t = {i, j, k}; std::sort(t.begin(), t.end()); tri.insert(t); }
            }
        for (auto& t : tri) {
            ATMTriple a;
            a.i = t[0]; a.j = t[1]; a.k = t[2];
            a.c6ij = c6_of(t[0], t[1]);
            a.c6ik = c6_of(t[0], t[2]);
            a.c6jk = c6_of(t[1], t[2]);
            if (t[0] == t[1]) a.scale = (t[0] == t[2]) ? 1.0 / 6.0 : 0.5;
            else a.scale = (t[0] != t[2] && t[1] != t[2]) ? 1.0 : 0.5;
            m.atm.push_back(a);
        }
    }
}

// ---------------------------------------------------------------------------------
// Bonded ATM (gfnff_method.cpp:3626-3650, b3list from :9494-9512)
// ---------------------------------------------------------------------------------
static void generate_batm(Ctx& c)
{
    Model& m = c.m;
    m.batm.clear();
    const double cr = std::pow(0.30, 1.0 / 3.0);
    auto zb = [&](int z) { return z == 1 ? -0.25 * cr : -(double)z * cr; };
    for (int i = 0; i < c.n; ++i)
        for (auto& p : c.tdist[i]) {
            const int j = p.first;
            if (j >= i || p.second != 3) continue;
            for (int k : m.adj[j]) m.batm.push_back({i, j, k, zb(c.Z[i]), zb(c.Z[j]), zb(c.Z[k])});
            for (int k : m.adj[i]) m.batm.push_back({i, j, k, zb(c.Z[i]), zb(c.Z[j]), zb(c.Z[k])});
        }
}

// ---------------------------------------------------------------------------------
// HB / XB detection: gfnff_method.cpp:7936-8495, :8520-8672, bond cross reference
// :3680-3712.  Uses the Phase-1 charges.
// ---------------------------------------------------------------------------------
static void basicity(const Ctx& c, const std::vector<double>& xb, std::vector<double>& bas)
{
    const Model& m = c.m;
    bas.assign(c.n, 0.0);
    for (int i = 0; i < c.n; ++i) {
        const int z = c.Z[i];
        bas[i] = (z < 74) ? hb_basicity[z] : 0.0;
        if (z == 8) {
            const bool cn1 = m.adj[i].size() == 1;
            if (cn1 && m.pi_frag[i] != 0 && c.Z[m.adj[i][0]] == 6 && m.pi_frag[m.adj[i][0]] != 0)
                bas[i] = 0.68;                                   // carbonyl O
            else if (cn1 && c.Z[m.adj[i][0]] == 7)
                bas[i] = 0.47;                                   // nitro O
        } else if (z == 6 && m.adj[i].size() == 2) {
            const int a = m.adj[i][0], b = m.adj[i][1];
            double v1[3], v2[3];
            for (int d = 0; d < 3; ++d) { v1[d] = xb[3 * a + d] - xb[3 * i + d]; v2[d] = xb[3 * b + d] - xb[3 * i + d]; }
            const double cphi = (v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2]) /
                                (std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]) *
                                 std::sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]));
            const double deg = std::acos(std::max(-1.0, std::min(1.0, cphi))) * 180.0 / M_PI;
            if (deg < 150.0 && m.qa[i] > -0.4) bas[i] = 1.46;
        }
    }
}

// per-atom inputs of the HB detection at the geometry xb (gfnff_method.cpp:7936-8100)
static HBAtoms hb_atoms(const Ctx& c, const std::vector<double>& xb)
{
    const Model& m = c.m;
    const int n = c.n;
    const std::vector<double>& q = m.qa;
    HBAtoms a;
    basicity(c, xb, a.bas);
    a.aci.assign(n, 0.0);
    for (int i = 0; i < n; ++i) a.aci[i] = (c.Z[i] < 74) ? hb_acidity[c.Z[i]] : 0.0;
    for (int i = 0; i < n; ++i)
        if (fg_amide_h(c, i)) a.aci[m.adj[i][0]] *= 0.80;
    a.hcand.assign(n, 0);
    for (int h = 0; h < n; ++h) {
        if (c.Z[h] != 1 || m.hyb[h] == 1 || m.adj[h].empty()) continue;
        const int A = *std::min_element(m.adj[h].begin(), m.adj[h].end());
        double thr = 0.01;
        if (c.Z[A] > 10) thr -= 0.20;
        if (m.hyb[A] == 3 && c.Z[A] == 6) thr += 0.05;
        if (q[h] > thr) a.hcand[h] = 1;
    }
    a.thr1 = 200.0 - std::log10(m.opt.hb_accuracy) * 50.0;
    a.thr2 = 400.0 - std::log10(m.opt.hb_accuracy) * 50.0;
    a.ok.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        if (c.Z[i] == 6 && m.pi_frag[i] == 0) continue;
        double t = 0.10;
        if (c.Z[i] > 10) t += 0.2;
        a.ok[i] = !(q[i] > t);
    }
    return a;
}

// the HB terms and the bond <-> HB cross reference (gfnff_method.cpp:7936-8495, :3680-3712)
static void detect_hb_terms(Ctx& c, const std::vector<double>& xb, const HBAtoms& at)
{
    Model& m = c.m;
    const int n = c.n;
    const std::vector<double>& q = m.qa;
    auto d2 = [&](int i, int j) {
        const double dx = xb[3 * i] - xb[3 * j], dy = xb[3 * i + 1] - xb[3 * j + 1], dz = xb[3 * i + 2] - xb[3 * j + 2];
        return dx * dx + dy * dy + dz * dz;
    };
    const std::vector<double>& bas = at.bas;
    const std::vector<double>& aci = at.aci;
    const std::vector<char>& hbh = at.hcand;
    const double hbthr1 = at.thr1, hbthr2 = at.thr2;
    auto ok_atom = [&](int i) { return at.ok[i] != 0; };
    std::vector<std::vector<int>> hyd_on(n);
    for (auto& b : m.topo_bonds) {
        if (hbh[b.first]) hyd_on[b.second].push_back(b.first);
        if (hbh[b.second]) hyd_on[b.first].push_back(b.second);
    }
    // spatial grid over the geometry for the pair / hydrogen searches
    Ctx tmp(m);
    tmp.xb = xb;
    std::vector<std::vector<int>> near_h(n);   // candidate H within sqrt(hbthr2) of each atom
    std::vector<std::pair<int, int>> ab;
    pairs_within(tmp, std::sqrt(hbthr2), false, [&](int i, int j, double r2) {
        if (hbh[j]) near_h[i].push_back(j);
        if (hbh[i]) near_h[j].push_back(i);
        if (r2 > hbthr1) return;
        if (!ok_atom(i) || !ok_atom(j)) return;
        const double s1 = bas[i] * aci[j], s2 = bas[j] * aci[i];
        if (s1 < 1e-6 && s2 < 1e-6) return;
        ab.push_back({std::max(i, j), std::min(i, j)});
    });
    std::sort(ab.begin(), ab.end());
    auto fill = [&](HBTerm& hb, int A, int H, int B) {
        hb.a = A; hb.h = H; hb.b = B;
        hb.bas_a = bas[A]; hb.bas_b = bas[B]; hb.aci_a = aci[A]; hb.aci_b = aci[B];
        hb.q_h = q[H]; hb.q_a = q[A]; hb.q_b = q[B];
    };
    auto nhb2 = [&](int A, int H, int B) {
        if (c.bonded(A, B)) return;
        HBTerm hb;
        fill(hb, A, H, B);
        hb.case_type = 2;
        if (c.Z[B] == 8 && m.adj[B].size() == 1) {
            const int p = m.adj[B][0];
            if (c.Z[p] == 6 || c.Z[p] == 7) { hb.case_type = 3; hb.parent_c = p; }
        } else if (c.Z[B] == 7 && m.adj[B].size() == 2) {
            hb.case_type = 4;
        }
        hb.nb_b = m.adj[B];
        if (hb.case_type == 3)
            for (int x : m.adj[hb.parent_c]) if (x != B) hb.nb_c.push_back(x);
        m.hbonds.push_back(hb);
    };
    m.hbonds.clear();
    for (auto& p : ab) {
        const int i = p.first, j = p.second;
        const double rab2 = d2(i, j);
        if (rab2 > hbthr1) continue;
        const bool nonb = !c.bonded(i, j);
        if (nonb) {
            for (int H : hyd_on[i]) nhb2(i, H, j);
            for (int H : hyd_on[j]) if (!c.bonded(i, H)) nhb2(j, H, i);
        }
        std::vector<int> hs = near_h[i];
        std::sort(hs.begin(), hs.end());
        for (int H : hs) {
            if (c.bonded(i, H) || c.bonded(j, H)) continue;
            if (rab2 + d2(i, H) + d2(j, H) < hbthr2) {
                HBTerm hb;
                fill(hb, i, H, j);
                hb.case_type = 1;
                m.hbonds.push_back(hb);
            }
        }
    }
    // bond <-> HB cross reference (A-H bonds whose HB acceptors are N or O)
    std::map<std::pair<int, int>, std::vector<int>> ahb;
    for (auto& hb : m.hbonds)
        if (c.Z[hb.b] == 7 || c.Z[hb.b] == 8) ahb[{hb.a, hb.h}].push_back(hb.b);
    m.bond_hb.clear();
    for (auto& b : m.bonds) {
        b.nr_hb = 0;
        b.hb_h = -1;
        int H = -1, A = -1;
        if (c.Z[b.i] == 1) { H = b.i; A = b.j; }
        else if (c.Z[b.j] == 1) { H = b.j; A = b.i; }
        else continue;
        if (c.Z[A] != 7 && c.Z[A] != 8) continue;
        auto it = ahb.find({A, H});
        if (it != ahb.end() && !it->second.empty()) {
            b.nr_hb = (int)it->second.size();
            b.hb_h = H;
            m.bond_hb.push_back({A, H, it->second});
        }
    }
}

// halogen bonds (gfnff_method.cpp:8520-8672)
static void detect_xbonds(Ctx& c, const std::vector<double>& xb, const std::vector<double>& bas)
{
    Model& m = c.m;
    const int n = c.n;
    const std::vector<double>& q = m.qa;
    auto d2 = [&](int i, int j) {
        const double dx = xb[3 * i] - xb[3 * j], dy = xb[3 * i + 1] - xb[3 * j + 1], dz = xb[3 * i + 2] - xb[3 * j + 2];
        return dx * dx + dy * dy + dz * dz;
    };
    m.xbonds.clear();
    auto isx = [](int z) {
        return z == 17 || z == 35 || z == 53 || z == 16 || z == 34 || z == 52 || z == 15 || z == 33 || z == 51;
    };
    for (auto& b : m.topo_bonds) {
        int X = -1, A = -1;
        if (isx(c.Z[b.first])) { X = b.first; A = b.second; }
        else if (isx(c.Z[b.second])) { X = b.second; A = b.first; }
        if (X < 0) continue;
        if (c.Z[X] == 16 && m.adj[X].size() > 2) continue;
        for (int B = 0; B < n; ++B) {
            if (d2(B, X) >= 100.0) continue;
            if (B == A || B == X) continue;
            if (bas[B] < 1e-6) continue;
            if (c.Z[B] == 6) {
                if (m.pi_frag[B] == 0 || q[B] >= 0.05) continue;
            } else if (q[B] > 0.05) continue;
            if (c.bonded(X, B)) continue;
            m.xbonds.push_back({A, X, B, (c.Z[X] < 72) ? xb_acidity[c.Z[X]] : 0.0, q[X], q[B]});
        }
    }
}

void detect_hbxb(Ctx& c, const std::vector<double>& xb)
{
    const HBAtoms a = hb_atoms(c, xb);
    if (!c.m.hb_on_device) detect_hb_terms(c, xb, a);
    detect_xbonds(c, xb, a.bas);
}

void generate_parameters(Ctx& c)
{
    generate_bonds(c);
    generate_angles(c);
    generate_torsions(c);
    generate_inversions(c);
    generate_storsions(c);
    generate_repulsion(c);
    setup_d4(c);
    generate_batm(c);
    if (c.m.opt.hbond) detect_hbxb(c, c.xb);
}

}  // namespace detail

void d4_weights(const Model& m, int i, double cn, double* w, double* dw)
{   // d4param_generator.cpp:1079-1140 and :1692-1740 (wf = 4)
    const int nr = m.nref[i];
    const double* rc = &m.refcn[(size_t)i * kMaxRef];
    double ex[kMaxRef] = {0}, dex[kMaxRef] = {0};
    double norm = 0.0, dnorm = 0.0;
    for (int r = 0; r < nr; ++r) {
        const double d = cn - rc[r];
        ex[r] = std::exp(-4.0 * d * d);
        dex[r] = (-2.0 * 4.0) * d * ex[r];
        norm += ex[r];
        dnorm += dex[r];
    }
    for (int r = 0; r < kMaxRef; ++r) { w[r] = 0.0; if (dw) dw[r] = 0.0; }
    if (nr == 0) return;
    if (norm > 1e-10) {
        const double inv = 1.0 / norm;
        for (int r = 0; r < nr; ++r) w[r] = ex[r] * inv;
        if (dw) {
            const double inv2 = 1.0 / (norm * norm);
            for (int r = 0; r < nr; ++r) dw[r] = (dex[r] * norm - ex[r] * dnorm) * inv2;
        }
    } else {
        w[0] = 1.0;
    }
}

Model build_model(int n, const int* Z, const double* xyz_ang, int charge, const SetupOptions& opt,
                  const BuildLists& lists, const char* topo_cache)
{
    if (n <= 0) throw std::runtime_error("no atoms");
    for (int i = 0; i < n; ++i)
        if (Z[i] < 1 || Z[i] > 86) throw std::runtime_error("element not supported by GFN-FF");
    Model m;
    m.n = n;
    m.charge = charge;
    m.opt = opt;
    m.hb_on_device = !lists.host_hb;
    m.disp_on_device = !lists.host_disp;
    m.Z.assign(Z, Z + n);
    detail::Ctx c(m);
    c.Z = m.Z.data();
    c.xa.assign(xyz_ang, xyz_ang + 3 * (size_t)n);
    c.xb.resize(3 * (size_t)n);
    for (size_t k = 0; k < 3 * (size_t)n; ++k) {
        if (!std::isfinite(xyz_ang[k])) throw std::runtime_error("non-finite coordinate");
        c.xb[k] = xyz_ang[k] * kAngToBohr;
    }
    m.xyz_setup = c.xb;
    c.rcov_cn.resize(n);
    m.rcov_cn.resize(n);
    m.rcov_d3.resize(n);
    m.rvdw.resize(n);
    for (int i = 0; i < n; ++i) {
        const int e = Z[i] - 1;
        c.rcov_cn[i] = (4.0 / 3.0) * gfnff_tables::cn_covalent_radii_ang[e] * kAngToBohrCN;
        m.rcov_cn[i] = c.rcov_cn[i];
        m.rcov_d3[i] = gfnff_tables::covalent_rad_d3[e];
        m.rvdw[i] = gfnff_tables::covalent_radii[e];
    }
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n && n <= 4000; ++j)
            if (detail::dist2_bohr(c, i, j) < 1e-20) throw std::runtime_error("coincident atoms");
    c.topo_cache = topo_cache;
    detail::compute_topology(c);
    detail::generate_parameters(c);
    return m;
}

bool refresh_topology(Model& m, const double* xyz_bohr, const char* topo_cache)
{
    const int n = m.n;
    Model t;
    t.n = n;
    t.charge = m.charge;
    t.opt = m.opt;
    t.Z = m.Z;
    detail::Ctx c(t);
    c.Z = t.Z.data();
    c.xb.assign(xyz_bohr, xyz_bohr + 3 * (size_t)n);
    c.xa.resize(c.xb.size());
    for (size_t k = 0; k < c.xb.size(); ++k) c.xa[k] = c.xb[k] / kAngToBohr;
    t.xyz_setup = c.xb;
    c.rcov_cn = m.rcov_cn;
    t.rcov_cn = m.rcov_cn;
    t.rcov_d3 = m.rcov_d3;
    t.rvdw = m.rvdw;
    c.topo_cache = topo_cache;
    detail::compute_topology(c);
    const bool same = t.topo_bonds == m.topo_bonds && t.adj == m.adj && t.hyb == m.hyb && t.pi_frag == m.pi_frag &&
                      t.frag == m.frag && t.nfrag == m.nfrag && t.qfrag == m.qfrag && t.qa == m.qa &&
                      t.chi_base == m.chi_base && t.gam == m.gam && t.alpeeq == m.alpeeq && t.cnf == m.cnf;
    if (same) return false;
    m.topo_bonds = t.topo_bonds; m.adj = t.adj; m.hyb = t.hyb; m.pi_frag = t.pi_frag;
    m.frag = t.frag; m.nfrag = t.nfrag; m.qfrag = t.qfrag; m.qa = t.qa;
    m.chi_base = t.chi_base; m.gam = t.gam; m.alpeeq = t.alpeeq; m.cnf = t.cnf;
    m.dxi = t.dxi; m.dgam = t.dgam; m.amide_h = t.amide_h; m.topo_cache_hit = t.topo_cache_hit;
    return true;
}

void redetect_hbxb(Model& m, const double* xyz_bohr)
{
    detail::Ctx c(m);
    c.Z = m.Z.data();
    c.xb.assign(xyz_bohr, xyz_bohr + 3 * (size_t)m.n);
    for (auto& b : m.topo_bonds) c.bondset.insert(detail::key(b.first, b.second));
    detail::detect_hbxb(c, c.xb);
}

HBAtoms hb_atom_data(Model& m, const double* xyz_bohr)
{
    detail::Ctx c(m);
    c.Z = m.Z.data();
    c.xb.assign(xyz_bohr, xyz_bohr + 3 * (size_t)m.n);
    for (auto& b : m.topo_bonds) c.bondset.insert(detail::key(b.first, b.second));
    return detail::hb_atoms(c, c.xb);
}

void complete_host_lists(Model& m, const double* hb_xyz_bohr)
{
    detail::Ctx c(m);
    c.Z = m.Z.data();
    for (auto& b : m.topo_bonds) c.bondset.insert(detail::key(b.first, b.second));
    if (m.disp_on_device && m.opt.dispersion) {
        c.xb = m.xyz_setup;
        detail::disp_list(c, detail::half_contraction(m));
    }
    if (m.hb_on_device && m.opt.hbond) {
        c.xb.assign(hb_xyz_bohr, hb_xyz_bohr + 3 * (size_t)m.n);
        detail::detect_hb_terms(c, c.xb, detail::hb_atoms(c, c.xb));
    }
    m.hb_on_device = m.disp_on_device = false;
}

}  // namespace gfnff
