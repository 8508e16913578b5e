// Bonded GFN-FF terms: one thread per term (one warp per bond), gradient scattered with
// FP64 atomics, term energies summed per molecule.  Included by engine.cu (one translation unit).
#pragma once

namespace {

// x^6 (the HB/XB damping exponent is the integer 6)
__device__ __forceinline__ double pow6(double x)
{
    const double x3 = x * x * x;
    return x3 * x3;
}

// ------------------------------------------------------------------------------------
// bonded terms
// ------------------------------------------------------------------------------------
struct BondSoA {
    int n;
    const int *i, *j, *hbh, *hb_off, *hb_b;
    const double *fc, *alpha, *r0i, *r0j, *cki, *ckj, *shift, *ff;
};

// bonds with the HB-modulated exponent and the r0(CN) chain rule
// (ff_workspace_gfnff.cpp:46-182).  One warp per bond: the lanes share the loops over the
// HB acceptors that modulate an X-H bond.
__global__ void __launch_bounds__(kBlock) k_bonds(View V, BondSoA B)
{
    const int t = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    double e = 0.0;
    if (t < B.n) {
        const int i = B.i[t], j = B.j[t];
        D3 pi = ld(V.pos, i), pj = ld(V.pos, j);
        D3 ij = pi - pj;
        const double r = nrm(ij);
        D3 d0 = (1.0 / r) * ij;
        const double r0 = (B.r0i[t] + B.cki[t] * V.cn[i] + B.r0j[t] + B.ckj[t] * V.cn[j] + B.shift[t]) * B.ff[t];
        const double dr = r - r0;
        double alpha = B.alpha[t];
        const int H = B.hbh[t];
        const double kn = 27.5, isp = 0.5641895835477563;
        D3 ph = mk(0.0, 0.0, 0.0);
        if (H >= 0) {
            double hcn = 0.0;
            ph = ld(V.pos, H);
            for (int p = B.hb_off[t] + lane; p < B.hb_off[t + 1]; p += 32) {
                const int b = B.hb_b[p];
                D3 d = ld(V.pos, b) - ph;
                const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                if (r2 > 900.0) continue;
                const double rr = sqrt(r2);
                const double rc = 1.78 * (4.0 / 3.0) * (V.rcov_d3[H] + V.rcov_d3[b]);
                const double arg = -kn * (rr - rc) / rc;
                hcn += 0.5 * (1.0 + erf(arg));
            }
            for (int o = 16; o > 0; o >>= 1) hcn += __shfl_xor_sync(full, hcn, o);
            alpha = (-(1.0 - 0.9) * hcn + 1.0) * B.alpha[t];
        }
        const double eb = B.fc[t] * exp(-alpha * dr * dr);
        const double dEdr = -2.0 * alpha * dr * eb;
        if (lane == 0) {
            e = eb;
            agrad(V.grad, i, dEdr * d0);
            agrad(V.grad, j, (-dEdr) * d0);
            const double yy = -dEdr;
            atomicAdd(V.dEdcn + i, yy * B.ff[t] * B.cki[t]);
            atomicAdd(V.dEdcn + j, yy * B.ff[t] * B.ckj[t]);
        }
        if (H >= 0) {
            const double zz = 0.1 * B.alpha[t] * dr * dr * eb;
            D3 gh = mk(0.0, 0.0, 0.0);
            for (int p = B.hb_off[t] + lane; p < B.hb_off[t + 1]; p += 32) {
                const int b = B.hb_b[p];
                D3 d = ld(V.pos, b) - ph;
                const double r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                if (r2 > 900.0) continue;
                const double rr = sqrt(r2);
                const double rc = 1.78 * (4.0 / 3.0) * (V.rcov_d3[H] + V.rcov_d3[b]);
                const double arg = -kn * (rr - rc) / rc;
                const double dcn = isp * (-kn / rc) * exp(-arg * arg) / rr;
                gh = gh + (zz * -dcn) * d;
                agrad(V.grad, b, (zz * dcn) * d);
            }
            for (int o = 16; o > 0; o >>= 1) {
                gh.x += __shfl_xor_sync(full, gh.x, o);
                gh.y += __shfl_xor_sync(full, gh.y, o);
                gh.z += __shfl_xor_sync(full, gh.z, o);
            }
            if (lane == 0) agrad(V.grad, H, gh);
        }
    }
    eadd(V, e, t < B.n ? V.mol[B.i[t]] : -1, T_BOND);
}

struct AngleSoA {
    int n;
    const int *i, *j, *k;
    const double *fc, *th0;
};

// angles with distance damping (ff_workspace_gfnff.cpp:187-280)
__global__ void k_angles(View V, AngleSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int ia = A.i[t], ja = A.j[t], ka = A.k[t];
        D3 pi = ld(V.pos, ia), pj = ld(V.pos, ja), pk = ld(V.pos, ka), d[3];
        double c = angle_cos(pi, pj, pk, d);
        c = fmax(-1.0, fmin(1.0, c));
        const double th = acos(c), th0 = A.th0[t], fc = A.fc[t];
        double e, dedth;
        if (fabs(kPi - th0) < 1e-6) {
            const double dt = th - th0;
            e = fc * dt * dt;
            dedth = 2.0 * fc * dt;
        } else {
            const double c0 = cos(th0), dc = c - c0;
            e = fc * dc * dc;
            dedth = 2.0 * fc * sin(th) * (c0 - c);
        }
        const double rij2 = dot(pi - pj, pi - pj), rjk2 = dot(pk - pj, pk - pj);
        const double ri = V.rcov43[ia], rj = V.rcov43[ja], rk = V.rcov43[ka];
        const double cij = 0.595 * (ri + rj) * (ri + rj), cjk = 0.595 * (rj + rk) * (rj + rk);
        double a1 = rij2 / cij; a1 = a1 * a1;
        double a2 = rjk2 / cjk; a2 = a2 * a2;
        const double dij = 1.0 / (1.0 + a1), djk = 1.0 / (1.0 + a2), damp = dij * djk;
        const double e2ij = rij2 > 1e-8 ? -2.0 * 2.0 * a1 / (rij2 * (1.0 + a1) * (1.0 + a1)) : 0.0;
        const double e2jk = rjk2 > 1e-8 ? -2.0 * 2.0 * a2 / (rjk2 * (1.0 + a2) * (1.0 + a2)) : 0.0;
        et = e * damp;
        D3 t1 = (e * e2ij * djk) * (pi - pj), t2 = (e * e2jk * dij) * (pk - pj);
        agrad(V.grad, ia, (dedth * damp) * d[0] + t1);
        agrad(V.grad, ja, (dedth * damp) * d[1] - t1 - t2);
        agrad(V.grad, ka, (dedth * damp) * d[2] + t2);
    }
    eadd(V, et, t < A.n ? V.mol[A.i[t]] : -1, T_ANGLE);
}

struct TorsSoA {
    int n;
    const int *i, *j, *k, *l;
    const double *V, *nn, *phi0;
};

// torsions + extra torsions (ff_workspace_gfnff.cpp:282-487), triple-bond torsions
// (:611-653) when storsion = true
__global__ void k_torsions(View V, TorsSoA T, int storsion)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < T.n) {
        const int a = T.i[t], b = T.j[t], c = T.k[t], d = T.l[t];
        D3 ri = ld(V.pos, a), rj = ld(V.pos, b), rk = ld(V.pos, c), rl = ld(V.pos, d), g[4];
        const double phi = dihedral(ri, rj, rk, rl, g);
        if (storsion) {
            const double eh = T.V[t];
            et = -eh * cos(2.0 * phi) + eh;
            const double dEdphi = 2.0 * eh * sin(2.0 * phi);
            agrad(V.grad, a, dEdphi * g[0]);
            agrad(V.grad, b, dEdphi * g[1]);
            agrad(V.grad, c, dEdphi * g[2]);
            agrad(V.grad, d, dEdphi * g[3]);
        } else {
            const double Vb = T.V[t], n = T.nn[t];
            const double c1 = n * (phi - T.phi0[t]) + kPi;
            const double e = Vb * (1.0 + cos(c1));
            const double rij2 = dot(ri - rj, ri - rj), rjk2 = dot(rj - rk, rj - rk), rkl2 = dot(rk - rl, rk - rl);
            const double qa = V.rcov43[a], qb = V.rcov43[b], qc = V.rcov43[c], qd = V.rcov43[d];
            const double cij = 0.505 * (qa + qb) * (qa + qb), cjk = 0.505 * (qb + qc) * (qb + qc),
                         ckl = 0.505 * (qc + qd) * (qc + qd);
            double a1 = rij2 / cij; a1 *= a1;
            double a2 = rjk2 / cjk; a2 *= a2;
            double a3 = rkl2 / ckl; a3 *= a3;
            const double dij = 1.0 / (1.0 + a1), djk = 1.0 / (1.0 + a2), dkl = 1.0 / (1.0 + a3);
            const double damp = dij * djk * dkl;
            et = e * damp;
            const double dEdphi = -Vb * n * sin(c1) * damp;
            const double e2ij = rij2 > 1e-8 ? -4.0 * a1 / (rij2 * (1.0 + a1) * (1.0 + a1)) : 0.0;
            const double e2jk = rjk2 > 1e-8 ? -4.0 * a2 / (rjk2 * (1.0 + a2) * (1.0 + a2)) : 0.0;
            const double e2kl = rkl2 > 1e-8 ? -4.0 * a3 / (rkl2 * (1.0 + a3) * (1.0 + a3)) : 0.0;
            D3 t1 = (e * e2ij * djk * dkl) * (ri - rj), t2 = (e * dij * e2jk * dkl) * (rj - rk),
               t3 = (e * dij * djk * e2kl) * (rk - rl);
            agrad(V.grad, a, dEdphi * g[0] + t1);
            agrad(V.grad, b, dEdphi * g[1] + t2 - t1);
            agrad(V.grad, c, dEdphi * g[2] + t3 - t2);
            agrad(V.grad, d, dEdphi * g[3] - t3);
        }
    }
    eadd(V, et, t < T.n ? V.mol[T.i[t]] : -1, storsion ? T_STORSION : T_TORSION);
}

struct InvSoA {
    int n;
    const int *i, *j, *k, *l, *type;
    const double *fc, *om0;
};

// inversions (ff_workspace_gfnff.cpp:489-609)
__global__ void k_inversions(View V, InvSoA I)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < I.n) {
        const int a = I.i[t], b = I.j[t], c = I.k[t], d = I.l[t];
        D3 rc = ld(V.pos, a), r1 = ld(V.pos, b), r2 = ld(V.pos, c), r3 = ld(V.pos, d), g[4];
        const double om = oop(rc, r1, r2, r3, g);
        const double ci = V.rcov43[a], c1 = V.rcov43[b], c2 = V.rcov43[c], c3 = V.rcov43[d];
        auto damp = [](double rsq, double x, double y) {
            const double cut = 0.505 * (x + y) * (x + y);
            const double rr = (rsq / cut) * (rsq / cut);
            return 1.0 / (1.0 + rr);
        };
        auto ddamp = [](double rsq, double x, double y) {
            if (rsq < 1e-8) return 0.0;
            const double cut = 0.505 * (x + y) * (x + y);
            const double rr = (rsq / cut) * (rsq / cut);
            return -4.0 * rr / (rsq * (1.0 + rr) * (1.0 + rr));
        };
        const double rij2 = dot(r1 - rc, r1 - rc), rjk2 = dot(r1 - r2, r1 - r2), rjl2 = dot(r1 - r3, r1 - r3);
        const double dij = damp(rij2, ci, c1), djk = damp(rjk2, c2, c1), djl = damp(rjl2, c1, c3);
        const double dmp = dij * djk * djl;
        double et, dEdom;
        const double fc = I.fc[t];
        if (I.type[t] == 0) {
            et = fc * (1.0 - cos(om));
            dEdom = fc * sin(om) * dmp;
        } else {
            const double df = cos(om) - cos(I.om0[t]);
            et = fc * df * df;
            dEdom = -2.0 * fc * sin(om) * df * dmp;
        }
        etot = et * dmp;
        const double e1 = ddamp(rij2, ci, c1), e2 = ddamp(rjk2, c2, c1), e3 = ddamp(rjl2, c1, c3);
        D3 t1 = (et * e1 * djk * djl) * (r1 - rc), t2 = (et * e2 * dij * djl) * (r1 - r2),
           t3 = (et * e3 * dij * djk) * (r1 - r3);
        agrad(V.grad, a, dEdom * g[0] - t1);
        agrad(V.grad, b, dEdom * g[1] + t1 + t2 + t3);
        agrad(V.grad, c, dEdom * g[2] - t2);
        agrad(V.grad, d, dEdom * g[3] - t3);
    }
    eadd(V, etot, t < I.n ? V.mol[I.i[t]] : -1, T_INVERSION);
}

struct TripSoA {
    int n;
    const int *i, *j, *k;
    const double *c9, *r0ij, *r0ik, *r0jk, *scale;   // ATM; BATM uses c9 only
};

// D4 ATM over bonded triplets (ff_workspace_gfnff.cpp:1526-1663)
__global__ void k_atm(View V, TripSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int a = A.i[t], b = A.j[t], c = A.k[t];
        D3 pi = ld(V.pos, a), pj = ld(V.pos, b), pk = ld(V.pos, c);
        D3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double rij = nrm(vij), rik = nrm(vik), rjk = nrm(vjk);
        const double r2ij = rij * rij, r2ik = rik * rik, r2jk = rjk * rjk;
        const double c9 = A.c9[t];
        const double rijk = rij * rik * rjk, r2ijk = r2ij * r2ik * r2jk, r3ijk = rijk * r2ijk;
        const double tmp = pow(A.r0ij[t] * A.r0ik[t] * A.r0jk[t] / rijk, 14.0 / 3.0);
        const double fdmp = 1.0 / (1.0 + 6.0 * tmp);
        const double X = r2ij + r2jk - r2ik, Y = r2ij + r2ik - r2jk, Zc = r2ik + r2jk - r2ij;
        const double ang = (0.375 * X * Y * Zc / r2ijk + 1.0) / r3ijk;
        const double sc = A.scale[t];
        et = ang * fdmp * c9 / 3.0 * sc;
        const double r5ijk = r2ijk * r3ijk;
        const double dfdmp = -2.0 * 14.0 * tmp * fdmp * fdmp;
        const double dij = -0.375 * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik) +
                                     r2ij * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ik + 3.0 * r2ik * r2ik) -
                                     5.0 * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) / r5ijk;
        const double dik = -0.375 * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij) +
                                     r2ik * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) / r5ijk;
        const double djk = -0.375 * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij) +
                                     r2jk * (3.0 * r2ik * r2ik + 2.0 * r2ik * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) / r5ijk;
        const double pre = -c9 * sc / 3.0;
        D3 gij = (pre * (-dij * fdmp + ang * dfdmp) / r2ij) * vij;
        D3 gik = (pre * (-dik * fdmp + ang * dfdmp) / r2ik) * vik;
        D3 gjk = (pre * (-djk * fdmp + ang * dfdmp) / r2jk) * vjk;
        agrad(V.grad, a, -1.0 * (gij + gik));
        agrad(V.grad, b, gij - gjk);
        agrad(V.grad, c, gik + gjk);
    }
    eadd(V, et, t < A.n ? V.mol[A.i[t]] : -1, T_ATM);
}

// bonded ATM with the Phase-1 charge factors folded into c9 (ff_workspace_gfnff.cpp:1665-1739)
__global__ void k_batm(View V, TripSoA A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double et = 0.0;
    if (t < A.n) {
        const int a = A.i[t], b = A.j[t], c = A.k[t];
        D3 pi = ld(V.pos, a), pj = ld(V.pos, b), pk = ld(V.pos, c);
        D3 vij = pj - pi, vik = pk - pi, vjk = pk - pj;
        const double r2ij = dot(vij, vij), r2jk = dot(vjk, vjk), r2ik = dot(vik, vik);
        const double rij = sqrt(r2ij), rjk = sqrt(r2jk), rik = sqrt(r2ik);
        const double rijk3 = r2ij * r2jk * r2ik;
        const double mijk = -r2ij + r2jk + r2ik, imjk = r2ij - r2jk + r2ik, ijmk = r2ij + r2jk - r2ik;
        const double ang = 0.375 * ijmk * imjk * mijk / rijk3;
        const double rav3 = pow(rijk3, 1.5);
        const double c9 = A.c9[t];
        et = c9 * ((ang + 1.0) / rav3);
        const double den = rijk3 * rav3;
        const double dij = -0.375 * (r2ij * r2ij * r2ij + r2ij * r2ij * (r2jk + r2ik) +
                                     r2ij * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ik + 3.0 * r2ik * r2ik) -
                                     5.0 * (r2jk - r2ik) * (r2jk - r2ik) * (r2jk + r2ik)) / (rij * den);
        const double djk = -0.375 * (r2jk * r2jk * r2jk + r2jk * r2jk * (r2ik + r2ij) +
                                     r2jk * (3.0 * r2ik * r2ik + 2.0 * r2ik * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2ik - r2ij) * (r2ik - r2ij) * (r2ik + r2ij)) / (rjk * den);
        const double dik = -0.375 * (r2ik * r2ik * r2ik + r2ik * r2ik * (r2jk + r2ij) +
                                     r2ik * (3.0 * r2jk * r2jk + 2.0 * r2jk * r2ij + 3.0 * r2ij * r2ij) -
                                     5.0 * (r2jk - r2ij) * (r2jk - r2ij) * (r2jk + r2ij)) / (rik * den);
        D3 gij = (-dij * c9 / rij) * vij, gjk = (-djk * c9 / rjk) * vjk, gik = (-dik * c9 / rik) * vik;
        agrad(V.grad, b, gjk - gij);
        agrad(V.grad, c, -1.0 * gik - gjk);
        agrad(V.grad, a, gij + gik);
    }
    eadd(V, et, t < A.n ? V.mol[A.i[t]] : -1, T_BATM);
}

struct HBSoA {
    int n;
    const int *a, *h, *b, *cas, *pc, *nbb_off, *nbb, *nbc_off, *nbc;
    const double *bas_a, *bas_b, *aci_a, *aci_b, *QH, *QA, *QB, *rv, *zlp;
    const int* nflag;   // acceptor is N with a single neighbour: neighbour cutoff 2.0
};

// hydrogen bonds, cases 1-4 (ff_workspace_gfnff.cpp:938-1409)
__global__ void __launch_bounds__(kBlock) k_hbonds(View V, HBSoA S)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < S.n) {
        const double HB_BACUT = 49.0, HB_SCUT = 22.0, HB_ALP = 6.0, HB_LONGCUT = 85.0, HB_NBCUT = 11.20;
        const double TORS_HB = 0.94, BEND_HB = 0.20, HBLPCUT = 56.0;
        const int A = S.a[t], H = S.h[t], Bq = S.b[t], cs = S.cas[t];
        D3 pA = ld(V.pos, A), pH = ld(V.pos, H), pB = ld(V.pos, Bq);
        const double rAH = nrm(pH - pA), rHB = nrm(pB - pH), rAB = nrm(pB - pA);
        if (rAB <= 50.0) {
            const double rAH4 = rAH * rAH * rAH * rAH, rHB4 = rHB * rHB * rHB * rHB;
            const double den = 1.0 / (rAH4 + rHB4);
            const double QH = S.QH[t], QA = S.QA[t], QB = S.QB[t];
            const double bas = (QA * S.bas_a[t] * rAH4 + QB * S.bas_b[t] * rHB4) * den;
            const double aci = (S.aci_b[t] * rAH4 + S.aci_a[t] * rHB4) * den;
            const double rv = S.rv[t];
            // HB_ALP = 6: integer powers
            const double ratio1 = pow6(rAB * rAB / HB_LONGCUT);
            const double ratio3 = pow6(HB_SCUT * rv / (rAB * rAB));
            const double dsh = 1.0 / (1.0 + ratio3);
            const double dlg = 1.0 / (1.0 + ratio1);
            const double denv = dsh * dlg;
            double doutl;
            {
                const double ex = (HB_BACUT / rv) * ((rAH + rHB) / rAB - 1.0);
                doutl = ex > 15.0 ? 0.0 : 2.0 / (1.0 + exp(ex));
            }
            const int nb0 = S.nbb_off[t], nb1 = S.nbb_off[t + 1];
            const double nbcut = S.nflag[t] ? 2.0 : HB_NBCUT;
            double onb = 1.0;
            if (cs >= 2)
                for (int p = nb0; p < nb1; ++p) {
                    D3 pn = ld(V.pos, S.nbb[p]);
                    const double ra = nrm(pn - pA), rb = nrm(pn - pB);
                    const double ex = (nbcut / rv) * ((ra + rb) / rAB - 1.0);
                    onb *= (2.0 / (1.0 + exp(-ex)) - 1.0);
                }
            const double rdamp = cs >= 2 ? denv * (1.8 / (rHB * rHB * rHB) - 0.8 / (rAB * rAB * rAB))
                                         : denv / (rAB * rAB * rAB);
            double olp = 1.0, lpd = 0.0;
            int nlp = 0;
            D3 lpv = mk(0, 0, 0), lpp = pB;
            if (cs == 4) {
                lpd = 0.50 - 0.018 * S.zlp[t];
                nlp = nb1 - nb0;
                for (int p = nb0; p < nb1; ++p) lpv = lpv + (ld(V.pos, S.nbb[p]) - pB);
                const double vn = nrm(lpv);
                if (vn > 1e-10 && nlp > 0) {
                    lpp = pB + (-lpd) * ((1.0 / vn) * lpv);
                    const double ral = nrm(pA - lpp);
                    const double ex = (HBLPCUT / rv) * ((ral + lpd + 1e-12) / rAB - 1.0);
                    olp = 2.0 / (1.0 + exp(ex));
                } else {
                    nlp = 0;
                    olp = 1.0;
                }
            }
            const double qhoutl = QH * doutl * onb * olp;
            double eangl = 1.0, etors = 1.0;
            D3 ga3[3] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)};
            const int Ci = S.pc[t];
            const bool c3 = (cs == 3 && Ci != -1);
            if (c3) {
                const double c0 = 120.0 * kPi / 180.0;
                const double kijk = (1.0 - BEND_HB) / ((cos(0.0) - cos(c0)) * (cos(0.0) - cos(c0)));
                D3 va = ld(V.pos, Ci), vb = pB, vc = pH;
                D3 vab = va - vb, vcb = vc - vb;
                const double rab2 = dot(vab, vab), rcb2 = dot(vcb, vcb);
                D3 vp = cross(vcb, vab);
                const double rp = nrm(vp) + 1e-14;
                double ca = dot(vab, vcb) / (sqrt(rab2) * sqrt(rcb2) + 1e-14);
                ca = fmax(-1.0, fmin(1.0, ca));
                const double th = acos(ca);
                const double ea = kijk * (ca - cos(c0)) * (ca - cos(c0));
                const double deddt = 2.0 * kijk * sin(th) * (cos(c0) - ca);
                eangl = 1.0 - ea;
                D3 deda = (-deddt / (rab2 * rp)) * cross(vab, vp);
                D3 dedc = (deddt / (rcb2 * rp)) * cross(vcb, vp);
                ga3[0] = deda + dedc;
                ga3[1] = -1.0 * deda;
                ga3[2] = -1.0 * dedc;
                for (int p = S.nbc_off[t]; p < S.nbc_off[t + 1]; ++p) {
                    const int D = S.nbc[p];
                    if (D == Bq) continue;
                    D3 g[4];
                    const double phi = dihedral(ld(V.pos, D), pB, va, pH, g);
                    const double fct = (1.0 - TORS_HB) / 2.0;
                    const double c1 = 2 * (phi - kPi / 2.0) + kPi;
                    etors *= (1.0 + cos(c1)) * fct + TORS_HB;
                }
            }
            double gs = 1.0;
            if (cs == 2 || cs == 4) gs = 0.268;
            else if (cs == 3) gs = 0.350;
            const double cst = S.aci_a[t] * S.bas_b[t] * QA * QB * gs;
            const double E = cs >= 2 ? -rdamp * qhoutl * cst * eangl * etors : -bas * aci * rdamp * qhoutl;
            etot = E;

            D3 drab = pA - pB, drah = pA - pH, drbh = pB - pH;
            const double rab2 = rAB * rAB, rbh2 = rHB * rHB, rah2 = rAH * rAH;
            const double rahprbh = rAH + rHB + 1e-12;
            const double ddamp = (-2.0 * HB_ALP * ratio1 / (1.0 + ratio1)) + (2.0 * HB_ALP * ratio3 / (1.0 + ratio3));
            const double expo = (HB_BACUT / rv) * (rahprbh / rAB - 1.0);
            if (expo <= 15.0) {
                const double ratio2 = exp(expo);
                D3 ga = mk(0, 0, 0), gb = mk(0, 0, 0), gh = mk(0, 0, 0);
                if (cs >= 2) {
                    const double rbhdamp = denv * 1.8 / (rbh2 * rHB);
                    const double rabdamp = denv * (-0.8) / (rab2 * rAB);
                    const double dterm = -qhoutl * eangl * etors * cst;
                    const double aterm = -rdamp * QH * onb * olp * eangl * etors * cst;
                    const double nbterm = -rdamp * QH * doutl * olp * eangl * etors * cst;
                    double gi = ((rabdamp + rbhdamp) * ddamp - 3.0 * rabdamp) / rab2;
                    gi *= dterm;
                    D3 dg = gi * drab;
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
                    D3 dgao = (tmp1 / rAH) * drah, dgbo = (tmp1 / rHB) * drbh;
                    ga = ga + dgao;
                    gb = gb + dgbo;
                    gh = gh - dgao - dgbo;
                    for (int p = nb0; p < nb1; ++p) {
                        const int nb = S.nbb[p];
                        D3 pn = ld(V.pos, nb);
                        D3 dranb = pA - pn, drbnb = pB - pn;
                        const double ranb = nrm(dranb), rbnb = nrm(drbnb);
                        const double sum = ranb + rbnb + 1e-12;
                        const double ex = (nbcut / rv) * (sum / rAB - 1.0);
                        const double r2n = exp(-ex);
                        const double oi = 2.0 / (1.0 + r2n) - 1.0;
                        const double others = fabs(oi) > 1e-12 ? onb / oi : 1.0;
                        const double tmp2 = 2.0 * nbterm * others * r2n * ex / ((1.0 + r2n) * (1.0 + r2n)) / (sum - rAB);
                        dg = (-tmp2 * sum / rab2) * drab;
                        ga = ga + dg;
                        gb = gb - dg;
                        D3 dgan = (tmp2 / ranb) * dranb, dgbn = (tmp2 / rbnb) * drbnb;
                        ga = ga + dgan;
                        gb = gb + dgbn;
                        agrad(V.grad, nb, -1.0 * dgan - dgbn);
                    }
                    if (cs == 4 && nlp > 0) {
                        const double lpterm = -rdamp * QH * doutl * onb * cst;
                        const double ral = nrm(pA - lpp);
                        const double sum = ral + lpd + 1e-12;
                        const double ex = (HBLPCUT / rv) * (sum / rAB - 1.0);
                        const double r2l = exp(ex);
                        const double tmp3 = -2.0 * lpterm * r2l * ex / ((1.0 + r2l) * (1.0 + r2l)) / (sum - rAB);
                        D3 dgl = (-tmp3 * sum / rab2) * drab;
                        ga = ga + dgl;
                        gb = gb - dgl;
                        D3 dral = pA - lpp;
                        D3 dgal = (tmp3 / (ral + 1e-12)) * dral;
                        ga = ga + dgal;
                        gb = gb - dgal;
                        D3 glp = -1.0 * dgal;
                        const double vn = nrm(lpv);
                        if (vn > 1e-10) {
                            const double lv[3] = {lpv.x, lpv.y, lpv.z}, gl3[3] = {glp.x, glp.y, glp.z};
                            double out[3] = {0, 0, 0};
                            const double vn3 = vn * vn * vn;
                            for (int col = 0; col < 3; ++col)
                                for (int row = 0; row < 3; ++row) {
                                    const double unit = (row == col) ? -1.0 : 0.0;
                                    out[row] += -lpd * (double)nlp * (unit / vn + lv[row] * lv[col] / vn3) * gl3[col];
                                }
                            D3 gnb = mk(out[0], out[1], out[2]);
                            gb = gb + gnb;
                            D3 share = (1.0 / (double)nlp) * gnb;
                            for (int p = nb0; p < nb1; ++p) agrad(V.grad, S.nbb[p], -1.0 * share);
                        }
                    }
                    if (c3) {
                        const double bterm = -rdamp * qhoutl * etors * cst;
                        const double tterm = -rdamp * qhoutl * eangl * cst;
                        agrad(V.grad, Bq, bterm * ga3[0]);
                        agrad(V.grad, Ci, bterm * ga3[1]);
                        agrad(V.grad, H, bterm * ga3[2]);
                        D3 va = ld(V.pos, Ci);
                        for (int p = S.nbc_off[t]; p < S.nbc_off[t + 1]; ++p) {
                            const int D = S.nbc[p];
                            if (D == Bq) continue;
                            D3 g[4];
                            const double phi = dihedral(ld(V.pos, D), pB, va, pH, g);
                            const double fct = (1.0 - TORS_HB) / 2.0;
                            const double c1 = 2 * (phi - kPi / 2.0) + kPi;
                            const double ek = (1.0 + cos(c1)) * fct + TORS_HB;
                            const double dij = -2 * sin(c1) * fct;
                            const double fk = fabs(ek) > 1e-12 ? etors / ek : 0.0;
                            const double tk = fk * tterm;
                            agrad(V.grad, D, (tk * dij) * g[0]);
                            agrad(V.grad, Bq, (tk * dij) * g[1]);
                            agrad(V.grad, Ci, (tk * dij) * g[2]);
                            agrad(V.grad, H, (tk * dij) * g[3]);
                        }
                    }
                } else {
                    const double caa = QA * S.bas_a[t], cbb = QB * S.bas_b[t];
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
                    gi = (S.aci_b[t] - S.aci_a[t]) * dd24a;
                    D3 dga = (gi * sterm) * drah;
                    ga = ga + dga;
                    gi = (S.aci_a[t] - S.aci_b[t]) * dd24b;
                    D3 dgb = (gi * sterm) * drbh;
                    gb = gb + dgb;
                    gh = gh - dga - dgb;
                    gi = rdamp * (ddamp - 3.0) / rab2;
                    D3 dg = (gi * dterm) * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    gi = aterm * 2.0 * ratio2 * expo * rahprbh / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB) / rab2;
                    dg = gi * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    const double to = -2.0 * aterm * ratio2 * expo / ((1.0 + ratio2) * (1.0 + ratio2)) / (rahprbh - rAB);
                    D3 dgao = (to / rAH) * drah, dgbo = (to / rHB) * drbh;
                    ga = ga + dgao;
                    gb = gb + dgbo;
                    gh = gh - dgao - dgbo;
                }
                agrad(V.grad, A, ga);
                agrad(V.grad, Bq, gb);
                agrad(V.grad, H, gh);
            }
        }
    }
    eadd(V, etot, t < S.n ? V.mol[S.a[t]] : -1, T_HB);
}

struct XBSoA {
    int n;
    const int *a, *x, *b;
    const double *pre, *rv;
};

// halogen bonds (ff_workspace_gfnff.cpp:1411-1524); pre = -Q_B * acidity_X * Q_X
__global__ void k_xbonds(View V, XBSoA S)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double etot = 0.0;
    if (t < S.n) {
        const double XB_BACUT = 70.0, XB_SCUT = 5.0, ALP = 6.0, LC = 70.0;
        D3 pA = ld(V.pos, S.a[t]), pX = ld(V.pos, S.x[t]), pB = ld(V.pos, S.b[t]);
        D3 vAX = pX - pA, vXB = pB - pX, vAB = pB - pA;
        const double rAX = nrm(vAX), rXB = nrm(vXB), rAB = nrm(vAB);
        const double ex = XB_BACUT * ((rAX + rXB) / rAB - 1.0);
        if (rXB <= 20.0 && ex <= 15.0) {
            const double rv = S.rv[t];
            const double dsh = 1.0 / (1.0 + pow6(XB_SCUT * rv / (rXB * rXB)));
            const double dlg = 1.0 / (1.0 + pow6(rXB * rXB / LC));
            const double dol = 2.0 / (1.0 + exp(ex));
            const double r3 = rXB * rXB * rXB;
            const double R = dsh * dlg * dol / r3;
            const double pre = S.pre[t];
            etot = R * pre;
            const double st = pow6(XB_SCUT * rv / (rXB * rXB));
            const double dds = -2.0 * ALP * dsh * st / (rXB * (1.0 + st));
            const double lt = pow6((rXB * rXB) / LC);
            const double ddl = -2.0 * ALP * rXB * dlg * lt / (LC * (1.0 + lt));
            const double et = exp(ex), de = 1.0 + et;
            const double do_ax = -2.0 * et * XB_BACUT / (rAB * de * de);
            const double do_ab = 2.0 * et * XB_BACUT * (rAX + rXB) / (rAB * rAB * de * de);
            const double dR_xb = (dds * dlg * dol + dsh * ddl * dol + dsh * dlg * do_ax) / r3 - 3.0 * R / rXB;
            const double eXB = pre * dR_xb, eAX = pre * dsh * dlg * do_ax / r3, eAB = pre * dsh * dlg * do_ab / r3;
            D3 uAX = (1.0 / (rAX + 1e-14)) * vAX, uXB = (1.0 / (rXB + 1e-14)) * vXB, uAB = (1.0 / (rAB + 1e-14)) * vAB;
            agrad(V.grad, S.a[t], -eAX * uAX - eAB * uAB);
            agrad(V.grad, S.x[t], eAX * uAX - eXB * uXB);
            agrad(V.grad, S.b[t], eXB * uXB + eAB * uAB);
        }
    }
    eadd(V, etot, t < S.n ? V.mol[S.a[t]] : -1, T_XB);
}

}  // namespace
