// Bonded GFN-FF terms: one thread per term (one warp per bond), gradient scattered with
// FP64 atomics, term energies summed per molecule.  Included by engine.cu (one translation unit).
#pragma once

// resident blocks per SM requested for the FP64 HB kernel: 4 caps it at 128 registers (a
// few spills), which measured 1.5x faster than the uncapped 190 registers at 2 blocks per
// SM.  The FP32 form needs 94 registers without spills and asks for 5 blocks.
#ifndef GFNFF_HB_MINBLOCKS
#define GFNFF_HB_MINBLOCKS 4
#endif

namespace {

// x^6 (the HB/XB damping exponent is the integer 6)
template <class R = double>
__device__ __forceinline__ R pow6(R x)
{
    const R x3 = x * x * x;
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
        const D3 ij = dmic(V, j, i);
        const double r = nrm(ij);
        D3 d0 = (1.0 / r) * ij;
        const double r0 = (B.r0i[t] + B.cki[t] * V.cn[i] + B.r0j[t] + B.ckj[t] * V.cn[j] + B.shift[t]) * B.ff[t];
        const double dr = r - r0;
        double alpha = B.alpha[t];
        const int H = B.hbh[t];
        const double kn = 27.5, isp = 0.5641895835477563;
        if (H >= 0) {
            double hcn = 0.0;
            for (int p = B.hb_off[t] + lane; p < B.hb_off[t + 1]; p += 32) {
                const int b = B.hb_b[p];
                const D3 d = dmic(V, H, b);
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
                const D3 d = dmic(V, H, b);
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
        // the two arms from the apex (minimum image with a cell); the apex is the origin
        const D3 pi = dmic(V, ja, ia), pj = mk(0.0, 0.0, 0.0), pk = dmic(V, ja, ka);
        D3 d[3];
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
    const int4* rec;                                     // per term {A, H, B, case}
    const double *qh, *qa, *bas, *aci, *rvdw, *zlp;      // per atom
    const int *pc, *nflag, *adj_off, *adj;               // per atom: carbonyl parent, N with one
                                                         // neighbour (cutoff 2.0), bond graph CSR
};

// Arithmetic of the HB kernel.  FP64 keeps IEEE operations but divides by reciprocals
// computed once per distance; FP32 (only the weak, strongly damped terms of the mixed
// form) uses the hardware approximations of 1/x, exp and 1/sqrt (relative error ~1e-7).
template <class R>
__device__ __forceinline__ R hb_rcp(R x) { return R(1.0) / x; }
template <>
__device__ __forceinline__ float hb_rcp<float>(float x) { return __fdividef(1.0f, x); }
template <class R>
__device__ __forceinline__ R hb_exp(R x) { return exp(x); }
template <>
__device__ __forceinline__ float hb_exp<float>(float x) { return __expf(x); }
// |v| and 1/|v| from one reciprocal square root
template <class R>
__device__ __forceinline__ R hb_len(V3<R> v, R& inv)
{
    const R d2 = dot(v, v);
    inv = rsqrt(d2);
    return d2 * inv;
}

// hydrogen bonds, cases 1-4 (ff_workspace_gfnff.cpp:938-1409).  R = double is the FP64
// form; R = float evaluates the term in FP32 relative to the H atom (the FP64 position
// differences are taken first), energies and gradients accumulate in FP64.  The damping
// derivatives use d(ex)/d(sum) = (cut / rv) / rAB in closed form instead of the
// reference's ex / (sum - rAB), which is the same value but 0/0 for collinear atoms.
// One thread per HB term of the range [t0, t1).  The list is sorted by the setup
// distance r_AB and split at 10 bohr: the mixed form evaluates the real hydrogen bonds
// before the split (up to ~0.01 Eh each) with R = double and only the weak remainder with
// R = float, because the FP32 rounding of per-element-pair constants is the same for
// every strong bond and would add up over thousands of them.
template <class R, bool CELL = false>
__global__ void __launch_bounds__(kBlock, sizeof(R) == 4 ? 5 : GFNFF_HB_MINBLOCKS) k_hbonds(View V, HBSoA S, int t0,
                                                                                        int t1)
{
    const int t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
    R etot = R(0.0);
    const int4 rec = t < t1 ? S.rec[t] : make_int4(-1, 0, 0, 0);
    if (t < t1) {
        using P3 = V3<R>;
        const double4 org = V.pos[rec.y];   // H as the local origin
        const R HB_BACUT = R(49.0), HB_SCUT = R(22.0), HB_ALP = R(6.0), HB_NBCUT = R(11.20);
        const R TORS_HB = R(0.94), BEND_HB = R(0.20), HBLPCUT = R(56.0);
        const int A = rec.x, H = rec.y, Bq = rec.z, cs = rec.w;
        P3 pA = ldr<R>(V.pos, A, org), pH = ldr<R>(V.pos, H, org), pB = ldr<R>(V.pos, Bq, org);
        // A-H, H-B and A-B: minimum-image vectors in a periodic cell (CELL); the acceptor-
        // neighbour, lone-pair and carbonyl vectors below stay plain differences, as in
        // curcuma's CUDA kernel
        P3 vAH = pH - pA, vHB = pB - pH, vAB = pB - pA;
        if constexpr (CELL) {
            const D3 a = dmic(V, A, H), b = dmic(V, H, Bq), c = dmic(V, A, Bq);
            vAH = P3{(R)a.x, (R)a.y, (R)a.z};
            vHB = P3{(R)b.x, (R)b.y, (R)b.z};
            vAB = P3{(R)c.x, (R)c.y, (R)c.z};
        }
        R irAH, irHB, irAB;
        const R rAH = hb_len(vAH, irAH), rHB = hb_len(vHB, irHB), rAB = hb_len(vAB, irAB);
        if (rAB <= R(50.0)) {
            const R rAH4 = rAH * rAH * rAH * rAH, rHB4 = rHB * rHB * rHB * rHB;
            const R den = hb_rcp(rAH4 + rHB4);
            const R QH = S.qh[H], QA = S.qa[A], QB = S.qa[Bq];
            const double bas_a = S.bas[A], bas_b = S.bas[Bq], aci_a = S.aci[A], aci_b = S.aci[Bq];
            const R bas = (QA * R(bas_a) * rAH4 + QB * R(bas_b) * rHB4) * den;
            const R aci = (R(aci_b) * rAH4 + R(aci_a) * rHB4) * den;
            const R rv = R(S.rvdw[A] + S.rvdw[Bq]);
            const R irv = hb_rcp(rv);
            const R rab2 = rAB * rAB, irab2 = irAB * irAB;
            // HB_ALP = 6: integer powers
            const R ratio1 = pow6<R>(rab2 * R(1.0 / 85.0));   // (r_AB^2 / HB_LONGCUT)^6
            const R ratio3 = pow6<R>(HB_SCUT * rv * irab2);
            const R dsh = hb_rcp(R(1.0) + ratio3);
            const R dlg = hb_rcp(R(1.0) + ratio1);
            const R denv = dsh * dlg;
            const R bacut = HB_BACUT * irv;
            R doutl;
            {
                const R ex = bacut * ((rAH + rHB) * irAB - R(1.0));
                doutl = ex > R(15.0) ? R(0.0) : R(2.0) * hb_rcp(R(1.0) + hb_exp(ex));
            }
            const int nb0 = S.adj_off[Bq], nb1 = S.adj_off[Bq + 1];
            const R nbc = (S.nflag[Bq] ? R(2.0) : HB_NBCUT) * irv;
            R onb = R(1.0);
            if (cs >= 2)
                for (int p = nb0; p < nb1; ++p) {
                    P3 pn = ldr<R>(V.pos, S.adj[p], org);
                    R ia, ib;
                    const R ra = hb_len(pn - pA, ia), rb = hb_len(pn - pB, ib);
                    const R ex = nbc * ((ra + rb) * irAB - R(1.0));
                    onb *= (R(2.0) * hb_rcp(R(1.0) + hb_exp(-ex)) - R(1.0));
                }
            const R irHB3 = irHB * irHB * irHB, irAB3 = irAB * irAB * irAB;
            const R rdamp = cs >= 2 ? denv * (R(1.8) * irHB3 - R(0.8) * irAB3) : denv * irAB3;
            R olp = R(1.0), lpd = R(0.0);
            int nlp = 0;
            P3 lpv = P3{0, 0, 0}, lpp = pB;
            if (cs == 4) {
                lpd = R(0.50) - R(0.018) * S.zlp[Bq];
                nlp = nb1 - nb0;
                for (int p = nb0; p < nb1; ++p) lpv = lpv + (ldr<R>(V.pos, S.adj[p], org) - pB);
                const R vn = nrm(lpv);
                if (vn > R(1e-10) && nlp > 0) {
                    lpp = pB + (-lpd) * (hb_rcp(vn) * lpv);
                    const R ral = nrm(pA - lpp);
                    const R ex = (HBLPCUT * irv) * ((ral + lpd + R(1e-12)) * irAB - R(1.0));
                    olp = R(2.0) * hb_rcp(R(1.0) + hb_exp(ex));
                } else {
                    nlp = 0;
                    olp = R(1.0);
                }
            }
            const R qhoutl = QH * doutl * onb * olp;
            R eangl = R(1.0), etors = R(1.0);
            P3 ga3[3] = {P3{0, 0, 0}, P3{0, 0, 0}, P3{0, 0, 0}};
            const int Ci = cs == 3 ? S.pc[Bq] : -1;
            const bool c3 = (cs == 3 && Ci != -1);
            if (c3) {
                const R c0 = R(120.0) * R(kPi) / R(180.0);
                const R kijk = (R(1.0) - BEND_HB) / ((cos(R(0.0)) - cos(c0)) * (cos(R(0.0)) - cos(c0)));
                P3 va = ldr<R>(V.pos, Ci, org), vb = pB, vc = pH;
                P3 vab = va - vb, vcb = vc - vb;
                const R rab2c = dot(vab, vab), rcb2 = dot(vcb, vcb);
                P3 vp = cross(vcb, vab);
                const R rp = nrm(vp) + R(1e-14);
                R ca = dot(vab, vcb) / (sqrt(rab2c) * sqrt(rcb2) + R(1e-14));
                ca = fmax(-R(1.0), fmin(R(1.0), ca));
                const R th = acos(ca);
                const R ea = kijk * (ca - cos(c0)) * (ca - cos(c0));
                const R deddt = R(2.0) * kijk * sin(th) * (cos(c0) - ca);
                eangl = R(1.0) - ea;
                P3 deda = (-deddt / (rab2c * rp)) * cross(vab, vp);
                P3 dedc = (deddt / (rcb2 * rp)) * cross(vcb, vp);
                ga3[0] = deda + dedc;
                ga3[1] = -R(1.0) * deda;
                ga3[2] = -R(1.0) * dedc;
                for (int p = S.adj_off[Ci]; p < S.adj_off[Ci + 1]; ++p) {
                    const int D = S.adj[p];
                    if (D == Bq) continue;
                    P3 g[4];
                    const R phi = dihedral(ldr<R>(V.pos, D, org), pB, va, pH, g);
                    const R fct = (R(1.0) - TORS_HB) / R(2.0);
                    const R c1 = 2 * (phi - R(kPi) / R(2.0)) + R(kPi);
                    etors *= (R(1.0) + cos(c1)) * fct + TORS_HB;
                }
            }
            R gs = R(1.0);
            if (cs == 2 || cs == 4) gs = R(0.268);
            else if (cs == 3) gs = R(0.350);
            const R cst = R(aci_a) * R(bas_b) * QA * QB * gs;
            const R E = cs >= 2 ? -rdamp * qhoutl * cst * eangl * etors : -bas * aci * rdamp * qhoutl;
            etot = E;

            P3 drab = -R(1.0) * vAB, drah = -R(1.0) * vAH, drbh = vHB;
            const R rahprbh = rAH + rHB + R(1e-12);
            const R ddamp = (-R(2.0) * HB_ALP * ratio1 * dlg) + (R(2.0) * HB_ALP * ratio3 * dsh);
            const R expo = bacut * (rahprbh * irAB - R(1.0));
            if (expo <= R(15.0)) {
                const R ratio2 = hb_exp(expo);
                const R i1r2 = hb_rcp(R(1.0) + ratio2);
                const R dsig = ratio2 * bacut * irAB * i1r2 * i1r2;   // ratio2 (cut/rv) / rAB / (1 + ratio2)^2
                P3 ga = P3{0, 0, 0}, gb = P3{0, 0, 0}, gh = P3{0, 0, 0};
                if (cs >= 2) {
                    const R rbhdamp = denv * R(1.8) * irHB3;
                    const R rabdamp = denv * (-R(0.8)) * irAB3;
                    const R dterm = -qhoutl * eangl * etors * cst;
                    const R aterm = -rdamp * QH * onb * olp * eangl * etors * cst;
                    const R nbterm = -rdamp * QH * doutl * olp * eangl * etors * cst;
                    R gi = ((rabdamp + rbhdamp) * ddamp - R(3.0) * rabdamp) * irab2;
                    gi *= dterm;
                    P3 dg = gi * drab;
                    ga = dg;
                    gb = -R(1.0) * dg;
                    gi = -R(3.0) * rbhdamp * (irHB * irHB);
                    gi *= dterm;
                    dg = gi * drbh;
                    gb = gb + dg;
                    gh = -R(1.0) * dg;
                    const R tmp1 = -R(2.0) * aterm * dsig;
                    gi = -tmp1 * rahprbh * irab2;
                    dg = gi * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    P3 dgao = (tmp1 * irAH) * drah, dgbo = (tmp1 * irHB) * drbh;
                    ga = ga + dgao;
                    gb = gb + dgbo;
                    gh = gh - dgao - dgbo;
                    for (int p = nb0; p < nb1; ++p) {
                        const int nb = S.adj[p];
                        P3 pn = ldr<R>(V.pos, nb, org);
                        P3 dranb = pA - pn, drbnb = pB - pn;
                        R ia, ib;
                        const R ranb = hb_len(dranb, ia), rbnb = hb_len(drbnb, ib);
                        const R sum = ranb + rbnb + R(1e-12);
                        const R ex = nbc * (sum * irAB - R(1.0));
                        const R r2n = hb_exp(-ex);
                        const R i1 = hb_rcp(R(1.0) + r2n);
                        const R oi = R(2.0) * i1 - R(1.0);
                        const R others = fabs(oi) > R(1e-12) ? onb * hb_rcp(oi) : R(1.0);
                        const R tmp2 = R(2.0) * nbterm * others * r2n * nbc * irAB * i1 * i1;
                        dg = (-tmp2 * sum * irab2) * drab;
                        ga = ga + dg;
                        gb = gb - dg;
                        P3 dgan = (tmp2 * ia) * dranb, dgbn = (tmp2 * ib) * drbnb;
                        ga = ga + dgan;
                        gb = gb + dgbn;
                        agrad(V.grad, nb, -R(1.0) * dgan - dgbn);
                    }
                    if (cs == 4 && nlp > 0) {
                        const R lpterm = -rdamp * QH * doutl * onb * cst;
                        const R ral = nrm(pA - lpp);
                        const R sum = ral + lpd + R(1e-12);
                        const R lpc = HBLPCUT * irv;
                        const R ex = lpc * (sum * irAB - R(1.0));
                        const R r2l = hb_exp(fmin(ex, R(80.0)));   // e^-80: the term vanishes, no overflow
                        const R i1 = hb_rcp(R(1.0) + r2l);
                        const R tmp3 = -R(2.0) * lpterm * r2l * lpc * irAB * i1 * i1;
                        P3 dgl = (-tmp3 * sum * irab2) * drab;
                        ga = ga + dgl;
                        gb = gb - dgl;
                        P3 dral = pA - lpp;
                        P3 dgal = (tmp3 * hb_rcp(ral + R(1e-12))) * dral;
                        ga = ga + dgal;
                        gb = gb - dgal;
                        P3 glp = -R(1.0) * dgal;
                        const R vn = nrm(lpv);
                        if (vn > R(1e-10)) {
                            const R lv[3] = {lpv.x, lpv.y, lpv.z}, gl3[3] = {glp.x, glp.y, glp.z};
                            R out[3] = {0, 0, 0};
                            const R ivn = hb_rcp(vn);
                            const R ivn3 = ivn * ivn * ivn;
                            for (int col = 0; col < 3; ++col)
                                for (int row = 0; row < 3; ++row) {
                                    const R unit = (row == col) ? -R(1.0) : R(0.0);
                                    out[row] += -lpd * (R)nlp * (unit * ivn + lv[row] * lv[col] * ivn3) * gl3[col];
                                }
                            P3 gnb = P3{out[0], out[1], out[2]};
                            gb = gb + gnb;
                            P3 share = (R(1.0) / (R)nlp) * gnb;
                            for (int p = nb0; p < nb1; ++p) agrad(V.grad, S.adj[p], -R(1.0) * share);
                        }
                    }
                    if (c3) {
                        const R bterm = -rdamp * qhoutl * etors * cst;
                        const R tterm = -rdamp * qhoutl * eangl * cst;
                        agrad(V.grad, Bq, bterm * ga3[0]);
                        agrad(V.grad, Ci, bterm * ga3[1]);
                        agrad(V.grad, H, bterm * ga3[2]);
                        P3 va = ldr<R>(V.pos, Ci, org);
                        for (int p = S.adj_off[Ci]; p < S.adj_off[Ci + 1]; ++p) {
                            const int D = S.adj[p];
                            if (D == Bq) continue;
                            P3 g[4];
                            const R phi = dihedral(ldr<R>(V.pos, D, org), pB, va, pH, g);
                            const R fct = (R(1.0) - TORS_HB) / R(2.0);
                            const R c1 = 2 * (phi - R(kPi) / R(2.0)) + R(kPi);
                            const R ek = (R(1.0) + cos(c1)) * fct + TORS_HB;
                            const R dij = -2 * sin(c1) * fct;
                            const R fk = fabs(ek) > R(1e-12) ? etors / ek : R(0.0);
                            const R tk = fk * tterm;
                            agrad(V.grad, D, (tk * dij) * g[0]);
                            agrad(V.grad, Bq, (tk * dij) * g[1]);
                            agrad(V.grad, Ci, (tk * dij) * g[2]);
                            agrad(V.grad, H, (tk * dij) * g[3]);
                        }
                    }
                } else {
                    const R caa = QA * R(bas_a), cbb = QB * R(bas_b);
                    const R rterm = -aci * rdamp * qhoutl, dterm = -aci * bas * qhoutl;
                    const R sterm = -rdamp * bas * qhoutl, aterm = -aci * bas * rdamp * QH;
                    const R tmp = den * den * R(4.0);
                    const R dd24a = (rAH * rAH) * rHB4 * tmp, dd24b = (rHB * rHB) * rAH4 * tmp;
                    R gi = (caa - cbb) * dd24a * rterm;
                    ga = gi * drah;
                    gi = (cbb - caa) * dd24b * rterm;
                    gb = gi * drbh;
                    gh = -R(1.0) * ga - gb;
                    gi = R(aci_b - aci_a) * dd24a;
                    P3 dga = (gi * sterm) * drah;
                    ga = ga + dga;
                    gi = R(aci_a - aci_b) * dd24b;
                    P3 dgb = (gi * sterm) * drbh;
                    gb = gb + dgb;
                    gh = gh - dga - dgb;
                    gi = rdamp * (ddamp - R(3.0)) * irab2;
                    P3 dg = (gi * dterm) * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    gi = aterm * R(2.0) * dsig * rahprbh * irab2;
                    dg = gi * drab;
                    ga = ga + dg;
                    gb = gb - dg;
                    const R to = -R(2.0) * aterm * dsig;
                    P3 dgao = (to * irAH) * drah, dgbo = (to * irHB) * drbh;
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
    eadd(V, (double)etot, t < t1 ? V.mol[rec.x] : -1, T_HB);
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
        const D3 vAX = dmic(V, S.a[t], S.x[t]), vXB = dmic(V, S.x[t], S.b[t]), vAB = dmic(V, S.a[t], S.b[t]);
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
            const double lt = pow6((rXB * rXB) / LC);
            // damping derivatives d dsh/dr and d dlg/dr.  curcuma's analytic gradient
            // (ff_workspace_gfnff.cpp:1465-1476) uses -2 a dsh s^a / (r (1 + s^a)) for the
            // short-range factor, whose true derivative has the opposite sign, and an extra
            // factor t = r^2/LC in the long-range one; the reference mode keeps those for
            // parity, the exact mode (the derivative of the energy) uses the true ones
            const double dds = V.exact ? 2.0 * ALP * dsh * dsh * st / rXB
                                       : -2.0 * ALP * dsh * st / (rXB * (1.0 + st));
            const double ddl = V.exact ? -2.0 * ALP * dlg * dlg * lt / rXB
                                       : -2.0 * ALP * rXB * dlg * lt / (LC * (1.0 + lt));
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
