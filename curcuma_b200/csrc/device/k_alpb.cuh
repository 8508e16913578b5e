// ALPB implicit solvation on the device (Ehlert, Stahn, Spicher, Grimme, J. Chem. Theory
// Comput. 2021, 17, 4250), the per-geometry part of curcuma's ff_methods/alpb_solvation.cpp
// (update, getEnergy, addGradient) for a single molecule:
//   k_alpb_born    Born radii from the descreening sum psi over the pairs within 35 A (one
//                  warp per atom, the partners in ascending order;
//                  alpb_solvation.cpp:502-694) and d brad / d psi;
//   k_alpb_sasa    the smoothed solvent-accessible surface of every atom on the 230-point
//                  Lebedev grid (one block per atom: the neighbours within the surface cut
//                  gathered in ascending order into shared memory, the grid points over the
//                  threads; alpb_solvation.cpp:696-805), the HB weights and the diagonal of the Born
//                  matrix; with GRAD, the surface gradient weighted per atom;
//   k_alpb_shape   the shape descriptor adet of the vdW spheres (one block);
//   the Born matrix enters the EEQ matrix and right-hand side through View::brad/bdiag
//   (k_eeq_M_tiles, eeq_a: A += B, eeq_solver.cpp:3781-3784; the shape constant cancels
//   in the reduced basis);
//   k_alpb_energy  after the solve: the Born pair energy and gradient at fixed charges and
//                  dE/d brad (P16 kernel, alpb_solvation.cpp:1139-1203), self, HB and surface
//                  energies (warp per atom, every partner);
//   k_alpb_chain   dE/d brad through the Born radii: per atom the pairs within 35 A, both
//                  sides of each pair (no atomics on partners);
//   k_alpb_shape_grad  the shape term's energy and gradient (alpb_solvation.cpp:940-1003) and the shift.
// Everything in FP64.  Included inside namespace gfnff by engine.cu, after common.cuh (the
// model constants of setup/alpb.h are included by engine.cu at file scope).
#pragma once

namespace {

constexpr int kAlpbSasaThreads = 128;
constexpr int kAlpbMaxNb = 1536;   // surface neighbours of one atom held in shared memory

struct AlpbArgs {
    int n;
    const double *vdwr, *rho, *svdw, *vdwsa, *trjlo, *trjhi, *wrp, *gamsasa, *hbmag;   // per atom
    const double4* grid;   // 230 points: unit vector, weight
    double keps, alpbet, born_scale, gshift, srcut2;
    int lhb;
    // per evaluation
    double *brad, *dpsi, *sasa, *hbw, *dhbdw, *bdiag, *dEdbr;
    double* shape;         // I (9), centre (3), total r^3, adet
    int* bad;              // set when an atom has more surface neighbours than kAlpbMaxNb
};

__device__ __forceinline__ void alpb_no_overlap(double r, double rho, double& g, double& dg)
{
    const double r1 = 1.0 / r, ap = r + rho, am = r - rho, ab = ap * am;
    const double rhab = rho / ab, lnab = 0.5 * log(am / ap) * r1;
    g += rhab + lnab;
    dg += -2.0 * rhab / ab + (rhab - lnab) * r1 * r1;
}

__device__ __forceinline__ void alpb_overlap(double r, double rho, double rvdw, double& g, double& dg)
{
    if (r + rho <= rvdw) return;
    const double r1 = 1.0 / r, r12 = 0.5 * r1, r24 = r12 * r12;
    const double ap = r + rho, am = r - rho, rh1 = 1.0 / rvdw, rhr1 = 1.0 / ap, aprh1 = ap * rh1;
    const double lnab = log(aprh1);
    g += rh1 - rhr1 + r12 * (0.5 * am * (rhr1 - rh1 * aprh1) - lnab);
    const double d = rhr1 * rhr1 * (1.0 - 0.25 * am * r1 * (1.0 + aprh1 * aprh1)) + rho * r24 * (rhr1 - rh1 * aprh1) +
                     r12 * (r1 * lnab - rhr1);
    dg += d * r1;
}

// contribution of partner b to psi_a and its derivative: d psi_a / d r_a = dg (r_a - r_b).
// The side is overlapping when r < rvdw_a + rho_b; two non-overlapping sides of (near) equal
// descreening radii take the lower-index atom's radius on both sides (the reference's
// symmetric branch)
__device__ __forceinline__ void alpb_psi_side(const AlpbArgs& A, int a, int b, double r, double& g, double& dg)
{
    const double rho_a = A.rho[a], rho_b = A.rho[b];
    const bool ov_ab = r < A.vdwr[a] + rho_b, ov_ba = r < rho_a + A.vdwr[b];
    if (ov_ab) {
        alpb_overlap(r, rho_b, A.vdwr[a], g, dg);
    } else {
        const bool sym = !ov_ba && fabs(rho_a - rho_b) < 1e-8;
        alpb_no_overlap(r, (sym && a < b) ? rho_a : rho_b, g, dg);
    }
}

__global__ void __launch_bounds__(256) k_alpb_born(View V, AlpbArgs A)
{
    const int a = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (a >= A.n) return;
    const double4 pa = V.pos[a];
    const int2 jr = V.jr[a];
    const double lr2 = gfnff::alpb::kLrCut * gfnff::alpb::kLrCut;
    double psi = 0.0;
    for (int b = jr.x + lane; b < jr.y; b += 32) {
        if (b == a) continue;
        const double4 pb = V.pos[b];
        const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= lr2) continue;
        double dg = 0.0;
        alpb_psi_side(A, a, b, sqrt(r2), psi, dg);
    }
    for (int o = 16; o > 0; o >>= 1) psi += __shfl_xor_sync(0xffffffffu, psi, o);
    if (lane == 0) {
        using namespace gfnff::alpb;
        const double s1 = 1.0 / A.svdw[a], v1 = 1.0 / A.vdwr[a], s2 = 0.5 * A.svdw[a];
        const double br = psi * s2;
        double arg2 = br * (kObcGamma * br - kObcBeta);
        const double arg = br * (kObcAlpha + arg2);
        arg2 = 2.0 * arg2 + kObcAlpha + kObcGamma * br * br;
        const double th = tanh(arg), ch = cosh(arg);
        A.brad[a] = A.born_scale / (s1 - v1 * th);
        double dp = ch * (s1 - v1 * th);
        dp = s2 * v1 * arg2 / (dp * dp);
        A.dpsi[a] = A.born_scale * dp;
    }
}

// surface of atom blockIdx.x; GRAD: adds w_a d sasa_a / d r into V.grad with
// w_a = gamsasa_a + dhbdw_a q_a^2, otherwise writes sasa, the HB weights and bdiag
template <bool GRAD>
__global__ void __launch_bounds__(kAlpbSasaThreads) k_alpb_sasa(View V, AlpbArgs A)
{
    using namespace gfnff::alpb;
    __shared__ int nb[kAlpbMaxNb];
    __shared__ double nx[kAlpbMaxNb], ny[kAlpbMaxNb], nz[kAlpbMaxNb];
    __shared__ int cnt;
    const int a = blockIdx.x;
    if (a >= A.n) return;
    const double4 pa = V.pos[a];
    const int2 jr = V.jr[a];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double w = 1.0;
    if (GRAD) {
        w = A.gamsasa[a] + A.dhbdw[a] * V.q[a] * V.q[a];
        if (w == 0.0) return;   // uniform over the block
    }
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    // neighbours within the surface cut, ascending: one warp takes 32 candidates at a time
    // in turn (warps in order through a shared counter per chunk)
    for (int c0 = jr.x; c0 < jr.y; c0 += kAlpbSasaThreads) {
        const int b = c0 + threadIdx.x;
        bool in = false;
        double4 pb = make_double4(0, 0, 0, 0);
        if (b < jr.y && b != a) {
            pb = V.pos[b];
            const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
            in = dx * dx + dy * dy + dz * dz < A.srcut2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        __shared__ int wcnt[kAlpbSasaThreads / 32];
        if (lane == 0) wcnt[warp] = __popc(m);
        __syncthreads();
        int base = cnt;
        for (int k = 0; k < warp; ++k) base += wcnt[k];
        if (in) {
            const int slot = base + __popc(m & ((1u << lane) - 1u));
            if (slot < kAlpbMaxNb) {
                nb[slot] = b;
                nx[slot] = pb.x;
                ny[slot] = pb.y;
                nz[slot] = pb.z;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int k = 0; k < kAlpbSasaThreads / 32; ++k) tot += wcnt[k];
            cnt += tot;
        }
        __syncthreads();
    }
    int nn = cnt;
    if (nn > kAlpbMaxNb) {
        if (threadIdx.x == 0) atomicOr(A.bad, 1);
        nn = kAlpbMaxNb;
    }
    const double R = A.vdwsa[a], wr = A.wrp[a];
    double s = 0.0, ga[3] = {0.0, 0.0, 0.0};
    for (int p = threadIdx.x; p < kNang; p += blockDim.x) {
        const double4 u = A.grid[p];
        const double px = pa.x + R * u.x, py = pa.y + R * u.y, pz = pa.z + R * u.z;
        double sp = 1.0;
        for (int k = 0; k < nn; ++k) {
            const int b = nb[k];
            const double t0 = px - nx[k], t1 = py - ny[k], t2 = pz - nz[k];
            const double tj2 = t0 * t0 + t1 * t1 + t2 * t2;
            if (tj2 >= A.trjhi[b]) continue;
            if (tj2 <= A.trjlo[b]) {
                sp = 0.0;
                break;
            }
            const double uj = sqrt(tj2) - A.vdwsa[b];
            sp *= kAh0 + (kAh1 + kAh3 * uj * uj) * uj;
        }
        if (!(sp > kTolSesp)) continue;
        const double wsa = u.w * wr * sp;
        s += wsa;
        if (GRAD) {
            for (int k = 0; k < nn; ++k) {
                const int b = nb[k];
                const double t0 = px - nx[k], t1 = py - ny[k], t2 = pz - nz[k];
                const double tj2 = t0 * t0 + t1 * t1 + t2 * t2;
                if (tj2 >= A.trjhi[b]) continue;
                const double sq = sqrt(tj2), uj = sq - A.vdwsa[b], ah3uj2 = kAh3 * uj * uj;
                const double sij = kAh0 + (kAh1 + ah3uj2) * uj;
                const double f = w * wsa * (kAh1 + 3.0 * ah3uj2) / (sij * sq);
                ga[0] += f * t0;
                ga[1] += f * t1;
                ga[2] += f * t2;
                atomicAdd(V.grad + 3 * b, -f * t0);
                atomicAdd(V.grad + 3 * b + 1, -f * t1);
                atomicAdd(V.grad + 3 * b + 2, -f * t2);
            }
        }
    }
    __shared__ double red[4][kAlpbSasaThreads / 32];
    double v[4] = {s, ga[0], ga[1], ga[2]};
    for (int c = 0; c < 4; ++c) {
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
        if (lane == 0) red[c][warp] = v[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0, 0, 0, 0};
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < kAlpbSasaThreads / 32; ++k) t[c] += red[c][k];
        if (GRAD) {
            for (int c = 0; c < 3; ++c) atomicAdd(V.grad + 3 * a + c, t[c + 1]);
        } else {
            A.sasa[a] = t[0];
            const double smaxd = 1.0 / (A.vdwsa[a] * A.vdwsa[a]);
            const double hbw = A.lhb ? A.hbmag[a] * t[0] * smaxd : 0.0;
            A.hbw[a] = hbw;
            A.dhbdw[a] = A.lhb ? A.hbmag[a] * smaxd : 0.0;
            A.bdiag[a] = A.keps / A.brad[a] + 2.0 * hbw;
        }
    }
}

// shape tensor of the vdW spheres and adet (one block)
__global__ void __launch_bounds__(256) k_alpb_shape(View V, AlpbArgs A)
{
    __shared__ double red[13][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double t[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) {
        const double r3 = A.vdwr[i] * A.vdwr[i] * A.vdwr[i];
        const double4 p = V.pos[i];
        t[0] += r3;
        t[1] += p.x * r3;
        t[2] += p.y * r3;
        t[3] += p.z * r3;
    }
    for (int c = 0; c < 4; ++c) {
        for (int o = 16; o > 0; o >>= 1) t[c] += __shfl_xor_sync(0xffffffffu, t[c], o);
        if (lane == 0) red[c][warp] = t[c];
    }
    __syncthreads();
    double tot3 = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        tot3 += red[0][k];
        cx += red[1][k];
        cy += red[2][k];
        cz += red[3][k];
    }
    cx /= tot3;
    cy /= tot3;
    cz /= tot3;
    __syncthreads();
    constexpr double tof = 2.0 / 5.0;
    double I[6] = {0, 0, 0, 0, 0, 0};   // xx yy zz xy xz yz
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) {
        const double r2a = A.vdwr[i] * A.vdwr[i], r3 = r2a * A.vdwr[i];
        const double4 p = V.pos[i];
        const double vx = p.x - cx, vy = p.y - cy, vz = p.z - cz, r2 = vx * vx + vy * vy + vz * vz;
        I[0] += r3 * (r2 + tof * r2a - vx * vx);
        I[1] += r3 * (r2 + tof * r2a - vy * vy);
        I[2] += r3 * (r2 + tof * r2a - vz * vz);
        I[3] -= r3 * vx * vy;
        I[4] -= r3 * vx * vz;
        I[5] -= r3 * vy * vz;
    }
    for (int c = 0; c < 6; ++c) {
        for (int o = 16; o > 0; o >>= 1) I[c] += __shfl_xor_sync(0xffffffffu, I[c], o);
        if (lane == 0) red[4 + c][warp] = I[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double J[6] = {0, 0, 0, 0, 0, 0};
        for (int c = 0; c < 6; ++c)
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) J[c] += red[4 + c][k];
        const double xx = J[0], yy = J[1], zz = J[2], xy = J[3], xz = J[4], yz = J[5];
        const double det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz);
        double* S = A.shape;
        S[0] = xx; S[1] = xy; S[2] = xz; S[3] = xy; S[4] = yy; S[5] = yz; S[6] = xz; S[7] = yz; S[8] = zz;
        S[9] = cx; S[10] = cy; S[11] = cz; S[12] = tot3;
        S[13] = sqrt(pow(det, 1.0 / 3.0) / (tof * tot3));
    }
}

// after the solve: Born pairs (P16) and self energy, dE/d brad, HB and surface energies
__global__ void __launch_bounds__(256) k_alpb_energy(View V, AlpbArgs A)
{
    using namespace gfnff::alpb;
    const int a = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    double e = 0.0;
    if (a < A.n) {
        const double4 pa = V.pos[a];
        const int2 jr = V.jr[a];
        const double qa = V.q[a], ba = A.brad[a];
        double de = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
        for (int b = jr.x + lane; b < jr.y; b += 32) {
            if (b == a) continue;
            const double4 pb = V.pos[b];
            const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double qq = qa * V.q[b];
            const double ab = sqrt(ba * A.brad[b]);
            const double a1 = ab / (ab + kZetaP16o16 * r);
            double a16 = a1 * a1;
            a16 *= a16;
            a16 *= a16;
            a16 *= a16;
            const double dfgb = 1.0 / (r + ab * a16), dfgb2 = dfgb * dfgb;
            e += 0.5 * qq * A.keps * dfgb;
            const double ap = (1.0 - kZetaP16 * a1 * a16) * dfgb2 * A.keps / r * qq;
            g0 -= ap * dx;
            g1 -= ap * dy;
            g2 -= ap * dz;
            const double bp = -0.5 * (r * kZetaP16 / ab * a1 + 1.0) / ab * a16 * dfgb2;
            de += A.brad[b] * bp * A.keps * qq;
        }
        for (int o = 16; o > 0; o >>= 1) {
            de += __shfl_xor_sync(0xffffffffu, de, o);
            g0 += __shfl_xor_sync(0xffffffffu, g0, o);
            g1 += __shfl_xor_sync(0xffffffffu, g1, o);
            g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        }
        if (lane == 0) {
            const double qb = qa / ba;
            e += 0.5 * qa * qb * A.keps + A.hbw[a] * qa * qa + A.sasa[a] * A.gamsasa[a];
            A.dEdbr[a] = de - 0.5 * A.keps * qb * qb;
            atomicAdd(V.grad + 3 * a, g0);
            atomicAdd(V.grad + 3 * a + 1, g1);
            atomicAdd(V.grad + 3 * a + 2, g2);
        }
    }
    eadd(V, e, 0, T_SOLV);
}

// dE/d brad through the Born radii: grad_a += sum_b (w_a dg_a(b) + w_b dg_b(a)) (r_a - r_b),
// w = dE/d brad * d brad / d psi, over the pairs within the Born cut
__global__ void __launch_bounds__(256) k_alpb_chain(View V, AlpbArgs A)
{
    const int a = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (a >= A.n) return;
    const double4 pa = V.pos[a];
    const int2 jr = V.jr[a];
    const double lr2 = gfnff::alpb::kLrCut * gfnff::alpb::kLrCut;
    const double wa = A.dEdbr[a] * A.dpsi[a];
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int b = jr.x + lane; b < jr.y; b += 32) {
        if (b == a) continue;
        const double4 pb = V.pos[b];
        const double dx = pa.x - pb.x, dy = pa.y - pb.y, dz = pa.z - pb.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= lr2) continue;
        const double r = sqrt(r2);
        double ga = 0.0, da = 0.0, gb = 0.0, db = 0.0;
        alpb_psi_side(A, a, b, r, ga, da);
        alpb_psi_side(A, b, a, r, gb, db);
        const double f = wa * da + A.dEdbr[b] * A.dpsi[b] * db;
        g0 += f * dx;
        g1 += f * dy;
        g2 += f * dz;
    }
    for (int o = 16; o > 0; o >>= 1) {
        g0 += __shfl_xor_sync(0xffffffffu, g0, o);
        g1 += __shfl_xor_sync(0xffffffffu, g1, o);
        g2 += __shfl_xor_sync(0xffffffffu, g2, o);
    }
    if (lane == 0) {
        atomicAdd(V.grad + 3 * a, g0);
        atomicAdd(V.grad + 3 * a + 1, g1);
        atomicAdd(V.grad + 3 * a + 2, g2);
    }
}

// the shape term 1/2 keps alpbet / adet (sum q)^2, its gradient, and the free-energy shift
// (one block)
__global__ void __launch_bounds__(256) k_alpb_shape_grad(View V, AlpbArgs A)
{
    __shared__ double red[8];
    __shared__ double qt_s;
    double qt = 0.0;
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) qt += V.q[i];
    for (int o = 16; o > 0; o >>= 1) qt += __shfl_xor_sync(0xffffffffu, qt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = qt;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
        qt_s = t;
    }
    __syncthreads();
    qt = qt_s;
    const double* S = A.shape;
    const double adet = S[13], tot3 = S[12];
    if (A.alpbet > 0.0) {
        const double (*I)[3] = reinterpret_cast<const double(*)[3]>(S);
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
        const double scale = (250.0 / (48.0 * tot3 * tot3 * tot3 * pow(adet, 5.0))) * (-0.5 * ke * qt * qt / (adet * adet));
        for (int i = threadIdx.x; i < A.n; i += blockDim.x) {
            const double r3 = A.vdwr[i] * A.vdwr[i] * A.vdwr[i];
            const double4 p = V.pos[i];
            const double v[3] = {p.x - S[9], p.y - S[10], p.z - S[11]};
            for (int c = 0; c < 3; ++c)
                atomicAdd(V.grad + 3 * i + c, r3 * scale * (D[c][0] * v[0] + D[c][1] * v[1] + D[c][2] * v[2]));
        }
    }
    if (threadIdx.x == 0) {
        const double e = (A.alpbet > 0.0 ? 0.5 * qt * qt * A.alpbet / adet * A.keps : 0.0) + A.gshift;
        atomicAdd(V.E + T_SOLV, e);
    }
}

}  // namespace
