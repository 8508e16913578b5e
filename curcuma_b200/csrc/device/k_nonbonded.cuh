// Non-bonded GFN-FF kernels: geometry in, coordination numbers, D4 weights, repulsion,
// all-pairs Coulomb + D4 dispersion, self energy, CN chain rule and the outputs.
// Included inside namespace gfnff by engine.cu (one translation unit).
//
// The all-pairs kernels share one layout: a block owns kTile consecutive atoms i (one per
// thread) and walks the partners j of its molecule range in tiles of kTile staged through
// shared memory, so every partner record is read from L2 once per block and broadcast to
// all threads.  grid.y splits the partner range of an i-block (nsplit slices) so that small
// systems still fill the 148 SMs; per-atom partial sums then meet in FP64 atomics.  Atoms
// are Morton-sorted at upload, so the lanes of a warp are spatial neighbours and the
// short-range branches (erf, exp) stay coherent.
#pragma once

namespace {

constexpr int kTile = 128;

// partner range [jb, je) of this block's slice
__device__ __forceinline__ void tile_range(const View& V, int i0, int nsplit, int& jb, int& je)
{
    const int last = min(V.n, i0 + kTile) - 1;
    const int lo = V.jr[i0].x, hi = V.jr[last].y;
    const int ntiles = (hi - lo + kTile - 1) / kTile;
    const int per = (ntiles + nsplit - 1) / nsplit;
    jb = lo + (int)blockIdx.y * per * kTile;
    je = min(hi, jb + per * kTile);
}

// ------------------------------------------------------------------------------------
// geometry in (caller order -> internal order) and the HB refresh metric
// (gfnff_method.cpp:2228-2259)
// ------------------------------------------------------------------------------------
// (nl_ref, nl_bad): reference geometry of the CN neighbour list; an atom more than
// sqrt(nl_lim2) away from it marks the list stale (kept until the host rebuilds it).
// msd[1] receives the topology refresh metric, the largest |coordinate change| since the
// geometry topo_ref of the last topology (gfnff_method.cpp:1021-1031), as the bits of a
// non-negative double (which order like the integers)
__global__ void k_positions(int n, const int* __restrict__ perm, const double* __restrict__ xyz, double scale,
                            double4* pos, const double4* __restrict__ ref, double* msd,
                            const double4* __restrict__ nl_ref, double nl_lim2, int* nl_bad,
                            const double4* __restrict__ topo_ref)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0.0, dmax = 0.0;
    if (i < n) {
        const int o = perm[i];
        const double x = xyz[3 * o] * scale, y = xyz[3 * o + 1] * scale, z = xyz[3 * o + 2] * scale;
        pos[i] = make_double4(x, y, z, 0.0);
        const double4 r = ref[i];
        s = (x - r.x) * (x - r.x) + (y - r.y) * (y - r.y) + (z - r.z) * (z - r.z);
        const double4 t = topo_ref[i];
        dmax = fmax(fabs(x - t.x), fmax(fabs(y - t.y), fabs(z - t.z)));
        if (nl_ref) {
            const double4 q = nl_ref[i];
            const double d2 = (x - q.x) * (x - q.x) + (y - q.y) * (y - q.y) + (z - q.z) * (z - q.z);
            if (d2 > nl_lim2) atomicOr(nl_bad, 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0 && dmax > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(msd + 1), (unsigned long long)__double_as_longlong(dmax));
    block_add(s, msd);
}

// ------------------------------------------------------------------------------------
// atom boxes: min/max corner of every run of 32 consecutive atoms.  Atoms are in Morton
// order within a molecule, so a run is fairly compact in space and the short-range pair
// kernels (CN, CN chain rule) skip partner tiles, and a warp partner runs of 32 atoms, whose
// box is farther than the cutoff from its own (single molecules of 8192 atoms or more;
// below that the tests cost more than they save, measured).  The box distance is a lower bound of every pair distance
// in floating point too (min/max are exact, rounding is monotonic), so the skipped pairs
// are exactly pairs the cutoff test rejects.
// ------------------------------------------------------------------------------------
constexpr int kBoxAtoms = 32;
__global__ void __launch_bounds__(kTile) k_boxes(int n, const double4* __restrict__ pos, double4* lo, double4* hi)
{
    const int i = blockIdx.x * kTile + threadIdx.x;
    const int b = i / kBoxAtoms;
    if (b * kBoxAtoms >= n) return;   // whole warp beyond the atoms
    const double4 p = pos[i < n ? i : b * kBoxAtoms];
    double v[6] = {p.x, p.y, p.z, -p.x, -p.y, -p.z};   // minima of x and of -x
#pragma unroll
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) v[k] = fmin(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    if ((threadIdx.x & 31) == 0) {
        lo[b] = make_double4(v[0], v[1], v[2], 0.0);
        hi[b] = make_double4(-v[3], -v[4], -v[5], 0.0);
    }
}

// box of the atoms [a, b) (b > a), as the union of the 32-atom boxes covering it
__device__ __forceinline__ void range_box(const View& V, int a, int b, double4& l, double4& h)
{
    l = V.boxlo[a / kBoxAtoms];
    h = V.boxhi[a / kBoxAtoms];
    for (int k = a / kBoxAtoms + 1; k <= (b - 1) / kBoxAtoms; ++k) {
        const double4 l2 = V.boxlo[k], h2 = V.boxhi[k];
        l = make_double4(fmin(l.x, l2.x), fmin(l.y, l2.y), fmin(l.z, l2.z), 0.0);
        h = make_double4(fmax(h.x, h2.x), fmax(h.y, h2.y), fmax(h.z, h2.z), 0.0);
    }
}

__device__ __forceinline__ bool boxes_far(double4 il, double4 ih, double4 jl, double4 jh, double cut2)
{
    const double dx = fmax(0.0, fmax(jl.x - ih.x, il.x - jh.x));
    const double dy = fmax(0.0, fmax(jl.y - ih.y, il.y - jh.y));
    const double dz = fmax(0.0, fmax(jl.z - ih.z, il.z - jh.z));
    return dx * dx + dy * dy + dz * dz >= cut2;
}

// true when every atom of [j0, j0 + cnt) is at least sqrt(cut2) from every atom of
// [i0, i0 + ni)
__device__ __forceinline__ bool ranges_far(const View& V, int i0, int ni, int j0, int cnt, double cut2)
{
    double4 il, ih, jl, jh;
    range_box(V, i0, i0 + ni, il, ih);
    range_box(V, j0, j0 + cnt, jl, jh);
    return boxes_far(il, ih, jl, jh, cut2);
}

// One counting term 0.5 (1 + erf(kn (r - rc) / rc)), kn = -7.5, of the GFN-FF CN
// (cn_calculator.cpp:367-428); d2 = r^2, rc = the pair's covalent radius sum (bohr).  FP64:
// as written.  FP32 (mixed form): the argument in FP64, then the identity 0.5 (1 + erf(z)) =
// 0.5 erfc(-z) with only the small tail erfc(|z|) in FP32, subtracted from an exact 1 for
// z >= 0 and accumulated in FP64: 1 + erf(z) in FP32 cancels to a few significant bits for
// the distant pairs, whose rounding then adds up over ~100 partners per atom.
template <class R>
__device__ __forceinline__ double cn_count(double d2, double rc)
{
    const double r = sqrt(d2);
    const double z = -7.5 * ((r - rc) / rc);
    if constexpr (std::is_same<R, double>::value) {
        return 0.5 * (1.0 + erf(z));
    } else {
        const double t = (double)erfcf((float)fabs(z));
        return z >= 0.0 ? 1.0 - 0.5 * t : 0.5 * t;
    }
}

// ------------------------------------------------------------------------------------
// coordination numbers: erf counting over partners closer than 6 bohr
// (cn_calculator.cpp:367-428); the log-squash is applied in k_d4_weights
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(kTile) k_cn(View V, int nsplit, const int* nl_bad)
{
    if (nl_bad && *nl_bad == 0) return;   // the neighbour-list kernel does the work
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sr[kTile];
    const int i0 = blockIdx.x * kTile, i = i0 + threadIdx.x;
    int jb, je;
    tile_range(V, i0, nsplit, jb, je);
    const bool act = i < V.n;
    const double4 pi = act ? V.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const double ri = act ? V.rcov_cn[i] : 0.0;
    const int2 rg = act ? V.jr[i] : make_int2(0, 0);
    double s = 0.0;
    const int ni = min(kTile, V.n - i0);
    const int w0 = i0 + (threadIdx.x & ~31), nw = max(0, min(32, V.n - w0));   // this warp's atoms
    for (int t0 = jb; t0 < je; t0 += kTile) {
        const int cnt = min(kTile, je - t0);
        if (V.boxlo && ranges_far(V, i0, ni, t0, cnt, 36.0)) continue;   // uniform in the block
        __syncthreads();
        const int jl = t0 + threadIdx.x;
        if (jl < je) {
            const double4 p = V.pos[jl];
            sx[threadIdx.x] = p.x; sy[threadIdx.x] = p.y; sz[threadIdx.x] = p.z;
            sr[threadIdx.x] = V.rcov_cn[jl];
        }
        __syncthreads();
        if (!act) continue;
        for (int js = 0; js < cnt; js += 32) {
            const int jn = min(32, cnt - js);
            if (V.boxlo && ranges_far(V, w0, nw, t0 + js, jn, 36.0)) continue;   // uniform in the warp
            for (int jj = js; jj < js + jn; ++jj) {
                double dx = pi.x - sx[jj], dy = pi.y - sy[jj], dz = pi.z - sz[jj];
                if (V.cell.on) mic(V.cell, dx, dy, dz);
                const double d2 = dx * dx + dy * dy + dz * dz;
                const int j = t0 + jj;
                if (!(d2 < 36.0) || j == i || j < rg.x || j >= rg.y) continue;
                s += cn_count<R>(d2, ri + sr[jj]);
            }
        }
    }
    if (act && s != 0.0) atomicAdd(V.cnraw + i, s);
}

// ------------------------------------------------------------------------------------
// CN log-squash (cnmax = 4.4) and its derivative, D4 Gaussian weights (wf = 4) and the
// half contraction with the reference C6 (d4param_generator.cpp:1079-1290, :1692-1740)
// ------------------------------------------------------------------------------------
__global__ void k_d4_weights(View V)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.n) return;
    {
        const double cnmax = 4.4, s = V.cnraw[i];
        V.cn[i] = log(1.0 + exp(cnmax)) - log(1.0 + exp(cnmax - s));
        V.dlog[i] = exp(cnmax) / (exp(cnmax) + exp(s));
    }
    const int nr = V.nref[i];
    const double cn = V.cn[i];
    double ex[7], dex[7], w[7], dw[7];
    double norm = 0.0, dnorm = 0.0;
    for (int r = 0; r < 7; ++r) {
        ex[r] = dex[r] = w[r] = dw[r] = 0.0;
        if (r < nr) {
            const double d = cn - V.refcn[i * 7 + r];
            ex[r] = exp(-4.0 * d * d);
            dex[r] = (-2.0 * 4.0) * d * ex[r];
            norm += ex[r];
            dnorm += dex[r];
        }
    }
    if (nr > 0) {
        if (norm > 1e-10) {
            const double inv = 1.0 / norm, inv2 = 1.0 / (norm * norm);
            for (int r = 0; r < nr; ++r) {
                w[r] = ex[r] * inv;
                dw[r] = (dex[r] * norm - ex[r] * dnorm) * inv2;
            }
        } else {
            w[0] = 1.0;
        }
    }
    for (int r = 0; r < 7; ++r) { V.w[i * 7 + r] = w[r]; V.dw[i * 7 + r] = dw[r]; }
    const int si = V.slot[i];
    for (int s = 0; s < V.K; ++s) {
        const double* C = V.c6ref + ((size_t)(si * V.K + s)) * 49;
        for (int b = 0; b < 7; ++b) {
            double g = 0.0, dg = 0.0;
            for (int a = 0; a < nr; ++a) {
                g += w[a] * C[a * 7 + b];
                dg += dw[a] * C[a * 7 + b];
            }
            V.hg[((size_t)i * V.K + s) * 7 + b] = g;
            V.hdg[((size_t)i * V.K + s) * 7 + b] = dg;
        }
    }
}

// ------------------------------------------------------------------------------------
// repulsion over per-atom CSR lists holding both pair directions
// (ff_workspace_gfnff.cpp:774-848); kind 0 = bonded, 1 = non-bonded.  One warp per atom.
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(kBlock) k_repulsion(View V, const int* off, const int* nbj, const double* alpha,
                                                     const double* repab, const unsigned char* kind)
{
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    double eb = 0.0, enb = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    if (i < V.n) {
        const double4 pi = V.pos[i];
        for (int p = off[i] + lane; p < off[i + 1]; p += 32) {
            const double4 pj = V.pos[nbj[p]];
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            if (V.cell.on) mic(V.cell, dx, dy, dz);
            const double d2 = dx * dx + dy * dy + dz * dz;
            const R r = sqrt((R)d2);
            if (r > R(20) || r < R(1e-8)) continue;
            const R sr = sqrt(r), al = (R)alpha[p];
            const R e = (R)repab[p] * exp(-al * (r * sr)) / r;
            if (kind[p]) enb += 0.5 * (double)e; else eb += 0.5 * (double)e;
            const R dEdr = -e / r - R(1.5) * al * sr * e;
            const double f = (double)(dEdr / r);
            gx += f * dx; gy += f * dy; gz += f * dz;
        }
        for (int o = 16; o > 0; o >>= 1) {
            gx += __shfl_down_sync(0xffffffffu, gx, o);
            gy += __shfl_down_sync(0xffffffffu, gy, o);
            gz += __shfl_down_sync(0xffffffffu, gz, o);
        }
        // atomics: the kernel runs beside others that add to the same gradient entries
        if (lane == 0) {
            if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
            if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
            if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
        }
    }
    const int m = i < V.n ? V.mol[i] : -1;
    eadd(V, eb, m, T_BREP);
    eadd(V, enb, m, T_NBREP);
}

// ------------------------------------------------------------------------------------
// all-pairs Coulomb (r <= 100 bohr; ff_workspace_gfnff.cpp:850-900) and D4 dispersion
// over the setup pair list (setup distance <= 60 bohr, evaluated for r <= 50;
// :715-772, d4param_generator.cpp:1959-2092) with the frozen setup C6 and the per-step
// dC6/dCN chain term.  Both directions of a pair are evaluated (row i collects its own
// gradient and dE/dCN_i); energies are halved.
//
// Coulomb fast path: erf(x) rounds to exactly 1 in double for x >= 6 (erfc(6) = 2.2e-17
// is below half an ulp of 1), i.e. for r^2 >= 36 (a_i + a_j); the pair is then q q / r and
// its exp(-x^2) gradient term is below 2e-15 relative, so both are dropped there.
// R is the arithmetic type of the D4 part beyond 15 bohr: double in the FP64 form,
// float in the mixed form (nearer D4 pairs are FP64 in both).  Coulomb (both branches), the distances and every sum stay FP64 in both forms:
// single Coulomb pairs reach 0.1 Eh and there are ~N^2/2 of them, so FP32 rounding in
// them would add up to more than 1e-6 Eh.
// ------------------------------------------------------------------------------------
// one D4 pair in arithmetic type R: energy e, dE/dr / r in dedr, dE/dCN_i in dc
template <class R>
__device__ __forceinline__ void d4_pair(double d2, const double* g0, const double* dg, const double (*sw0)[kTile],
                                        const double (*sw)[kTile], int jj, int nr, double szi, double szj,
                                        double zz_d, double& e, double& dedr, double& dc)
{
    R c6 = R(0), dc6 = R(0);
    for (int b = 0; b < nr; ++b) {
        c6 += (R)__ldg(g0 + b) * (R)sw0[b][jj];
        dc6 += (R)dg[b] * (R)sw[b][jj];
    }
    const R q2 = (R)d2;
    const R r4r2 = R(3) * (R)szi * (R)szj;
    const R t = R(0.58) * sqrt(r4r2) + R(4.80);
    const R r0sq = t * t;
    const R zz = (R)zz_d;
    const R r6 = q2 * q2 * q2, r06 = r0sq * r0sq * r0sq;
    const R t6 = R(1) / (r6 + r06);
    const R t8 = R(1) / (r6 * q2 + r06 * r0sq);
    const R sum = t6 + R(2) * r4r2 * t8;
    e = -(double)(c6 * sum * zz);
    const R d6 = R(-6) * q2 * q2 * t6 * t6, d8 = R(-8) * r6 * t8 * t8;
    dedr = -(double)(c6 * zz * (d6 + R(2) * r4r2 * d8));
    dc = -(double)(dc6 * sum * zz);
}

template <class R>
__global__ void __launch_bounds__(kTile) k_pairs(View V, int nsplit)
{
    __shared__ double sx[kTile], sy[kTile], sz[kTile], s0x[kTile], s0y[kTile], s0z[kTile];
    __shared__ double sq[kTile], sa[kTile], sze[kTile], ssz[kTile];
    __shared__ double sw0[7][kTile], sw[7][kTile];
    __shared__ int ssl[kTile], snr[kTile];
    const int i0 = blockIdx.x * kTile, i = i0 + threadIdx.x;
    int jb, je;
    tile_range(V, i0, nsplit, jb, je);
    const bool act = i < V.n;
    const int ic = act ? i : i0;
    const double4 pi = V.pos[ic], p0i = V.pos0[ic];
    const double ai = V.alpeeq[ic], qi = V.q[ic], zi = V.zeta[ic], szi = V.szr[ic];
    const int2 rg = act ? V.jr[i] : make_int2(0, 0);
    const double* g0i = V.g0 + (size_t)ic * V.K * 7;
    const double* dgi = V.hdg + (size_t)ic * V.K * 7;
    const double tsp = 2.0 / 1.772453850905516;
    double ec = 0.0, ed = 0.0, gx = 0.0, gy = 0.0, gz = 0.0, dcn = 0.0, cfar = 0.0;
    for (int t0 = jb; t0 < je; t0 += kTile) {
        __syncthreads();
        const int jl = t0 + threadIdx.x;
        if (jl < je) {
            const int u = threadIdx.x;
            const double4 p = V.pos[jl], p0 = V.pos0[jl];
            sx[u] = p.x; sy[u] = p.y; sz[u] = p.z;
            s0x[u] = p0.x; s0y[u] = p0.y; s0z[u] = p0.z;
            sq[u] = V.q[jl]; sa[u] = V.alpeeq[jl]; sze[u] = V.zeta[jl]; ssz[u] = V.szr[jl];
            ssl[u] = V.slot[jl]; snr[u] = V.nref[jl];
#pragma unroll
            for (int b = 0; b < 7; ++b) {
                sw0[b][u] = V.w0[(size_t)jl * 7 + b];
                sw[b][u] = V.w[(size_t)jl * 7 + b];
            }
        }
        __syncthreads();
        const int cnt = min(kTile, je - t0);
        if (!act) continue;
        for (int jj = 0; jj < cnt; ++jj) {
            const int j = t0 + jj;
            if (j == i || j < rg.x || j >= rg.y) continue;
            double dx = pi.x - sx[jj], dy = pi.y - sy[jj], dz = pi.z - sz[jj];
            if (V.cell.on) mic(V.cell, dx, dy, dz);
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < 1e-20) continue;
            double f = 0.0;   // dE/dr / r
            if (d2 <= 10000.0) {
                const double s = ai + sa[jj];
                const double qq = qi * sq[jj];
                if (d2 >= 36.0 * s) {
                    const double ir = rsqrt(d2);
                    const double e = qq * ir;
                    ec += e;
                    f -= e * ir * ir;
                } else {
                    const double r = sqrt(d2);
                    const double g = 1.0 / sqrt(s);
                    const double gr = g * r;
                    const double ef = erf(gr);
                    ec += qq * ef / r;
                    f += qq * ((g * exp(-gr * gr) * tsp) / r - ef / d2) / r;
                }
            } else if (V.cfar) {
                cfar += sq[jj] * rsqrt(d2);   // cut pair: its EEQ element is 1/r
            }
            if (d2 <= 2500.0 &&
                d2_exact(p0i, make_double4(s0x[jj], s0y[jj], s0z[jj], 0.0)) <= 3600.0) {
                const int sj = ssl[jj], nr = snr[jj];
                const double* g0 = g0i + sj * 7;
                const double* dg = dgi + sj * 7;
                double e, dedr, dc;
                // mixed form: pairs closer than 15 bohr (the strong ones) stay FP64
                if (sizeof(R) == sizeof(double) || d2 < 225.0)
                    d4_pair<double>(d2, g0, dg, sw0, sw, jj, nr, szi, ssz[jj], zi * sze[jj], e, dedr, dc);
                else
                    d4_pair<R>(d2, g0, dg, sw0, sw, jj, nr, szi, ssz[jj], zi * sze[jj], e, dedr, dc);
                ed += e;
                f += dedr;
                if (!V.exact) dcn += dc;
            }
            gx += f * dx; gy += f * dy; gz += f * dz;
        }
    }
    if (act) {
        if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
        if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
        if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
        if (dcn != 0.0) atomicAdd(V.dEdcn + i, dcn);
        if (cfar != 0.0) atomicAdd(V.cfar + i, cfar);
    }
    const int m = act ? V.mol[i] : -1;
    eadd(V, 0.5 * ec, m, T_COUL);
    eadd(V, 0.5 * ed, m, T_DISP);
}

// ------------------------------------------------------------------------------------
// The same Coulomb + D4 pair terms with every pair evaluated once (Newton's third law).
// Blocks take T x T tiles (i tile <= j tile, listed at set-up; only j > i within a
// diagonal tile; T = 64 for single molecules, 32 for batches of small molecules, whose
// tiles would otherwise straddle molecules).  Row i keeps its sums in registers as in k_pairs; the j side of every
// pair (gradient, dE/dCN_j from j's half contraction against i's current weights, and the
// far-pair potential of the exact-gradient mode) is summed over the warp's 32 rows with
// shuffles and kept per warp in shared memory, then added once per tile.
// ------------------------------------------------------------------------------------
constexpr int kST = 64;

// one D4 pair in arithmetic type R with both CN derivatives: energy e, dE/dr / r in dedr,
// dE/dCN_i in dci, dE/dCN_j in dcj (wi: current weights of i in registers)
template <class R, int T>
__device__ __forceinline__ void d4_pair_sym(double d2, const double* g0, const double* dgi, const double* dgj,
                                            const double (*sw0)[T], const double (*sw)[T], int jj, int nrj,
                                            int nri, const double (&wi)[7], double r4r2_d, double sr4r2_d,
                                            double zz_d, bool want_dc, double& e, double& dedr, double& dci,
                                            double& dcj)
{
    R c6 = R(0), dc6i = R(0), dc6j = R(0);
    for (int b = 0; b < nrj; ++b) c6 += (R)__ldg(g0 + b) * (R)sw0[b][jj];
    if (want_dc) {
        for (int b = 0; b < nrj; ++b) dc6i += (R)__ldg(dgi + b) * (R)sw[b][jj];
#pragma unroll
        for (int a = 0; a < 7; ++a)
            if (a < nri) dc6j += (R)__ldg(dgj + a) * (R)wi[a];
    }
    const R q2 = (R)d2;
    const R r4r2 = (R)r4r2_d;
    const R t = R(0.58) * (R)sr4r2_d + R(4.80);   // sr4r2_d = sqrt(r4r2) from per-atom roots
    const R r0sq = t * t;
    const R zz = (R)zz_d;
    const R r6 = q2 * q2 * q2, r06 = r0sq * r0sq * r0sq;
    // 1/a and 1/b from one division: a*b stays below 1e24 for r <= 50 bohr
    const R a6 = r6 + r06, a8 = r6 * q2 + r06 * r0sq;
    const R inv = R(1) / (a6 * a8);
    const R t6 = a8 * inv, t8 = a6 * inv;
    const R sum = t6 + R(2) * r4r2 * t8;
    e = -(double)(c6 * sum * zz);
    const R d6 = R(-6) * q2 * q2 * t6 * t6, d8 = R(-8) * r6 * t8 * t8;
    dedr = -(double)(c6 * zz * (d6 + R(2) * r4r2 * d8));
    dci = -(double)(dc6i * sum * zz);
    dcj = -(double)(dc6j * sum * zz);
}

// PART selects the terms: kPairCoul (needs this step's charges), kPairD4 (needs only the
// CN weights, so it can run beside the EEQ solve), or both in one pass
constexpr int kPairCoul = 1, kPairD4 = 2, kPairBoth = 3;
template <class R, int MINB, int T, int PART>
__global__ void __launch_bounds__(T, MINB) k_pairs_sym(View V, const int2* __restrict__ tiles)
{
    constexpr bool COUL = (PART & kPairCoul) != 0, D4 = (PART & kPairD4) != 0;
    constexpr int NA = 5;   // j-side sums: fx, fy, fz, dE/dCN_j (D4), far potential (Coulomb)
    __shared__ double sx[T], sy[T], sz[T];
    __shared__ double sq[COUL ? T : 1], sa[COUL ? T : 1];
    __shared__ double s0x[D4 ? T : 1], s0y[D4 ? T : 1], s0z[D4 ? T : 1];
    __shared__ double sze[D4 ? T : 1], ssz[D4 ? T : 1], srz[D4 ? T : 1];
    __shared__ double sw0[D4 ? 7 : 1][T], sw[D4 ? 7 : 1][T];
    __shared__ int ssl[D4 ? T : 1], snr[D4 ? T : 1];
    __shared__ double jacc[T / 32][NA][T];
    const int2 tp = tiles[blockIdx.x];
    const int i0 = tp.x, j0 = tp.y, i = i0 + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool act = i < V.n;
    const int ic = act ? i : i0;
    const double4 pi = V.pos[ic];
    const int2 rg = act ? V.jr[i] : make_int2(0, 0);
    double ai = 0.0, qi = 0.0;
    if constexpr (COUL) { ai = V.alpeeq[ic]; qi = V.q[ic]; }
    double4 p0i = make_double4(0.0, 0.0, 0.0, 0.0);
    double zi = 0.0, szi = 0.0, s3i = 0.0;
    int si = 0, nri = 0;
    double wi[7];
    const double* g0i = nullptr;
    const double* dgi = nullptr;
    if constexpr (D4) {
        p0i = V.pos0[ic];
        zi = V.zeta[ic]; szi = V.szr[ic];
        s3i = sqrt(3.0 * szi);   // sqrt(r4r2) of a pair = s3i * sqrt(szr_j)
        si = V.slot[ic]; nri = V.nref[ic];
#pragma unroll
        for (int a = 0; a < 7; ++a) wi[a] = V.w[(size_t)ic * 7 + a];
        g0i = V.g0 + (size_t)ic * V.K * 7;
        dgi = V.hdg + (size_t)ic * V.K * 7;
    }
    const bool want_dc = !V.exact, want_far = COUL && V.cfar != nullptr;
    {
        const int jl = j0 + threadIdx.x;
        if (jl < V.n) {
            const int u = threadIdx.x;
            const double4 p = V.pos[jl];
            sx[u] = p.x; sy[u] = p.y; sz[u] = p.z;
            if constexpr (COUL) { sq[u] = V.q[jl]; sa[u] = V.alpeeq[jl]; }
            if constexpr (D4) {
                const double4 p0 = V.pos0[jl];
                s0x[u] = p0.x; s0y[u] = p0.y; s0z[u] = p0.z;
                sze[u] = V.zeta[jl]; ssz[u] = V.szr[jl]; srz[u] = sqrt(ssz[u]);
                ssl[u] = V.slot[jl]; snr[u] = V.nref[jl];
#pragma unroll
                for (int b = 0; b < 7; ++b) {
                    sw0[b][u] = V.w0[(size_t)jl * 7 + b];
                    sw[b][u] = V.w[(size_t)jl * 7 + b];
                }
            }
        }
    }
    // j-side sums, per warp in shared memory, in two passes over the tile's partners.
    // Coulomb pass: at step k lane t of the block takes partner (t + k) mod T, so the lanes of
    // a warp always hold distinct partners and add their j-side terms without shuffles or
    // conflicts (1000 waters, Coulomb launch: 104 -> 53 us against warp-wide reductions).
    // D4 pass: the lanes take the same partner and the j-side sums are reduced over the warp
    // (rotated partners made the per-partner reference loops diverge: D4 61 -> 122 us); a
    // warp runs it only when one of its pairs is within the 50 bohr D4 range, which the
    // Coulomb pass records.
#pragma unroll
    for (int k = 0; k < NA; ++k)
        for (int u = lane; u < T; u += 32) jacc[warp][k][u] = 0.0;
    __syncthreads();
    const double tsp = 2.0 / 1.772453850905516;
    double ec = 0.0, ed = 0.0, gx = 0.0, gy = 0.0, gz = 0.0, dcn = 0.0, cfar = 0.0;
    const int cnt = min(T, V.n - j0);
    bool near = !COUL;   // a pair within the D4 range (D4-only launches: assume one)
    if constexpr (COUL) {
        for (int k = 0; k < T; ++k) {
            const int jj = (threadIdx.x + k) & (T - 1);
            if (jj >= cnt) continue;
            const int j = j0 + jj;
            if (!(act && j > i && j >= rg.x && j < rg.y)) continue;
            double dx = pi.x - sx[jj], dy = pi.y - sy[jj], dz = pi.z - sz[jj];
            if (V.cell.on) mic(V.cell, dx, dy, dz);
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (!(d2 >= 1e-20)) continue;
            double f = 0.0, cfj = 0.0;   // dE/dr / r
            if (d2 <= 10000.0) {
                const double s = ai + sa[jj];
                const double qq = qi * sq[jj];
                if (d2 >= 36.0 * s) {
                    const double ir = rsqrt(d2);
                    const double e = qq * ir;
                    ec += e;
                    f -= e * ir * ir;
                } else {
                    const double r = sqrt(d2);
                    const double g = 1.0 / sqrt(s);
                    const double gr = g * r;
                    const double ef = erf(gr);
                    ec += qq * ef / r;
                    f += qq * ((g * exp(-gr * gr) * tsp) / r - ef / d2) / r;
                }
            } else if (want_far) {
                const double ir = rsqrt(d2);   // cut pair: its EEQ element is 1/r
                cfar += sq[jj] * ir;
                cfj = qi * ir;
            }
            if (D4) near |= d2 <= 2500.0;
            gx += f * dx; gy += f * dy; gz += f * dz;
            jacc[warp][0][jj] -= f * dx;
            jacc[warp][1][jj] -= f * dy;
            jacc[warp][2][jj] -= f * dz;
            if (want_far) jacc[warp][4][jj] += cfj;
        }
    }
    if constexpr (D4) {
        if (__any_sync(0xffffffffu, near)) {
            for (int k = 0; k < cnt; ++k) {
                const int jj = k;
                const int j = j0 + jj;
                double fx = 0.0, fy = 0.0, fz = 0.0, dcj = 0.0;
                bool hit = false;   // this lane has a j-side contribution
                if (act && j > i && j >= rg.x && j < rg.y) {
                    double dx = pi.x - sx[jj], dy = pi.y - sy[jj], dz = pi.z - sz[jj];
                    if (V.cell.on) mic(V.cell, dx, dy, dz);
                    const double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 >= 1e-20 && d2 <= 2500.0 &&
                        d2_exact(p0i, make_double4(s0x[jj], s0y[jj], s0z[jj], 0.0)) <= 3600.0) {
                        hit = true;
                        const int sj = ssl[jj], nrj = snr[jj];
                        const double* dgj = V.hdg + ((size_t)j * V.K + si) * 7;
                        const double r4r2 = 3.0 * szi * ssz[jj], sr4r2 = s3i * srz[jj], zz = zi * sze[jj];
                        double e, dedr, dci;
                        // mixed form: pairs closer than 15 bohr (the strong ones) stay FP64
                        if (sizeof(R) == sizeof(double) || d2 < 225.0)
                            d4_pair_sym<double, T>(d2, g0i + sj * 7, dgi + sj * 7, dgj, sw0, sw, jj, nrj, nri, wi,
                                                   r4r2, sr4r2, zz, want_dc, e, dedr, dci, dcj);
                        else
                            d4_pair_sym<R, T>(d2, g0i + sj * 7, dgi + sj * 7, dgj, sw0, sw, jj, nrj, nri, wi, r4r2,
                                              sr4r2, zz, want_dc, e, dedr, dci, dcj);
                        ed += e;
                        dcn += dci;
                        gx += dedr * dx; gy += dedr * dy; gz += dedr * dz;
                        fx = -dedr * dx; fy = -dedr * dy; fz = -dedr * dz;
                    }
                }
                if (__any_sync(0xffffffffu, hit)) {
                    for (int o = 16; o > 0; o >>= 1) {
                        fx += __shfl_xor_sync(0xffffffffu, fx, o);
                        fy += __shfl_xor_sync(0xffffffffu, fy, o);
                        fz += __shfl_xor_sync(0xffffffffu, fz, o);
                    }
                    if (want_dc)
                        for (int o = 16; o > 0; o >>= 1) dcj += __shfl_xor_sync(0xffffffffu, dcj, o);
                    if (lane == 0) {
                        jacc[warp][0][jj] += fx; jacc[warp][1][jj] += fy; jacc[warp][2][jj] += fz;
                        jacc[warp][3][jj] += dcj;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
        const int j = j0 + threadIdx.x;
        double a[NA];
#pragma unroll
        for (int k = 0; k < NA; ++k) {
            a[k] = 0.0;
#pragma unroll
            for (int w = 0; w < T / 32; ++w) a[k] += jacc[w][k][threadIdx.x];
        }
        if (a[0] != 0.0) atomicAdd(V.grad + 3 * j, a[0]);
        if (a[1] != 0.0) atomicAdd(V.grad + 3 * j + 1, a[1]);
        if (a[2] != 0.0) atomicAdd(V.grad + 3 * j + 2, a[2]);
        if (a[3] != 0.0) atomicAdd(V.dEdcn + j, a[3]);
        if (a[4] != 0.0) atomicAdd(V.cfar + j, a[4]);
    }
    if (act) {
        if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
        if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
        if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
        if (dcn != 0.0) atomicAdd(V.dEdcn + i, dcn);
        if (cfar != 0.0) atomicAdd(V.cfar + i, cfar);
    }
    const int m = act ? V.mol[i] : -1;
    if constexpr (COUL) eadd(V, ec, m, T_COUL);
    if constexpr (D4) eadd(V, ed, m, T_DISP);
}

// ------------------------------------------------------------------------------------
// EEQ charge response (exact-gradient mode): with u = B M^-1 B^T w and w = dE/dq of the
// Coulomb pairs cut at 100 bohr, the gradient gains -sum_ij u_i q_j dA_ij/dr over all
// pairs (A is the uncut EEQ matrix) and u_i dx_i/dCN_i through the CN chain (k_post).
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) k_resp_pairs(View V, int nsplit)
{
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sq[kTile], su[kTile], sa[kTile];
    const int i0 = blockIdx.x * kTile, i = i0 + threadIdx.x;
    int jb, je;
    tile_range(V, i0, nsplit, jb, je);
    const bool act = i < V.n;
    const int ic = act ? i : i0;
    const double4 pi = V.pos[ic];
    const double qi = V.q[ic], ui = V.u[ic], ai = V.alpeeq[ic];
    const int2 rg = act ? V.jr[i] : make_int2(0, 0);
    const double tsp = 2.0 / 1.772453850905516;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int t0 = jb; t0 < je; t0 += kTile) {
        __syncthreads();
        const int jl = t0 + threadIdx.x;
        if (jl < je) {
            const double4 p = V.pos[jl];
            sx[threadIdx.x] = p.x; sy[threadIdx.x] = p.y; sz[threadIdx.x] = p.z;
            sq[threadIdx.x] = V.q[jl]; su[threadIdx.x] = V.u[jl]; sa[threadIdx.x] = V.alpeeq[jl];
        }
        __syncthreads();
        const int cnt = min(kTile, je - t0);
        if (!act) continue;
        for (int jj = 0; jj < cnt; ++jj) {
            const int j = t0 + jj;
            if (j == i || j < rg.x || j >= rg.y) continue;
            const double dx = pi.x - sx[jj], dy = pi.y - sy[jj], dz = pi.z - sz[jj];
            const double d2 = dx * dx + dy * dy + dz * dz;
            const double s = ai + sa[jj];
            double dadr_r;   // dA/dr / r
            if (d2 >= 36.0 * s) {
                const double ir = rsqrt(d2);
                dadr_r = -ir * ir * ir;
            } else {
                const double r = sqrt(d2), g = 1.0 / sqrt(s), gr = g * r;
                dadr_r = ((g * exp(-gr * gr) * tsp) / r - erf(gr) / d2) / r;
            }
            const double f = -(ui * sq[jj] + su[jj] * qi) * dadr_r;
            gx += f * dx; gy += f * dy; gz += f * dz;
        }
    }
    if (act) {
        if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
        if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
        if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
    }
}

// ------------------------------------------------------------------------------------
// Coulomb self terms and the CN-chain weight u = dlogCN (dE/dCN - q cnf/(2 sqrt CN))
// (ff_workspace.cpp:415-536)
// ------------------------------------------------------------------------------------
__global__ void k_post(View V)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < V.n) {
        const double q = V.q[i], cn = fmax(V.cn[i], 0.0);
        const int2 rg = V.jr[i];
        if (rg.y - rg.x >= 2 && V.alpeeq[i] > 0.0) {
            const double chi = V.chi_base[i] + V.cnf[i] * sqrt(cn);
            e = -q * chi + 0.5 * q * q * V.adiag[i];
        }
        // the EEQ charge response u adds u dx/dCN (exact-gradient mode)
        const double qe = V.u ? q - V.u[i] : q;
        V.v[i] = V.dlog[i] * (V.dEdcn[i] - qe * V.cnf[i] / (2.0 * sqrt(cn) + 1e-16));
    }
    eadd(V, e, i < V.n ? V.mol[i] : -1, T_COUL);
}

// CN chain rule: grad_i += sum_j dS_ij/dr (u_i + u_j) (x_i - x_j)/r over the 6 bohr
// neighbours (gfnff_method.cpp:5837-6260, forcefieldthread.h:80-109)
template <class R>
__global__ void __launch_bounds__(kTile) k_cn_chain(View V, int nsplit, const int* nl_bad)
{
    if (nl_bad && *nl_bad == 0) return;   // the neighbour-list kernel does the work
    __shared__ double sx[kTile], sy[kTile], sz[kTile], sr[kTile], su[kTile];
    const int i0 = blockIdx.x * kTile, i = i0 + threadIdx.x;
    int jb, je;
    tile_range(V, i0, nsplit, jb, je);
    const bool act = i < V.n;
    const double4 pi = act ? V.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const double ri = act ? V.rcov_cn[i] : 0.0;
    const double ui = act ? V.v[i] : 0.0;
    const int2 rg = act ? V.jr[i] : make_int2(0, 0);
    const double kn = -7.5, sqrtpi = 1.77245385091;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    const int ni = min(kTile, V.n - i0);
    const int w0 = i0 + (threadIdx.x & ~31), nw = max(0, min(32, V.n - w0));   // this warp's atoms
    for (int t0 = jb; t0 < je; t0 += kTile) {
        const int cnt = min(kTile, je - t0);
        if (V.boxlo && ranges_far(V, i0, ni, t0, cnt, 36.0)) continue;   // uniform in the block
        __syncthreads();
        const int jl = t0 + threadIdx.x;
        if (jl < je) {
            const double4 p = V.pos[jl];
            sx[threadIdx.x] = p.x; sy[threadIdx.x] = p.y; sz[threadIdx.x] = p.z;
            sr[threadIdx.x] = V.rcov_cn[jl];
            su[threadIdx.x] = V.v[jl];
        }
        __syncthreads();
        if (!act) continue;
        for (int js = 0; js < cnt; js += 32) {
        const int jn = min(32, cnt - js);
        if (V.boxlo && ranges_far(V, w0, nw, t0 + js, jn, 36.0)) continue;   // uniform in the warp
        for (int jj = js; jj < js + jn; ++jj) {
            double dx = sx[jj] - pi.x, dy = sy[jj] - pi.y, dz = sz[jj] - pi.z;
            if (V.cell.on) mic(V.cell, dx, dy, dz);
            const double d2 = dx * dx + dy * dy + dz * dz;
            const int j = t0 + jj;
            if (!(d2 < 36.0) || j == i || j < rg.x || j >= rg.y) continue;
            const R r = sqrt((R)d2);
            const R rs = (R)(ri + sr[jj]);
            const R dr = (r - rs) / rs;
            const R de = R(kn / sqrtpi) * exp(R(-kn * kn) * dr * dr) / rs;
            const double f = -(double)(de / r) * (ui + su[jj]);
            gx += f * dx; gy += f * dy; gz += f * dz;
        }
        }
    }
    if (act) {
        if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
        if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
        if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
    }
}

// ------------------------------------------------------------------------------------
// outputs in the caller's atom order, finiteness flags per molecule
// ------------------------------------------------------------------------------------
__global__ void k_outputs(View V, double* gout, double* qout, double* cnout, int* bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V.n) return;
    const int o = V.perm[i];
    const double gx = V.grad[3 * i], gy = V.grad[3 * i + 1], gz = V.grad[3 * i + 2];
    gout[3 * o] = gx;
    gout[3 * o + 1] = gy;
    gout[3 * o + 2] = gz;
    qout[o] = V.q[i];
    cnout[o] = V.cn[i];
    if (!isfinite(gx) || !isfinite(gy) || !isfinite(gz)) atomicOr(bad + V.mol[i], 1);
}

// per molecule: total energy, status (NOT_SPD from the EEQ factorisation, NONFINITE)
__global__ void k_finish(View V, const int* eeq_info, const int* bad, const double* e0, double* out_e)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= V.nmol) return;
    double tot = e0[m];
    for (int t = 0; t < T_TOTAL; ++t) tot += V.E[16 * m + t];
    V.E[16 * m + T_TOTAL] = tot;
    if (out_e) out_e[m] = tot;
    int st = 0;
    if (eeq_info && eeq_info[m] == 2) st = GFNFF_CUDA_ERROR;
    else if (eeq_info && eeq_info[m] == 3) st = GFNFF_REFINE_NOT_CONVERGED;
    else if (eeq_info && eeq_info[m] != 0) st = GFNFF_NOT_SPD;
    else if (!isfinite(tot) || bad[m]) st = GFNFF_NONFINITE;
    V.status[m] = st;
}

// device enumeration of the D4 pair list at the setup geometry (topology check)
__global__ void k_disp_count(int n, const double4* pos0, const int2* jr, unsigned long long* cnt, int2* out,
                             unsigned long long cap)
{
    const int i = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j <= i || j >= n || j >= jr[i].y) return;
    if (d2_exact(pos0[i], pos0[j]) <= 3600.0) {
        const unsigned long long s = atomicAdd(cnt, 1ull);
        if (out && s < cap) out[s] = make_int2(i, j);
    }
}


// ------------------------------------------------------------------------------------
// CN and CN chain rule over a Verlet neighbour list (pairs within 6 + 1 bohr at the list's
// reference geometry, same molecule; CSR by atom, both directions): a warp per atom, lanes
// over its partners.  Valid while no atom moved more than half the 1-bohr skin (checked in
// k_positions every evaluation); a stale list hands the work back to the all-pairs kernels
// above in the same launch sequence, and the host rebuilds it.  Same arithmetic per pair as
// k_cn / k_cn_chain; only the summation order of an atom's partners differs.
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(kBlock) k_cn_nl(View V, const int* __restrict__ off, const int* __restrict__ nbr,
                                                 const int* nl_bad)
{
    if (*nl_bad) return;
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= V.n) return;
    const double4 pi = V.pos[i];
    const double ri = V.rcov_cn[i];
    double s = 0.0;
    for (int p = off[i] + lane; p < off[i + 1]; p += 32) {
        const int j = nbr[p];
        const double4 pj = V.pos[j];
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < 36.0)) continue;
        s += cn_count<R>(d2, ri + V.rcov_cn[j]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0 && s != 0.0) atomicAdd(V.cnraw + i, s);
}

__global__ void __launch_bounds__(kBlock) k_cn_chain_nl(View V, const int* __restrict__ off,
                                                       const int* __restrict__ nbr, const int* nl_bad)
{
    if (*nl_bad) return;
    const int i = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= V.n) return;
    const double4 pi = V.pos[i];
    const double ri = V.rcov_cn[i], ui = V.v[i];
    const double kn = -7.5, sqrtpi = 1.77245385091;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int p = off[i] + lane; p < off[i + 1]; p += 32) {
        const int j = nbr[p];
        const double4 pj = V.pos[j];
        const double dx = pj.x - pi.x, dy = pj.y - pi.y, dz = pj.z - pi.z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < 36.0)) continue;
        const double r = sqrt(d2);
        const double rs = ri + V.rcov_cn[j];
        const double dr = (r - rs) / rs;
        const double de = (kn / sqrtpi) * exp(-kn * kn * dr * dr) / rs;
        const double f = -(de / r) * (ui + V.v[j]);
        gx += f * dx; gy += f * dy; gz += f * dz;
    }
    for (int o = 16; o > 0; o >>= 1) {
        gx += __shfl_down_sync(0xffffffffu, gx, o);
        gy += __shfl_down_sync(0xffffffffu, gy, o);
        gz += __shfl_down_sync(0xffffffffu, gz, o);
    }
    if (lane == 0) {
        if (gx != 0.0) atomicAdd(V.grad + 3 * i, gx);
        if (gy != 0.0) atomicAdd(V.grad + 3 * i + 1, gy);
        if (gz != 0.0) atomicAdd(V.grad + 3 * i + 2, gz);
    }
}

}  // namespace
