// Device-built set-up lists.
//
// Device enumeration of the hydrogen-bond terms of one molecule (gfnff_method.cpp:7936-8495,
// the host restatement is detect_hb_terms in setup/parameters.cpp), term for term in the
// host's order, so that the lists are identical:
//   * A-B pairs (i > j, taken in ascending (i, j) order) of acceptor/donor atoms with
//     bas_i aci_j or bas_j aci_i at least 1e-6 and r_ij^2 <= thr1;
//   * for a non-bonded pair: the H candidates bonded to i (term i-H...j), then those bonded
//     to j and not to i (term j-H...i), in topology-bond order; the term's case is 2, or 3
//     (acceptor O with a single C/N neighbour) or 4 (acceptor N with two neighbours);
//   * case 1: every H candidate other than i, in ascending order, bonded to neither i nor j,
//     with r_ij^2 + r_iH^2 + r_jH^2 < thr2.
// One warp per atom i: the warp scans the partners j < i 32 at a time and takes the pairs
// that pass in ascending order (ballot), then scans the H candidates 32 at a time and
// writes the case-1 terms at their ballot ranks.  A count pass, an exclusive scan and a
// fill pass place the terms.  Squared distances use round-to-nearest products and sums in
// the host's order (no contraction into FMA), so every comparison is the host's.
// The engine then sorts the terms by the squared A-B distance at the set-up geometry
// (stable radix sort: the host's stable_sort), maps them to its atom order and derives the
// bond <-> HB cross reference from the terms with an N or O acceptor.
// Included inside namespace gfnff by engine.cu, after common.cuh.
#pragma once

namespace {

struct HBDetArgs {
    int n;
    const double* x;                 // 3n, bohr, caller order
    const unsigned char* fl;         // bit 0: acceptor/donor atom, bit 1: H candidate
    const double *bas, *aci;
    const unsigned char* bcase;      // case of a term whose acceptor is this atom (2, 3, 4)
    const int *bo, *bl;              // topology-bond partners, CSR
    const int *ho, *hl;              // H candidates bonded to the atom, topology-bond order
    const int* hc;                   // all H candidates, ascending
    int nhc;
    double thr1, thr2;
    long long* cnt;                  // count pass: terms per atom i
    const long long* off;            // fill pass: first term of atom i
    int4* out;                       // (A, H, B, case), caller order
};

__device__ __forceinline__ double hb_d2(const double* __restrict__ x, int i, int j)
{
    const double dx = __dsub_rn(x[3 * i], x[3 * j]), dy = __dsub_rn(x[3 * i + 1], x[3 * j + 1]),
                 dz = __dsub_rn(x[3 * i + 2], x[3 * j + 2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ bool hb_bonded(const HBDetArgs& A, int i, int j)
{
    for (int k = A.bo[i]; k < A.bo[i + 1]; ++k)
        if (A.bl[k] == j) return true;
    return false;
}

template <bool FILL>
__global__ void __launch_bounds__(256) k_hb_detect(HBDetArgs A)
{
    const int i = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= A.n) return;   // warp-uniform
    long long pos = FILL ? A.off[i] : 0;
    long long count = 0;
    auto emit1 = [&](int a, int h, int b, int cs) {   // one term, written by lane 0
        if (FILL && lane == 0) A.out[pos + count] = make_int4(a, h, b, cs);
        ++count;
    };
    if (A.fl[i] & 1) {
        const double bi = A.bas[i], ai = A.aci[i];
        for (int j0 = 0; j0 < i; j0 += 32) {
            const int j = j0 + lane;
            bool pass = false;
            if (j < i && (A.fl[j] & 1)) {
                const double s1 = bi * A.aci[j], s2 = A.bas[j] * ai;
                if (!(s1 < 1e-6 && s2 < 1e-6)) pass = hb_d2(A.x, i, j) <= A.thr1;
            }
            unsigned m = __ballot_sync(0xffffffffu, pass);
            while (m) {
                const int jj = j0 + __ffs(m) - 1;
                m &= m - 1;
                const double rab2 = hb_d2(A.x, i, jj);
                if (!hb_bonded(A, i, jj)) {
                    for (int k = A.ho[i]; k < A.ho[i + 1]; ++k) emit1(i, A.hl[k], jj, A.bcase[jj]);
                    for (int k = A.ho[jj]; k < A.ho[jj + 1]; ++k) {
                        const int H = A.hl[k];
                        if (!hb_bonded(A, i, H)) emit1(jj, H, i, A.bcase[i]);
                    }
                }
                for (int h0 = 0; h0 < A.nhc; h0 += 32) {
                    const int hk = h0 + lane;
                    bool c1 = false;
                    int H = -1;
                    if (hk < A.nhc) {
                        H = A.hc[hk];
                        if (H != i) {
                            const double s = __dadd_rn(__dadd_rn(rab2, hb_d2(A.x, i, H)), hb_d2(A.x, jj, H));
                            c1 = s < A.thr2 && !hb_bonded(A, i, H) && !hb_bonded(A, jj, H);
                        }
                    }
                    const unsigned mm = __ballot_sync(0xffffffffu, c1);
                    if (FILL && c1) A.out[pos + count + __popc(mm & ((1u << lane) - 1u))] = make_int4(i, H, jj, 1);
                    count += __popc(mm);
                }
            }
        }
    }
    if (!FILL && lane == 0) A.cnt[i] = count;
}

// sort keys: the squared A-B distance at the set-up geometry (non-negative doubles order
// like their bit patterns), values: the term index
__global__ void k_hb_keys(long long nt, const int4* __restrict__ rec, const double* __restrict__ x0,
                          unsigned long long* key, int* val)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int4 r = rec[t];
    key[t] = (unsigned long long)__double_as_longlong(hb_d2(x0, r.x, r.z));
    val[t] = (int)t;
}

// sorted terms in the engine's atom order; near = number with a key below 100 bohr^2
__global__ void k_hb_gather(long long nt, const int4* __restrict__ rec, const int* __restrict__ order,
                            const unsigned long long* __restrict__ key, const int* __restrict__ map,
                            int4* out, int* near)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int4 r = rec[order[t]];
    out[t] = make_int4(map[r.x], map[r.y], map[r.z], r.w);
    const bool in = __longlong_as_double((long long)key[t]) < 100.0;
    const bool next_in = t + 1 < nt && __longlong_as_double((long long)key[t + 1]) < 100.0;
    if (in && !next_in) *near = (int)(t + 1);
}

// the terms that enter the bond <-> HB cross reference: an N or O acceptor, an N or O donor
// A, and (A, H) a bond term of the set-up (ffo/ffl: the bond-term partners of every atom).
// Case 2-4 terms have H bonded to A in the topology; with a refreshed topology a bond term's
// A-H pair can also be the (A, H) of a case-1 term.
__global__ void k_hb_xref_flags(long long nt, const int4* __restrict__ rec, const int* __restrict__ Z,
                                const int* __restrict__ ffo, const int* __restrict__ ffl, unsigned char* flag)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int4 r = rec[t];
    const int za = Z[r.x], zb = Z[r.z];
    bool f = (za == 7 || za == 8) && (zb == 7 || zb == 8);
    if (f) {
        bool bond = false;
        for (int k = ffo[r.y]; k < ffo[r.y + 1]; ++k) bond |= ffl[k] == r.x;
        f = bond;
    }
    flag[t] = f;
}

// CN neighbour list on the device: for every atom i the partners j of its molecule with
// |r_i - r_j|^2 < rc2 (round-to-nearest products and sums in x, y, z order), ascending; one
// warp per atom, count pass, exclusive scan, fill pass (the rows of the host grid builder)
template <bool FILL>
__global__ void __launch_bounds__(256) k_cnl_build(int n, const double4* __restrict__ p, const int2* __restrict__ jr,
                                                   double rc2, int* cnt, const int* __restrict__ off, int* js)
{
    const int i = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;   // warp-uniform
    const double4 a = p[i];
    const int2 r = jr[i];
    int count = 0;
    const int base = FILL ? off[i] : 0;
    for (int j0 = r.x; j0 < r.y; j0 += 32) {
        const int j = j0 + lane;
        bool in = false;
        if (j < r.y && j != i) {
            const double4 b = p[j];
            const double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y), dz = __dsub_rn(a.z, b.z);
            in = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)) < rc2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (FILL && in) js[base + count + __popc(m & ((1u << lane) - 1u))] = j;
        count += __popc(m);
    }
    if (!FILL && lane == 0) cnt[i] = count;
}

}  // namespace
