// GFN-FF per-geometry energy + analytic gradient on B200 (sm_100a), FP64 form.
//
// Pipeline of one evaluation (single stream, every buffer device-resident):
//   positions -> CN (erf counting, 6 bohr) -> D4 Gaussian weights + half contraction
//   -> EEQ: reduced Coulomb matrix built from the geometry, fragment constraints
//      eliminated in the null space, Cholesky solve -> charges
//   -> bonded terms (bond/angle/torsion/inversion/sTors/BATM/ATM/HB/XB, one thread per
//      term, gradient scattered with FP64 atomics)
//   -> repulsion (per-atom CSR lists) and all-pairs Coulomb + D4 dispersion (shared-
//      memory partner tiles)
//   -> self energy, CN chain rule (dE/dCN - q*cnf/(2 sqrt CN)) * dCN/dr, outputs.
//
// The engine holds one molecule or a batch of independent molecules: atoms are stored
// molecule by molecule, Morton-sorted inside each molecule, and every pair loop is
// restricted to the atom's own molecule.  The EEQ of a batch is block diagonal and is
// solved by one thread block per molecule.
//
// Every kernel restates the curcuma routine cited beside it (paths relative to
// src/core/energy_calculators/ff_methods/).
#include "engine.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <type_traits>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../../include/gfnff_b200.h"
#include "../setup/alpb.h"
#include "../tables/gfnff_tables.inc"

namespace gfnff {

#include "common.cuh"
#include "k_bonded.cuh"
#include "k_nonbonded.cuh"
#include "k_alpb.cuh"
#include "k_eeq.cuh"
#include "k_eeq_tc.cuh"
#include "k_chol.cuh"
#include "k_pcg.cuh"
#include "k_lu.cuh"
#include "k_hbdetect.cuh"
}  // namespace gfnff
#include "../setup/linalg.h"
namespace gfnff {

namespace {

inline int nblk(long n, int b = kBlock) { return (int)((n + b - 1) / b); }

// Morton order of n points (bohr): order[s] = index of the s-th point along the curve
std::vector<int> morton_order(const double* xyz, int n)
{
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    if (n < 3) return ord;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], xyz[3 * i + d]);
            hi[d] = std::max(hi[d], xyz[3 * i + d]);
        }
    double ext = 1e-12;
    for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d]);
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffULL;
        v = (v | v << 16) & 0x1f0000ff0000ffULL;
        v = (v | v << 8) & 0x100f00f00f00f00fULL;
        v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
        v = (v | v << 2) & 0x1249249249249249ULL;
        return v;
    };
    std::vector<uint64_t> code(n);
    for (int i = 0; i < n; ++i) {
        uint64_t c = 0;
        for (int d = 0; d < 3; ++d) {
            const double t = (xyz[3 * i + d] - lo[d]) / ext;
            const uint64_t q = (uint64_t)std::min(1048575.0, std::max(0.0, t * 1048575.0));
            c |= spread(q) << d;
        }
        code[i] = c;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return code[a] < code[b]; });
    return ord;
}

// Atom order inside one molecule: fragments (bonded components) contiguous, ordered
// along a Morton curve of their centroids, atoms of a fragment along a Morton curve of
// their positions.  Spatial neighbours share warps in the pair kernels, and the EEQ
// unknowns of a fragment form one contiguous range.
std::vector<int> fragment_order(const Model& m)
{
    const int n = m.n, nf = std::max(1, m.nfrag);
    std::vector<std::vector<int>> members(nf);
    for (int i = 0; i < n; ++i) members[m.frag[i]].push_back(i);
    std::vector<double> cen(3 * (size_t)nf, 0.0);
    for (int f = 0; f < nf; ++f) {
        for (int i : members[f])
            for (int d = 0; d < 3; ++d) cen[3 * f + d] += m.xyz_setup[3 * i + d];
        for (int d = 0; d < 3; ++d) cen[3 * f + d] /= std::max<size_t>(1, members[f].size());
    }
    const std::vector<int> ford = morton_order(cen.data(), nf);
    std::vector<int> ord;
    ord.reserve(n);
    for (int f : ford) {
        const auto& mem = members[f];
        std::vector<double> x(3 * mem.size());
        for (size_t k = 0; k < mem.size(); ++k)
            for (int d = 0; d < 3; ++d) x[3 * k + d] = m.xyz_setup[3 * mem[k] + d];
        for (int k : morton_order(x.data(), (int)mem.size())) ord.push_back(mem[k]);
    }
    return ord;
}

// HB terms by increasing setup distance r_AB, so that neighbouring threads of the HB
// kernel take the same branch (strong terms near the front of the list)
std::vector<int> hb_order(const Model& m)
{
    std::vector<double> d(m.hbonds.size());
    for (size_t k = 0; k < d.size(); ++k) {
        const auto& t = m.hbonds[k];
        double s = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double x = m.xyz_setup[3 * t.a + c] - m.xyz_setup[3 * t.b + c];
            s += x * x;
        }
        d[k] = s;
    }
    std::vector<int> o(d.size());
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](int x, int y) { return d[x] < d[y]; });
    return o;
}

int hb_near_count(const Model& m)
{
    int c = 0;
    for (const auto& t : m.hbonds) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double x = m.xyz_setup[3 * t.a + k] - m.xyz_setup[3 * t.b + k];
            s += x * x;
        }
        c += s < 100.0;
    }
    return c;
}

// Hydrogen-bond data for the device: one int4 {A, H, B, case} per term (set-up distance
// order) and per-atom tables, because every other term parameter is a function of one of
// the three atoms (ff_workspace_gfnff.cpp:938-1409 reads them per term; here the terms of
// one acceptor share them): charge scalings qs(q_H), qs(-q_A/B), basicity, acidity, vdW
// radius, lone-pair parameter and the N-with-one-neighbour flag of an acceptor, its carbonyl
// parent (case 3), and the bond graph (the neighbours of an acceptor and of its parent).
struct HBHost {
    std::vector<int4> rec;
    std::vector<double> qh, qa, bas, aci, rvdw, zlp;
    std::vector<int> pc, nfl;
    std::vector<std::vector<int>> nbr;
    int mismatch = 0;
    explicit HBHost(int n) : qh(n, 0.0), qa(n, 0.0), bas(n, 0.0), aci(n, 0.0), rvdw(n, 0.0), zlp(n, 1.0),
                             pc(n, -1), nfl(n, 0), nbr(n) {}
    void set(double& slot, bool& seen, double v)
    {
        if (seen && slot != v) ++mismatch;
        slot = v;
        seen = true;
    }
    static double qs(double q) { const double e = std::exp(15.0 * q); return e / (e + 1.0); }
    // the per-atom data that does not depend on the terms
    template <class Map>
    void topology(const Model& M, Map X)
    {
        for (int a = 0; a < M.n; ++a) {
            const int i = X(a);
            rvdw[i] = M.rvdw[a];
            for (int x : M.adj[a]) nbr[i].push_back(X(x));
            const int z = M.Z[a];
            zlp[i] = (z >= 1 && z <= 86) ? gfnff_tables::repz[z - 1] : 1.0;
            nfl[i] = (z == 7 && M.adj[a].size() == 1) ? 1 : 0;
        }
    }
    template <class Map>
    void add(const Model& M, Map X)
    {
        std::vector<char> sh(M.n, 0), sa(M.n, 0), sb(M.n, 0), sc(M.n, 0);
        topology(M, X);
        for (int ti : hb_order(M)) {
            const HBTerm& t = M.hbonds[ti];
            const int A = X(t.a), H = X(t.h), B = X(t.b);
            rec.push_back(make_int4(A, H, B, t.case_type));
            bool s1 = sh[t.h], s2 = sa[t.a], s3 = sa[t.b], s4 = sb[t.a], s5 = sb[t.b], s6 = sc[t.a], s7 = sc[t.b];
            set(qh[H], s1, qs(t.q_h));
            set(qa[A], s2, qs(-t.q_a));
            set(qa[B], s3, qs(-t.q_b));
            set(bas[A], s4, t.bas_a);
            set(bas[B], s5, t.bas_b);
            set(aci[A], s6, t.aci_a);
            set(aci[B], s7, t.aci_b);
            sh[t.h] = 1; sa[t.a] = sa[t.b] = 1; sb[t.a] = sb[t.b] = 1; sc[t.a] = sc[t.b] = 1;
            if (t.case_type == 3 && t.parent_c >= 0) pc[B] = X(t.parent_c);
            if (t.case_type >= 2 && t.nb_b != M.adj[t.b]) ++mismatch;
        }
    }
};

// blocks of a tiled pair kernel: enough partner slices to give every SM a few blocks
int pair_splits(int n, int max_range)
{
    const int iblocks = (n + kTile - 1) / kTile;
    const int jtiles = std::max(1, (max_range + kTile - 1) / kTile);
    const int want = (148 * 4 + iblocks - 1) / iblocks;
    return std::max(1, std::min(want, jtiles));
}

}  // namespace

// TMA descriptor of the FP32 copy of the reduced matrix (n x n, column-major, leading
// dimension lda floats, a multiple of 4) in boxes of 128 rows x 64 columns; elements past n
// read as zero.  cuTensorMapEncodeTiled comes from the driver through the runtime.
CUtensorMap tmap_f32_tiles(const float* base, int n, int lda)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)lda * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kPcgT, 64u};
    const cuuint32_t es[2] = {1u, 1u};
    const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

// ====================================================================================
// Engine implementation
// ====================================================================================
struct Engine::Impl {
    EngineOptions opt;
    cudaStream_t stream = nullptr;
    // second stream of the evaluation: the terms that do not depend on the charges (HB,
    // XB, repulsion after the positions; bonded and ATM after the CN) run beside the EEQ
    // chain and join before the CN chain rule.  GFNFF_STREAMS=1 keeps one stream.
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork0 = nullptr, ev_fork1 = nullptr, ev_join = nullptr;
    // D4 pairs, when split from the Coulomb pairs, on a stream of their own beside the side
    // terms (GFNFF_D4_STREAM=0: before them on the side stream)
    cudaStream_t side_d4 = nullptr;
    cudaEvent_t ev_join_d4 = nullptr;
    bool side_early = false;   // GFNFF_SIDE_EARLY=1: fork at the start of the evaluation
    cusolverDnHandle_t sol = nullptr;
    int n = 0, nfrag = 0, K = 0, nred = 0, nmol = 0, nsplit = 1;
    // Coulomb + D4 pairs: each pair once over a tile-pair list (default), or both
    // directions by rows (GFNFF_PAIRS=rows)
    DBuf<int2> symtiles;
    DBuf<double4> boxlo, boxhi;   // per run of kBoxAtoms atoms
    // CN neighbour list (k_cn_nl, k_cn_chain_nl): pairs within 6 + kCnSkin bohr of the
    // reference geometry cnl_ref, CSR by atom; cnl_bad = 1 once an atom moved more than
    // kCnSkin / 2 from it (GFNFF_CN_LIST=0: all-pairs kernels only)
    static constexpr double kCnSkin = 1.0;
    bool cnl_on = false;
    int* cnl_bad_host = nullptr;   // pinned; refreshed by fetch()
    DBuf<int> cnl_off, cnl_j, cnl_bad;
    DBuf<double4> cnl_ref;
    // the list from device positions d_p (engine order): k_cnl_build count, scan, fill;
    // GFNFF_CN_LIST=host builds it on the host instead (the same rows)
    DBuf<int> cnl_cnt;
    DBuf<unsigned char> cnl_tmp;
    void build_cn_list_device(const double4* d_p)
    {
        const int nn = n;
        const double rc = 6.0 + kCnSkin, rc2 = rc * rc;
        const unsigned grid = (unsigned)(((long)nn * 32 + 255) / 256);
        cnl_cnt.alloc(nn + 1);
        cnl_off.alloc(nn + 1);
        CK(cudaMemsetAsync(cnl_cnt.p + nn, 0, sizeof(int), stream));
        k_cnl_build<false><<<grid, 256, 0, stream>>>(nn, d_p, jr.p, rc2, cnl_cnt.p, nullptr, nullptr);
        CK(cudaGetLastError());
        size_t b = 0;
        CK(cub::DeviceScan::ExclusiveSum(nullptr, b, cnl_cnt.p, cnl_off.p, nn + 1, stream));
        if (cnl_tmp.n < b) cnl_tmp.alloc(b);
        b = cnl_tmp.n;
        CK(cub::DeviceScan::ExclusiveSum(cnl_tmp.p, b, cnl_cnt.p, cnl_off.p, nn + 1, stream));
        int total = 0;
        CK(cudaMemcpyAsync(&total, cnl_off.p + nn, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        cnl_j.alloc(std::max(1, total));
        k_cnl_build<true><<<grid, 256, 0, stream>>>(nn, d_p, jr.p, rc2, nullptr, cnl_off.p, cnl_j.p);
        CK(cudaGetLastError());
        cnl_ref.alloc(nn);
        CK(cudaMemcpyAsync(cnl_ref.p, d_p, (size_t)nn * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
        if (!cnl_bad.p) cnl_bad.alloc(1);
        CK(cudaMemsetAsync(cnl_bad.p, 0, sizeof(int), stream));
        CK(cudaStreamSynchronize(stream));
    }
    void build_cn_list(const std::vector<double4>& p, const std::vector<int2>& jr)
    {
        const int nn = (int)p.size();
        const double rc = 6.0 + kCnSkin, rc2 = rc * rc;
        std::vector<std::vector<int>> rows(nn);
        for (int a0 = 0; a0 < nn;) {   // per molecule (contiguous atom range)
            const int a1 = jr[a0].y;
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int i = a0; i < a1; ++i) {
                const double c[3] = {p[i].x, p[i].y, p[i].z};
                for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], c[d]); hi[d] = std::max(hi[d], c[d]); }
            }
            int dim[3];
            for (int d = 0; d < 3; ++d) dim[d] = std::max(1, std::min(256, (int)((hi[d] - lo[d]) / rc) + 1));
            auto cell = [&](const double4& q, int d) {
                const double c = d == 0 ? q.x : (d == 1 ? q.y : q.z);
                return std::min(dim[d] - 1, std::max(0, (int)((c - lo[d]) / rc)));
            };
            std::vector<std::vector<int>> grid((size_t)dim[0] * dim[1] * dim[2]);
            for (int i = a0; i < a1; ++i)
                grid[((size_t)cell(p[i], 2) * dim[1] + cell(p[i], 1)) * dim[0] + cell(p[i], 0)].push_back(i);
            for (int i = a0; i < a1; ++i) {
                const int cx = cell(p[i], 0), cy = cell(p[i], 1), cz = cell(p[i], 2);
                for (int z = std::max(0, cz - 1); z <= std::min(dim[2] - 1, cz + 1); ++z)
                    for (int y = std::max(0, cy - 1); y <= std::min(dim[1] - 1, cy + 1); ++y)
                        for (int x = std::max(0, cx - 1); x <= std::min(dim[0] - 1, cx + 1); ++x)
                            for (int j : grid[((size_t)z * dim[1] + y) * dim[0] + x]) {
                                if (j == i) continue;
                                const double dx = p[i].x - p[j].x, dy = p[i].y - p[j].y, dz = p[i].z - p[j].z;
                                if (dx * dx + dy * dy + dz * dz < rc2) rows[i].push_back(j);
                            }
                std::sort(rows[i].begin(), rows[i].end());
            }
            a0 = a1;
        }
        std::vector<int> off{0}, js;
        for (auto& r : rows) {
            js.insert(js.end(), r.begin(), r.end());
            off.push_back((int)js.size());
        }
        cnl_off.upload(off);
        cnl_j.upload(js);
        cnl_ref.upload(p);
        const int zero = 0;
        cnl_bad.upload(std::vector<int>{zero});
    }
    bool box_cull = false;        // CN kernels skip far tiles (single molecules >= 8192 atoms)
    Cell cell{};                  // periodic cell (cell.on = 0: isolated system)
    int nsym = 0;
    bool pairs_sym = true;
    bool pairs_occ = false;   // 10 blocks per SM (96 registers) instead of the unbounded 116
    int pair_tile = 64;       // tile edge of k_pairs_sym
    // Coulomb + D4 pair kernel variant, chosen at set-up by timing (tune_pairs): tile edge
    // (atoms per block side) and blocks per SM of k_pairs_sym, or both directions by rows
    enum { PAIRS_SYM32 = 0, PAIRS_SYM64 = 1, PAIRS_SYM64_OCC = 2, PAIRS_ROWS = 3 };
    int pair_variant = PAIRS_SYM64;
    DBuf<int2> symtiles32;    // tile list of the 32-atom variant (symtiles: 64)
    int nsym32 = 0;
    float pair_ms[4] = {-1.f, -1.f, -1.f, -1.f};   // the tuner's timings (ms per launch)
    // D4 pairs (charge-independent) on the side stream beside the EEQ solve, Coulomb pairs
    // after it on the main stream (GFNFF_PAIRS_SPLIT=0: both in one pass after the solve)
    int pairs_split = 1;   // 0 off, 1 unless the solver fills every SM, 2 always
    // molecule structure and atom order
    DBuf<int> mol, perm;
    DBuf<int2> jr;
    std::vector<int> h_perm, h_iperm, h_aoff;
    std::vector<int> h_anchor, h_r2a;   // EEQ null-space maps (host copies)
    DBuf<double> e0;
    // model
    DBuf<double4> pos, pos0, hbref, toporef;
    DBuf<double> rcov_cn, rcov43, rcov_d3, chi_base, cnf, gam, alpeeq, adiag, qa, refcn, w0, g0, c6ref, zeta, szr;
    DBuf<int> slot, nref;
    // EEQ structure
    DBuf<int> red2atom, atom2red, anchor, frag_off, frag_atoms, qlist, roff;
    DBuf<long long> moff;
    DBuf<double> q0;
    int nq = 0;
    long long msize = 0;
    // batched EEQ (k_eeq_batch): molecules by decreasing size, work counter, launch shape
    DBuf<int> border, bnext;
    DBuf<int4> bitems;
    int nbitems = 0;
    int batch_smem_max = 0, batch_grid = 1;
    size_t batch_smem = 0;
    // mixed form: molecules with kWarpMaxRed < nr <= kTcMaxRed are factored on the tensor
    // cores (FP32, 3xTF32 updates) and refined in FP64 against their FP64 lower tiles M64
    bool batch_tc = false;
    DBuf<double> M64;
    DBuf<long long> m64off;
    DBuf<int> refine;      // largest number of refinement corrections of the last launch
    DBuf<int4> tc_tiles;   // {molecule, R, C} of every FP64 tile (k_eeq_tc_tiles)
    int n_tc_tiles = 0;
    // bonded lists
    DBuf<int> b_i, b_j, b_h, b_off, b_hb;
    DBuf<double> b_fc, b_al, b_r0i, b_r0j, b_cki, b_ckj, b_sh, b_ff;
    DBuf<int> a_i, a_j, a_k;
    DBuf<double> a_fc, a_th;
    DBuf<int> t_i, t_j, t_k, t_l;
    DBuf<double> t_V, t_n, t_p;
    DBuf<int> s_i, s_j, s_k, s_l;
    DBuf<double> s_e;
    DBuf<int> v_i, v_j, v_k, v_l, v_t;
    DBuf<double> v_fc, v_om;
    DBuf<int> at_i, at_j, at_k;
    DBuf<double> at_c9, at_r0ij, at_r0ik, at_r0jk, at_sc;
    DBuf<int> ba_i, ba_j, ba_k;
    DBuf<double> ba_c9;
    DBuf<int4> h_rec;
    DBuf<double> h_qh, h_qa, h_bas, h_aci, h_rvdw, h_zlp;
    DBuf<int> h_pc, h_nfl, h_adjo, h_adj;
    void upload_hb_atoms(const HBHost& T)
    {
        if (T.mismatch) throw std::runtime_error("HB set-up: per-term parameters differ for one atom");
        std::vector<int> off{0}, adj;
        for (auto& l : T.nbr) {
            adj.insert(adj.end(), l.begin(), l.end());
            off.push_back((int)adj.size());
        }
        h_qh.upload(T.qh); h_qa.upload(T.qa); h_bas.upload(T.bas); h_aci.upload(T.aci);
        h_rvdw.upload(T.rvdw); h_zlp.upload(T.zlp); h_pc.upload(T.pc); h_nfl.upload(T.nfl);
        h_adjo.upload(off); h_adj.upload(adj);
    }
    void upload_hb(const HBHost& T)
    {
        upload_hb_atoms(T);
        h_rec.upload(T.rec);
        nhb = (int)T.rec.size();
    }
    // ---- HB terms detected on the device (Model::hb_on_device; k_hbdetect.cuh) ----
    struct HBDev {
        const Model* topo = nullptr;   // the model whose topology inputs are loaded
        int na = 0, nhc = 0;
        std::vector<unsigned char> bcase;
        DBuf<unsigned char> fl, bc, flag, tmp;
        DBuf<double> bas, aci, x, x0;
        DBuf<int> Zc, bo, bl, ho, hl, hc, map, val, val2, near, nsel, ffo, ffl;
        DBuf<long long> cnt, off;
        DBuf<int4> raw, xref;
        DBuf<unsigned long long> key, key2;
        long long nt = 0;
    } hbd;
    void detect_hb(const Model& m, const double* xb, std::vector<int>& bond_h, std::map<int, std::vector<int>>& byH);
    // ---- ALPB implicit solvation (single molecules; k_alpb.cuh) ----
    bool alpb_on = false;
    struct AlpbDev {
        double keps = 0.0, alpbet = 0.0, born_scale = 0.0, gshift = 0.0, srcut2 = 0.0;
        int lhb = 0;
        DBuf<double> vdwr, rho, svdw, vdwsa, trjlo, trjhi, wrp, gamsasa, hbmag;
        DBuf<double4> grid;
        DBuf<double> brad, dpsi, sasa, hbw, dhbdw, bdiag, dEdbr, shape;
    } ab;
    AlpbArgs alpb_args()
    {
        AlpbArgs A;
        A.n = n;
        A.vdwr = ab.vdwr.p; A.rho = ab.rho.p; A.svdw = ab.svdw.p; A.vdwsa = ab.vdwsa.p; A.trjlo = ab.trjlo.p;
        A.trjhi = ab.trjhi.p; A.wrp = ab.wrp.p; A.gamsasa = ab.gamsasa.p; A.hbmag = ab.hbmag.p; A.grid = ab.grid.p;
        A.keps = ab.keps; A.alpbet = ab.alpbet; A.born_scale = ab.born_scale; A.gshift = ab.gshift;
        A.srcut2 = ab.srcut2; A.lhb = ab.lhb;
        A.brad = ab.brad.p; A.dpsi = ab.dpsi.p; A.sasa = ab.sasa.p; A.hbw = ab.hbw.p; A.dhbdw = ab.dhbdw.p;
        A.bdiag = ab.bdiag.p; A.dEdbr = ab.dEdbr.p; A.shape = ab.shape.p; A.bad = bad.p;
        return A;
    }
    // per-atom ALPB data in the engine's atom order (internal atom s is caller atom h_perm[s])
    void upload_alpb(const AlpbModel& M)
    {
        alpb_on = M.on;
        if (!alpb_on) return;
        if (nmol != 1) throw std::runtime_error("ALPB solvation: single molecules only");
        auto perm_of = [&](const std::vector<double>& v) {
            std::vector<double> o(n);
            for (int s2 = 0; s2 < n; ++s2) o[s2] = v[h_perm[s2]];
            return o;
        };
        ab.keps = M.keps; ab.alpbet = M.alpbet; ab.born_scale = M.born_scale; ab.gshift = M.gshift;
        ab.srcut2 = M.srcut * M.srcut; ab.lhb = M.lhb ? 1 : 0;
        ab.vdwr.upload(perm_of(M.vdwr)); ab.rho.upload(perm_of(M.rho)); ab.svdw.upload(perm_of(M.svdw));
        ab.vdwsa.upload(perm_of(M.vdwsa)); ab.trjlo.upload(perm_of(M.trj2_lo)); ab.trjhi.upload(perm_of(M.trj2_hi));
        ab.wrp.upload(perm_of(M.wrp)); ab.gamsasa.upload(perm_of(M.gamsasa)); ab.hbmag.upload(perm_of(M.hbmag));
        std::vector<double4> g(gfnff::alpb::kNang);
        for (int p = 0; p < gfnff::alpb::kNang; ++p)
            g[p] = make_double4(M.grid[3 * p], M.grid[3 * p + 1], M.grid[3 * p + 2], M.weight[p]);
        ab.grid.upload(g);
        ab.brad.alloc(n); ab.dpsi.alloc(n); ab.sasa.alloc(n); ab.hbw.alloc(n); ab.dhbdw.alloc(n);
        ab.bdiag.alloc(n); ab.dEdbr.alloc(n); ab.shape.alloc(16);
    }
    // geometry part before the EEQ matrix; energy and gradient after the solve
    void alpb_pre(cudaStream_t s)
    {
        const View V = view();
        const AlpbArgs A = alpb_args();
        const unsigned gw = (unsigned)(((long)n * 32 + 255) / 256);
        k_alpb_born<<<gw, 256, 0, s>>>(V, A);
        k_alpb_sasa<false><<<n, kAlpbSasaThreads, 0, s>>>(V, A);
        k_alpb_shape<<<1, 256, 0, s>>>(V, A);
    }
    void alpb_post(cudaStream_t s)
    {
        const View V = view();
        const AlpbArgs A = alpb_args();
        const unsigned gw = (unsigned)(((long)n * 32 + 255) / 256);
        k_alpb_energy<<<gw, 256, 0, s>>>(V, A);
        k_alpb_chain<<<gw, 256, 0, s>>>(V, A);
        k_alpb_sasa<true><<<n, kAlpbSasaThreads, 0, s>>>(V, A);
        k_alpb_shape_grad<<<1, 256, 0, s>>>(V, A);
    }
    DBuf<int> x_a, x_x, x_b;
    DBuf<double> x_pre, x_rv;
    DBuf<int> r_off, r_j;
    DBuf<double> r_al, r_ab;
    DBuf<unsigned char> r_kind;
    // per step
    DBuf<double> cnraw, cn, dlog, w, dw, hg, hdg, q, dEdcn, v, grad, E, M, bvec, xyz_stage, msd;
    DBuf<double> gout, qout, cnout;
    DBuf<double> work;
    DBuf<int> info, info2, status, ipiv, bad;
    int lwork = 0;
    int lda = 4;           // leading dimension of M (>= nred + 1, a multiple of 4; row nred holds b for k_chol)
    bool use_lu = false;   // reduced EEQ matrix not positive definite: pivoted LU instead
    // in-house pivoted LU (k_lu_factor): grid, pivot candidates, grid barrier
    int lu_grid = 1;
    DBuf<double> lupart;
    DBuf<unsigned int> lubar;
    // EEQ solver of a single-molecule engine (chosen at upload, see upload_batch)
    enum { SOLVE_LIBRARY = 0, SOLVE_TILED = 1, SOLVE_PCG = 2, SOLVE_BATCH = 3 };
    bool batch_ready = false;   // the batched kernel's structures exist (batches, small molecules)
    int solver = SOLVE_TILED;
    // persistent tiled Cholesky (k_chol)
    DBuf<int4> ctasks;
    DBuf<int> cflags;      // next, err, cnt[nt*nt], fin[nt*nt], ydone[nt]
    DBuf<double> rdiag, ysol;
    int chol_nt = 0, chol_ntasks = 0, chol_grid = 0;
    size_t chol_smem = 0;
    void chol_launch()
    {
        CK(cudaMemsetAsync(cflags.p, 0, cflags.n * sizeof(int), stream));
        CholArgs A;
        A.M = M.p; A.lda = lda; A.n = nred; A.nt = chol_nt; A.tasks = ctasks.p; A.ntasks = chol_ntasks;
        A.next = cflags.p; A.err = cflags.p + 1; A.cnt = cflags.p + 2; A.fin = A.cnt + chol_nt * chol_nt;
        A.ydone = A.fin + chol_nt * chol_nt; A.rdiag = rdiag.p; A.y = ysol.p;
        void* args[] = {&A};
        CK(cudaLaunchCooperativeKernel((const void*)k_chol, dim3(chol_grid), dim3(kCholThreads), args, chol_smem, stream));
        k_chol_info<<<1, 1, 0, stream>>>(cflags.p + 1, info.p);
    }
    // block-Jacobi PCG (k_pcg)
    DBuf<int2> pblocks;
    DBuf<long long> pboff;
    DBuf<int4> ppart;
    DBuf<int> prblk;
    DBuf<double> px, pz, ppartial;
    DBuf<unsigned int> pbar;
    DBuf<int> piters;
    int pcg_grid = 0, pcg_max_iter = 200, pcg_maxrows = 1, pcg_maxinv = 1;
    size_t pcg_smem = 0;
    bool pcg_ready = false;
    // warm[0]: px holds the last converged solution of the main solve, warm[1]: xres of the
    // response solve; probes (pcg_warm false) start from zero so that their timing is fair
    DBuf<int> pwarm;
    bool pcg_warm = false;
    // Molecules with fragments of more than 32 unknowns (chains): the block-Jacobi inverses
    // come from the set-up geometry, computed once on the host (blocks up to 128 unknowns,
    // applied from global memory), instead of being recomputed in every launch from the
    // current matrix.  The preconditioner is then slightly stale, which costs iterations
    // only; the solve stays exact (GFNFF_PCG_PRE=0: off).
    bool pcg_pre = false;
    DBuf<double> pbinv;
    // matrices beyond L2 keep only their lower triangle; the PCG multiplies by tiles
    bool pcg_lower = false;
    // mixed form, lower-triangle PCG, GFNFF_PCG_F32=1: M stored in FP32 (half the bytes per
    // product; the solution is exact for the rounded matrix, whose charges enter the energy
    // only at second order, the EEQ energy being stationary in them).  Measured slower than
    // the FP64 form on the 20k cluster (9.2 vs 5.2 ms), so it is off by default.
    bool pcg_f32 = false;
    DBuf<float> Mf;
    DBuf<float> p32;   // k_pcg_ir: the two FP32 direction buffers
    CUtensorMap pcg_tmap{};   // k_pcg_ir: TMA descriptor of Mf (128 x 64 boxes)
    // mixed form, lower-triangle systems: k_pcg_ir (FP32-matrix CG inside FP64 refinement,
    // both triangles of M built in one pass: FP64 for the residuals, FP32 for the products)
    bool pcg_ir = false;
    size_t pcg_smem_ir = 0;
    // pipelined CG (one grid barrier per iteration; GFNFF_PCG=classic|pipelined forces one)
    bool pcg_pipe = true;
    size_t pcg_smem_pipe = 0;
    // shared-memory resident PCG (k_pcg_res, GFNFF_PCG_RES=1): the lower triangle of M lives
    // in the SMs' shared memory for the whole solve, built there from the atoms.  Measured
    // slower on 1000 waters (0.27 ms against 0.23 ms for build kernel + streamed PCG: the
    // in-kernel build runs at one 256-thread block per SM, and the atomics-based product
    // needs a second barrier per iteration), so it is off by default.
    bool pcg_res = false;
    size_t pcg_smem_res = 0;
    int pcg_res_ntiles = 0, pcg_res_ntl = 0, pcg_res_gscratch = 0;
    DBuf<int2> prtiles;
    DBuf<double> pz2;
    int pcg_cols = 1;   // 1: 4 columns per warp step, 2: 8 (GFNFF_PCG_COLS=8)
    DBuf<double> pyA;
    DBuf<int2> ptiles;
    int pcg_ntiles = 0;
    void pcg_launch(const double* rhs, double* x, int* inf, int slot)
    {
        CK(cudaMemsetAsync(pbar.p, 0, sizeof(unsigned int), stream));
        PCGArgs A;
        A.M = M.p; A.lda = lda; A.n = nred; A.b = rhs; A.x = x; A.z = pz.p; A.z2 = pz2.p;
        A.blocks = pblocks.p; A.boff = pboff.p; A.maxrows = pcg_maxrows; A.maxinv = pcg_maxinv; A.part = ppart.p; A.rblk = prblk.p; A.partial = ppartial.p;
        A.bar = pbar.p; A.info = inf; A.iters = piters.p; A.max_iter = pcg_max_iter;
        // true residual (FP64) <= 1e-12 max|b| in the FP64 form; <= 1e-10 absolute in the mixed
        // form (kRefineTol, the bar of its refined solves); not reached within max_iter:
        // REFINE_NOT_CONVERGED, and the host entry point retries with the direct solver
        A.tol = 1e-12;
        A.tol_abs = opt.precision == 1 ? kRefineTol : 0.0;
        A.warm = pcg_warm ? pwarm.p + slot : nullptr;
        A.lower = pcg_lower ? pcg_cols : 0; A.yA = pyA.p; A.tiles = ptiles.p; A.ntiles = pcg_ntiles;
        A.Mf = (pcg_f32 || pcg_ir) ? Mf.p : nullptr;
        A.p32[0] = pcg_ir ? p32.p : nullptr;
        A.p32[1] = pcg_ir ? p32.p + ((nred + 3) & ~3) : nullptr;
        A.max_outer = 6;
        {
            const char* er = std::getenv("GFNFF_PCG_IR_REL");
            A.inner_rel = er ? std::atof(er) : 1e-6;
        }
        A.binv_pre = pcg_pre ? pbinv.p : nullptr;
        void* args[] = {&A};
        if (pcg_ir) {
            void* irargs[] = {&A, &pcg_tmap};
            CK(cudaLaunchCooperativeKernel((const void*)k_pcg_ir, dim3(pcg_grid), dim3(kPcgThreads), irargs,
                                           pcg_smem_ir, stream));
        } else if (pcg_res) {
            PCGRes R{view(), red2atom.p, anchor.p, prtiles.p, pcg_res_ntiles, pcg_res_ntl, pcg_res_gscratch};
            void* rargs[] = {&A, &R};
            CK(cudaLaunchCooperativeKernel((const void*)k_pcg_res, dim3(pcg_grid), dim3(kPcgPipeThreads), rargs,
                                           pcg_smem_res, stream));
        } else if (pcg_pipe)
            CK(cudaLaunchCooperativeKernel((const void*)k_pcg_pipe, dim3(pcg_grid), dim3(kPcgPipeThreads), args,
                                           pcg_smem_pipe, stream));
        else
            CK(cudaLaunchCooperativeKernel((const void*)k_pcg, dim3(pcg_grid), dim3(kPcgThreads), args, pcg_smem,
                                           stream));
    }
    bool timing = false;
    // One evaluation is ~20 kernels and memsets.  Everything after the positions is
    // captured once as a CUDA graph and replayed while the model and the solver choice
    // stay the same (removing the per-launch host cost).  Phase timing (events between
    // phases, which cannot be timed inside a graph) and GFNFF_GRAPHS=0 use direct
    // launches, and a capture that fails falls back to them for good.
    cudaGraphExec_t graph = nullptr;
    bool graphs_ok = true;
    int graph_kernels = -1;   // kernel nodes of this library in the captured step graph
    DBuf<double> etot;   // molecule totals of the last evaluation
    // exact-gradient mode: EEQ charge response of the Coulomb pairs cut at 100 bohr
    bool resp_on = false;
    DBuf<double> cfar, ures, bres, xres;
    DBuf<int> info3;
    void drop_graphs()
    {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    // one launch of the chosen Coulomb + D4 pair kernel variant (PART: the terms)
    template <int PART>
    void launch_pairs_sym(int variant, const View& V, cudaStream_t st)
    {
        if (variant == PAIRS_SYM32)
            k_pairs_sym<double, 16, 32, PART><<<nsym32, 32, 0, st>>>(V, symtiles32.p);
        else if (variant == PAIRS_SYM64_OCC)
            k_pairs_sym<double, 10, kST, PART><<<nsym, kST, 0, st>>>(V, symtiles.p);
        else
            k_pairs_sym<double, 8, kST, PART><<<nsym, kST, 0, st>>>(V, symtiles.p);
    }
    cudaEvent_t ev[Engine::kNumPhases + 1] = {};
    void mark(int k)
    {
        if (timing) CK(cudaEventRecord(ev[k], stream));
    }
    int nb = 0, na = 0, nt = 0, ns = 0, ninv = 0, natm = 0, nbatm = 0, nhb = 0, nxb = 0;
    int nhb_near = 0;   // HB terms (sorted by setup r_AB) with setup r_AB < 10 bohr

    View view() const
    {
        View V;
        V.n = n; V.nfrag = nfrag; V.K = K; V.nred = nred; V.nmol = nmol;
        V.mol = mol.p; V.jr = jr.p; V.perm = perm.p;
        V.pos = pos.p; V.pos0 = pos0.p; V.rcov_cn = rcov_cn.p; V.rcov43 = rcov43.p; V.rcov_d3 = rcov_d3.p;
        V.chi_base = chi_base.p; V.cnf = cnf.p; V.gam = gam.p; V.alpeeq = alpeeq.p; V.adiag = adiag.p; V.qa = qa.p;
        V.slot = slot.p; V.nref = nref.p; V.refcn = refcn.p; V.w0 = w0.p; V.g0 = g0.p; V.c6ref = c6ref.p;
        V.zeta = zeta.p; V.szr = szr.p;
        V.cnraw = cnraw.p; V.cn = cn.p; V.dlog = dlog.p; V.w = w.p; V.dw = dw.p; V.hg = hg.p; V.hdg = hdg.p;
        V.q = q.p; V.dEdcn = dEdcn.p; V.v = v.p; V.grad = grad.p; V.E = E.p; V.status = status.p;
        V.brad = alpb_on ? ab.brad.p : nullptr;
        V.bdiag = alpb_on ? ab.bdiag.p : nullptr;
        V.keps = alpb_on ? ab.keps : 0.0;
        V.exact = opt.exact_gradient ? 1 : 0;
        V.cfar = resp_on ? cfar.p : nullptr;
        V.u = resp_on ? ures.p : nullptr;
        V.boxlo = box_cull ? boxlo.p : nullptr;
        V.boxhi = box_cull ? boxhi.p : nullptr;
        V.cell = cell;
        return V;
    }
    // caller index (molecule m, local atom a) -> internal index
    int ix(int m, int a) const { return h_iperm[h_aoff[m] + a]; }
};

Engine::Engine(const EngineOptions& opt) : p_(new Impl)
{
    p_->opt = opt;
    CK(cudaSetDevice(opt.device));
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    // the EEQ chain is the critical path: its stream gets the higher priority
    CK(cudaStreamCreateWithPriority(&p_->stream, cudaStreamNonBlocking, hi));
    const char* se = std::getenv("GFNFF_SIDE_EARLY");
    p_->side_early = se && !std::strcmp(se, "1");
    const char* st = std::getenv("GFNFF_STREAMS");
    if (!(st && !std::strcmp(st, "1"))) {
        CK(cudaStreamCreateWithPriority(&p_->side, cudaStreamNonBlocking, lo));
        CK(cudaEventCreateWithFlags(&p_->ev_fork0, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&p_->ev_fork1, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&p_->ev_join, cudaEventDisableTiming));
        const char* ds = std::getenv("GFNFF_D4_STREAM");
        if (!(ds && !std::strcmp(ds, "0"))) {
            CK(cudaStreamCreateWithPriority(&p_->side_d4, cudaStreamNonBlocking, lo));
            CK(cudaEventCreateWithFlags(&p_->ev_join_d4, cudaEventDisableTiming));
        }
    }
    CS(cusolverDnCreate(&p_->sol));
    CS(cusolverDnSetStream(p_->sol, p_->stream));
}

const char* const Engine::kPhaseNames[] = {"positions", "cn", "d4_weights", "eeq_matrix", "eeq_rhs",
                                           "eeq_solve", "bonded", "hbonds", "repulsion", "pairs",
                                           "post_chain", "finish"};

void Engine::set_timing(bool on)
{
    if (on && !p_->ev[0])
        for (int k = 0; k <= kNumPhases; ++k) CK(cudaEventCreate(&p_->ev[k]));
    p_->timing = on;
}

std::vector<double> Engine::phase_ms()
{
    std::vector<double> out(kNumPhases, 0.0);
    if (!p_->timing) return out;
    CK(cudaEventSynchronize(p_->ev[kNumPhases]));
    for (int k = 0; k < kNumPhases; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p_->ev[k], p_->ev[k + 1]));
        out[k] = ms;
    }
    return out;
}

Engine::~Engine()
{
    p_->drop_graphs();
    for (auto& e : p_->ev)
        if (e) cudaEventDestroy(e);
    if (p_->sol) cusolverDnDestroy(p_->sol);
    if (p_->cnl_bad_host) cudaFreeHost(p_->cnl_bad_host);
    for (cudaEvent_t e : {p_->ev_fork0, p_->ev_fork1, p_->ev_join, p_->ev_join_d4})
        if (e) cudaEventDestroy(e);
    if (p_->side) cudaStreamDestroy(p_->side);
    if (p_->side_d4) cudaStreamDestroy(p_->side_d4);
    if (p_->stream) cudaStreamDestroy(p_->stream);
}

// HB terms of a single molecule detected on the device at xb (bohr, caller order): the
// topology inputs once per model, the geometry-dependent basicity at every detection; the
// terms sorted into h_rec, the bond cross reference returned for the bond upload
void Engine::Impl::detect_hb(const Model& m, const double* xb, std::vector<int>& bond_h,
                             std::map<int, std::vector<int>>& byH)
{
    HBDev& D = hbd;
    const int na = m.n;
    cudaStream_t s = stream;
    const HBAtoms at = hb_atom_data(const_cast<Model&>(m), xb);
    auto X = [&](int a) { return ix(0, a); };
    if (D.topo != &m) {
        D.na = na;
        std::vector<int> Zc(m.Z.begin(), m.Z.end());
        std::vector<std::vector<int>> part(na), hyd(na);
        for (auto& b : m.topo_bonds) {
            part[b.first].push_back(b.second);
            part[b.second].push_back(b.first);
            if (at.hcand[b.first]) hyd[b.second].push_back(b.first);
            if (at.hcand[b.second]) hyd[b.first].push_back(b.second);
        }
        auto csr = [](const std::vector<std::vector<int>>& l, std::vector<int>& o, std::vector<int>& v) {
            o.assign(1, 0);
            v.clear();
            for (auto& r : l) {
                v.insert(v.end(), r.begin(), r.end());
                o.push_back((int)v.size());
            }
        };
        std::vector<int> bo, bl, ho, hl, hc, map(na), ffo, ffl;
        csr(part, bo, bl);
        csr(hyd, ho, hl);
        {
            std::vector<std::vector<int>> ff(na);   // partners of the set-up's bond terms
            for (const auto& bd : m.bonds) {
                ff[bd.i].push_back(bd.j);
                ff[bd.j].push_back(bd.i);
            }
            csr(ff, ffo, ffl);
        }
        std::vector<unsigned char> fl(na);
        D.bcase.assign(na, 2);
        for (int a = 0; a < na; ++a) {
            fl[a] = (at.ok[a] ? 1 : 0) | (at.hcand[a] ? 2 : 0);
            if (at.hcand[a]) hc.push_back(a);
            map[a] = X(a);
            const int z = m.Z[a];
            if (z == 8 && m.adj[a].size() == 1) {
                const int p = m.adj[a][0];
                if (m.Z[p] == 6 || m.Z[p] == 7) D.bcase[a] = 3;
            } else if (z == 7 && m.adj[a].size() == 2) {
                D.bcase[a] = 4;
            }
        }
        D.nhc = (int)hc.size();
        D.Zc.upload(Zc); D.bo.upload(bo); D.bl.upload(bl); D.ho.upload(ho); D.hl.upload(hl);
        D.hc.upload(hc); D.map.upload(map); D.fl.upload(fl); D.bc.upload(D.bcase);
        D.ffo.upload(ffo); D.ffl.upload(ffl.empty() ? std::vector<int>{0} : ffl);
        D.aci.upload(at.aci);
        D.x0.upload(m.xyz_setup);
        D.cnt.alloc(na); D.off.alloc(na); D.near.alloc(1); D.nsel.alloc(1);
        D.topo = &m;
    }
    D.x.upload(std::vector<double>(xb, xb + 3 * (size_t)na));
    D.bas.upload(at.bas);
    // the engine's per-atom HB data (every atom; the kernel reads those of its terms)
    {
        HBHost T(n);
        T.topology(m, X);
        for (int a = 0; a < na; ++a) {
            const int i = X(a);
            T.qh[i] = HBHost::qs(m.qa[a]);
            T.qa[i] = HBHost::qs(-m.qa[a]);
            T.bas[i] = at.bas[a];
            T.aci[i] = at.aci[a];
            if (D.bcase[a] == 3) T.pc[i] = X(m.adj[a][0]);
        }
        upload_hb_atoms(T);
    }
    HBDetArgs A{na, D.x.p, D.fl.p, D.bas.p, D.aci.p, D.bc.p, D.bo.p, D.bl.p, D.ho.p, D.hl.p, D.hc.p, D.nhc,
                at.thr1, at.thr2, D.cnt.p, D.off.p, nullptr};
    const unsigned grid = (unsigned)(((long)na * 32 + 255) / 256);
    k_hb_detect<false><<<grid, 256, 0, s>>>(A);
    CK(cudaGetLastError());
    size_t need = 0, b = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, b, D.cnt.p, D.off.p, na, s));
    need = b;
    if (D.tmp.n < need) D.tmp.alloc(need);
    CK(cub::DeviceScan::ExclusiveSum(D.tmp.p, b, D.cnt.p, D.off.p, na, s));
    long long last[2] = {0, 0};
    CK(cudaMemcpyAsync(&last[0], D.off.p + na - 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&last[1], D.cnt.p + na - 1, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const long long nt = last[0] + last[1];
    if (nt > (long long)std::numeric_limits<int>::max() / 2) throw std::runtime_error("HB detection: too many terms");
    D.nt = nt;
    int near = 0;
    std::vector<int4> xr;
    if (nt > 0) {
        const int ni = (int)nt;
        D.raw.alloc(ni); D.key.alloc(ni); D.key2.alloc(ni); D.val.alloc(ni); D.val2.alloc(ni);
        D.flag.alloc(ni); D.xref.alloc(ni);
        A.out = D.raw.p;
        k_hb_detect<true><<<grid, 256, 0, s>>>(A);
        const unsigned g2 = (unsigned)((nt + 255) / 256);
        k_hb_keys<<<g2, 256, 0, s>>>(nt, D.raw.p, D.x0.p, D.key.p, D.val.p);
        CK(cub::DeviceRadixSort::SortPairs(nullptr, b, D.key.p, D.key2.p, D.val.p, D.val2.p, ni, 0, 64, s));
        need = b;
        CK(cub::DeviceSelect::Flagged(nullptr, b, D.raw.p, D.flag.p, D.xref.p, D.nsel.p, ni, s));
        need = std::max(need, b);
        if (D.tmp.n < need) D.tmp.alloc(need);
        b = D.tmp.n;
        CK(cub::DeviceRadixSort::SortPairs(D.tmp.p, b, D.key.p, D.key2.p, D.val.p, D.val2.p, ni, 0, 64, s));
        h_rec.alloc(ni);
        CK(cudaMemsetAsync(D.near.p, 0, sizeof(int), s));
        k_hb_gather<<<g2, 256, 0, s>>>(nt, D.raw.p, D.val2.p, D.key2.p, D.map.p, h_rec.p, D.near.p);
        k_hb_xref_flags<<<g2, 256, 0, s>>>(nt, D.raw.p, D.Zc.p, D.ffo.p, D.ffl.p, D.flag.p);
        b = D.tmp.n;
        CK(cub::DeviceSelect::Flagged(D.tmp.p, b, D.raw.p, D.flag.p, D.xref.p, D.nsel.p, ni, s));
        int nsel = 0;
        CK(cudaMemcpyAsync(&near, D.near.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&nsel, D.nsel.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        xr.resize(nsel);
        if (nsel) CK(cudaMemcpy(xr.data(), D.xref.p, (size_t)nsel * sizeof(int4), cudaMemcpyDeviceToHost));
        CK(cudaGetLastError());
    } else {
        h_rec.free();
    }
    nhb = (int)nt;
    nhb_near = near;
    // bond -> (H, acceptors): the A-H bonds of an N or O donor with terms of that pair, the
    // acceptors in detection order (the host cross reference, gfnff_method.cpp:3680-3712)
    std::map<std::pair<int, int>, std::vector<int>> ahb;
    for (const int4& r : xr) ahb[{r.x, r.y}].push_back(r.z);
    bond_h.assign(m.bonds.size(), -1);
    byH.clear();
    for (size_t k = 0; k < m.bonds.size(); ++k) {
        const auto& bd = m.bonds[k];
        int H = -1, Ad = -1;
        if (m.Z[bd.i] == 1) { H = bd.i; Ad = bd.j; }
        else if (m.Z[bd.j] == 1) { H = bd.j; Ad = bd.i; }
        else continue;
        if (m.Z[Ad] != 7 && m.Z[Ad] != 8) continue;
        auto it = ahb.find({Ad, H});
        if (it == ahb.end() || it->second.empty()) continue;
        bond_h[k] = H;
        byH[H].insert(byH[H].end(), it->second.begin(), it->second.end());
    }
}

std::vector<int> Engine::hb_terms() const
{
    const Impl& P = *p_;
    std::vector<int> v;
    if (P.hbd.topo == nullptr || P.hbd.nt == 0) return v;
    std::vector<int4> r((size_t)P.hbd.nt);
    CK(cudaStreamSynchronize(P.stream));
    CK(cudaMemcpy(r.data(), P.hbd.raw.p, r.size() * sizeof(int4), cudaMemcpyDeviceToHost));
    v.reserve(4 * r.size());
    for (auto& t : r) v.insert(v.end(), {t.x, t.y, t.z, t.w});
    return v;
}

long long Engine::hb_count() const { return p_->nhb; }

void Engine::upload_hbxb(const Model& m, const double* hb_xyz_bohr)
{
    p_->drop_graphs();
    if (p_->nmol != 1) throw std::runtime_error("upload_hbxb: single-molecule engines only");
    Impl& P = *p_;
    auto X = [&](int a) { return P.ix(0, a); };
    // HB terms: the model's host lists, or detected here on the device (hb_on_device);
    // either way the bond -> (H, acceptors) cross reference for the bond modulation
    std::vector<int> bond_h(m.bonds.size(), -1);
    std::map<int, std::vector<int>> byH;
    if (!m.hb_on_device) {
        for (auto& e : m.bond_hb) byH[e.h].insert(byH[e.h].end(), e.b_atoms.begin(), e.b_atoms.end());
        for (size_t k = 0; k < m.bonds.size(); ++k)
            if (m.bonds[k].nr_hb >= 1) bond_h[k] = m.bonds[k].hb_h;
        HBHost T(P.n);
        T.add(m, X);
        P.upload_hb(T);
        P.nhb_near = hb_near_count(m);
    } else {
        P.detect_hb(m, hb_xyz_bohr ? hb_xyz_bohr : m.xyz_setup.data(), bond_h, byH);
    }
    // bonds carry the HB modulation data
    {
        std::vector<int> bi, bj, bh, off{0}, hb;
        std::vector<double> fc, al, r0i, r0j, cki, ckj, sh, ff;
        for (size_t k = 0; k < m.bonds.size(); ++k) {
            const auto& b = m.bonds[k];
            bi.push_back(X(b.i)); bj.push_back(X(b.j));
            fc.push_back(b.fc); al.push_back(b.alpha); r0i.push_back(b.r0_base_i); r0j.push_back(b.r0_base_j);
            cki.push_back(b.cnfak_i); ckj.push_back(b.cnfak_j); sh.push_back(b.rabshift); ff.push_back(b.ff);
            const int H = bond_h[k];
            bh.push_back(H >= 0 ? X(H) : -1);
            if (H >= 0) for (int a : byH[H]) hb.push_back(X(a));
            off.push_back((int)hb.size());
        }
        P.nb = (int)m.bonds.size();
        P.b_i.upload(bi); P.b_j.upload(bj); P.b_h.upload(bh); P.b_off.upload(off); P.b_hb.upload(hb);
        P.b_fc.upload(fc); P.b_al.upload(al); P.b_r0i.upload(r0i); P.b_r0j.upload(r0j);
        P.b_cki.upload(cki); P.b_ckj.upload(ckj); P.b_sh.upload(sh); P.b_ff.upload(ff);
    }
    {
        std::vector<int> a, x, b;
        std::vector<double> pre, rv;
        auto qs = [](double q, double st, double sf) { const double e = std::exp(st * q); return e / (e + sf); };
        for (auto& t : m.xbonds) {
            a.push_back(X(t.a)); x.push_back(X(t.x)); b.push_back(X(t.b));
            pre.push_back(-qs(-t.q_b, 15.0, 0.03) * t.aci_x * qs(t.q_x, 15.0, 0.03));
            rv.push_back(m.rvdw[t.a] + m.rvdw[t.b]);
        }
        P.nxb = (int)m.xbonds.size();
        P.x_a.upload(a); P.x_x.upload(x); P.x_b.upload(b); P.x_pre.upload(pre); P.x_rv.upload(rv);
    }
}

void Engine::upload(const Model& m, const AlpbModel* solv) { upload_batch({&m}, solv); }

void Engine::upload_batch(const std::vector<const Model*>& mols, const AlpbModel* solv)
{
    Impl& P = *p_;
    P.drop_graphs();
    {
        const char* env = std::getenv("GFNFF_GRAPHS");
        P.graphs_ok = !(env && env[0] == '0');
    }
    CK(cudaSetDevice(P.opt.device));
    if (mols.empty()) throw std::runtime_error("upload: no molecules");
    P.hbd.topo = nullptr;
    const int nm = (int)mols.size();
    if (P.cell.on && nm > 1) throw std::runtime_error("upload: a periodic cell needs a single molecule");
    P.nmol = nm;
    // ---- atom order: molecules contiguous, Morton order inside each molecule ----
    P.h_aoff.assign(nm + 1, 0);
    for (int m = 0; m < nm; ++m) P.h_aoff[m + 1] = P.h_aoff[m] + mols[m]->n;
    const int n = P.h_aoff[nm];
    P.n = n;
    P.h_perm.resize(n);
    P.h_iperm.resize(n);
    std::vector<int> hmol(n);
    std::vector<int2> hjr(n);
    for (int m = 0; m < nm; ++m) {
        const int a0 = P.h_aoff[m], na = mols[m]->n;
        auto ord = fragment_order(*mols[m]);
        for (int s = 0; s < na; ++s) {
            P.h_perm[a0 + s] = a0 + ord[s];
            P.h_iperm[a0 + ord[s]] = a0 + s;
            hmol[a0 + s] = m;
            hjr[a0 + s] = make_int2(a0, a0 + na);
        }
    }
    P.perm.upload(P.h_perm);
    P.mol.upload(hmol);
    P.jr.upload(hjr);
    int max_range = 0;
    for (int m = 0; m < nm; ++m) max_range = std::max(max_range, mols[m]->n);
    P.nsplit = pair_splits(n, max_range);
    {   // tile pairs (i tile <= j tile, both within the tile's molecules) of k_pairs_sym
        // both tile edges (the tuner picks one): tile pairs I <= J within the rows' molecules
        auto tiles = [&](int T) {
            std::vector<int2> tl;
            const int nt = (n + T - 1) / T;
            for (int I = 0; I < nt; ++I) {
                const int i0 = I * T, hi = hjr[std::min(n, i0 + T) - 1].y;
                for (int J = I; J * T < hi; ++J) tl.push_back(make_int2(i0, J * T));
            }
            return tl;
        };
        const std::vector<int2> tl = tiles(kST), tl32 = tiles(32);
        P.symtiles.upload(tl);
        P.symtiles32.upload(tl32);
        P.nsym32 = (int)tl32.size();
        P.pair_tile = nm > 1 ? 32 : kST;
        P.boxlo.alloc((n + kBoxAtoms - 1) / kBoxAtoms);
        P.boxhi.alloc((n + kBoxAtoms - 1) / kBoxAtoms);
        // box tests compare plain coordinates: off in a periodic cell
        P.box_cull = nm == 1 && n >= 8192 && !P.cell.on;
        P.nsym = (int)tl.size();
        const char* pe = std::getenv("GFNFF_PAIRS");
        P.pairs_sym = !(pe && !std::strcmp(pe, "rows"));
        const char* po = std::getenv("GFNFF_PAIRS_OCC");
        P.pairs_occ = po && !std::strcmp(po, "1");
        // the variant before tuning (batches: 32-atom tiles, which straddle fewer molecules)
        P.pair_variant = !P.pairs_sym ? Impl::PAIRS_ROWS
                         : (P.pair_tile == 32 ? Impl::PAIRS_SYM32
                                              : (P.pairs_occ ? Impl::PAIRS_SYM64_OCC : Impl::PAIRS_SYM64));
        const char* ps = std::getenv("GFNFF_PAIRS_SPLIT");
        P.pairs_split = !ps ? 1 : (!std::strcmp(ps, "0") ? 0 : (!std::strcmp(ps, "1") ? 2 : 1));
    }
    // ---- global element table (union of the molecules' D4 element slots) ----
    std::vector<int> gZ;
    std::vector<std::vector<int>> gslot(nm);
    for (int m = 0; m < nm; ++m) {
        for (int z : mols[m]->present_Z) {
            auto it = std::find(gZ.begin(), gZ.end(), z);
            gslot[m].push_back(it == gZ.end() ? (gZ.push_back(z), (int)gZ.size() - 1) : (int)(it - gZ.begin()));
        }
    }
    const int K = (int)gZ.size();
    P.K = K;
    std::vector<double> c6g((size_t)K * K * 49, 0.0);
    {
        std::vector<char> have((size_t)K * K, 0);
        for (int m = 0; m < nm; ++m) {
            const Model& M = *mols[m];
            const int km = (int)M.present_Z.size();
            for (int a = 0; a < km; ++a)
                for (int b = 0; b < km; ++b) {
                    const int ga = gslot[m][a], gb = gslot[m][b];
                    if (have[(size_t)ga * K + gb]) continue;
                    have[(size_t)ga * K + gb] = 1;
                    std::copy_n(&M.c6ref[((size_t)a * km + b) * 49], 49, &c6g[((size_t)ga * K + gb) * 49]);
                }
        }
    }
    // ---- per-atom data in internal order ----
    std::vector<double4> p0(n);
    std::vector<double> rcn(n), r43(n), rd3(n), chi(n), cnf(n), gam(n), alp(n), adg(n), qa(n), zeta(n), szr(n);
    std::vector<double> rcn7((size_t)n * 7), w07((size_t)n * 7), g0((size_t)n * K * 7, 0.0);
    std::vector<int> slot(n), nref(n);
    std::vector<double> e0(nm);
    for (int m = 0; m < nm; ++m) {
        const Model& M = *mols[m];
        e0[m] = M.e0;
        for (int a = 0; a < M.n; ++a) {
            const int s = P.ix(m, a);
            p0[s] = make_double4(M.xyz_setup[3 * a], M.xyz_setup[3 * a + 1], M.xyz_setup[3 * a + 2], 0.0);
            rcn[s] = M.rcov_cn[a]; r43[s] = M.rcov_d3[a] * (4.0 / 3.0); rd3[s] = M.rcov_d3[a];
            chi[s] = M.chi_base[a]; cnf[s] = M.cnf[a]; gam[s] = M.gam[a]; alp[s] = M.alpeeq[a];
            adg[s] = M.gam[a] + 0.797884560802866 / std::sqrt(M.alpeeq[a]);
            qa[s] = M.qa[a]; zeta[s] = M.zeta[a]; szr[s] = M.sqrt_zr4r2[a];
            slot[s] = gslot[m][M.slot[a]]; nref[s] = M.nref[a];
            for (int r = 0; r < 7; ++r) { rcn7[(size_t)s * 7 + r] = M.refcn[(size_t)a * 7 + r]; w07[(size_t)s * 7 + r] = M.w_setup[(size_t)a * 7 + r]; }
            // frozen half contraction at the setup weights (d4param_generator.cpp:1235-1290)
            for (int t = 0; t < K; ++t) {
                const double* C = &c6g[(((size_t)slot[s] * K + t) * 7) * 7];
                for (int b = 0; b < 7; ++b) {
                    double v = 0.0;
                    for (int r = 0; r < nref[s]; ++r) v += w07[(size_t)s * 7 + r] * C[r * 7 + b];
                    g0[((size_t)s * K + t) * 7 + b] = v;
                }
            }
        }
    }
    P.pos0.upload(p0); P.hbref.upload(p0); P.toporef.upload(p0); P.pos.alloc(n);
    {
        // the CN neighbour list is built from plain distances: a periodic cell takes the
        // all-pairs CN kernels, which apply the minimum image to every pair
        const char* ecl = std::getenv("GFNFF_CN_LIST");
        P.cnl_on = !(ecl && !std::strcmp(ecl, "0")) && !P.cell.on;
        if (P.cnl_on) {
            if (!P.cnl_bad_host) CK(cudaMallocHost(&P.cnl_bad_host, sizeof(int)));
            *P.cnl_bad_host = 0;
            if (ecl && !std::strcmp(ecl, "host")) P.build_cn_list(p0, hjr);
            else P.build_cn_list_device(P.pos0.p);
        }
    }
    P.rcov_cn.upload(rcn); P.rcov43.upload(r43); P.rcov_d3.upload(rd3);
    P.chi_base.upload(chi); P.cnf.upload(cnf); P.gam.upload(gam); P.alpeeq.upload(alp); P.adiag.upload(adg);
    P.qa.upload(qa); P.slot.upload(slot); P.nref.upload(nref); P.refcn.upload(rcn7); P.w0.upload(w07);
    P.c6ref.upload(c6g); P.zeta.upload(zeta); P.szr.upload(szr); P.g0.upload(g0); P.e0.upload(e0);
    // ---- EEQ null-space structure (global fragment ids, reduced index per molecule) ----
    {
        std::vector<int> fragi(n);
        std::vector<double> qf;
        int fbase = 0;
        for (int m = 0; m < nm; ++m) {
            const Model& M = *mols[m];
            for (int a = 0; a < M.n; ++a) fragi[P.ix(m, a)] = fbase + M.frag[a];
            for (int f = 0; f < M.nfrag; ++f) qf.push_back(M.qfrag[f]);
            fbase += M.nfrag;
        }
        const int nf = fbase;
        P.nfrag = nf;
        std::vector<int> first(nf, -1), cntf(nf, 0), anchor(n), a2r(n), r2a, roff{0}, ql;
        std::vector<long long> moff;
        std::vector<double> q0(n);
        for (int i = 0; i < n; ++i) { const int f = fragi[i]; if (first[f] < 0) first[f] = i; ++cntf[f]; }
        long long ms = 0;
        for (int m = 0; m < nm; ++m) {
            for (int i = P.h_aoff[m]; i < P.h_aoff[m + 1]; ++i) {
                const int f = fragi[i];
                anchor[i] = first[f];
                q0[i] = qf[f] / (double)cntf[f];
                if (q0[i] != 0.0) ql.push_back(i);
                if (i == first[f]) a2r[i] = -f - 1;
                else { a2r[i] = (int)r2a.size(); r2a.push_back(i); }
            }
            const int nr = (int)r2a.size() - roff.back();
            moff.push_back(ms);
            ms += (long long)(nr + 1) * nr;   // only used by molecules beyond the shared-memory path
            roff.push_back((int)r2a.size());
        }
        std::vector<int> off(nf + 1, 0), fa(n);
        for (int f = 0; f < nf; ++f) off[f + 1] = off[f] + cntf[f];
        std::vector<int> fill = off;
        for (int i = 0; i < n; ++i) fa[fill[fragi[i]]++] = i;
        P.nred = (int)r2a.size();
        P.msize = ms;
        P.nq = (int)ql.size();
        P.anchor.upload(anchor); P.atom2red.upload(a2r); P.red2atom.upload(r2a);
        P.h_anchor = anchor;
        P.h_r2a = r2a;
        P.frag_off.upload(off); P.frag_atoms.upload(fa); P.q0.upload(q0); P.qlist.upload(ql);
        P.roff.upload(roff); P.moff.upload(moff);
        // batches, and single molecules small enough for the batched kernel's staging
        // (a candidate EEQ solver for them)
        P.batch_ready = nm > 1 || n <= kStageAtoms;
        if (P.batch_ready) {
            std::vector<int> ord(nm);
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(),
                             [&](int x, int y) { return roff[x + 1] - roff[x] > roff[y + 1] - roff[y]; });
            P.border.upload(ord);
            P.bnext.alloc(1);
            // mixed form: the tensor-core path (k_eeq_tc.cuh) for every molecule of at most
            // kTcMaxRed unknowns (GFNFF_BATCH_TC=0: the FP64 paths)
            const char* etc = std::getenv("GFNFF_BATCH_TC");
            P.batch_tc = P.opt.precision == 1 && !(etc && !std::strcmp(etc, "0"));
            // work items: large molecules one per block, small ones in packs of kWarpMols
            // (one warp each, FP64); in the mixed form every molecule is a block item (one
            // small molecule on a block's tensor-core path measured far below a warp item of
            // eight, whose column-by-column FP64 updates are latency-bound)
            std::vector<int4> items;
            for (int k = 0; k < nm;) {
                const int nr = roff[ord[k] + 1] - roff[ord[k]];
                if (P.batch_tc || nr > kWarpMaxRed || mols[ord[k]]->n > kWarpAtoms) {
                    items.push_back(make_int4(k, 1, 0, 0));
                    ++k;
                } else {
                    const int cnt = std::min(kWarpMols, nm - k);
                    items.push_back(make_int4(k, cnt, 1, 0));
                    k += cnt;
                }
            }
            P.bitems.upload(items);
            P.nbitems = (int)items.size();
            // shared-memory path: staged atoms + packed (nr+1) x nr matrix + two vectors
            // within ~210 KB
            const long long budget = 210 * 1024 / 8 - kStageDoubles - kStageInts / 2;
            int smax = 0;
            while ((long long)(smax + 1) * (smax + 4) / 2 + 2 * (smax + 1) + 1 <= budget) ++smax;
            int big = 0;
            for (int m = 0; m < nm; ++m) big = std::max(big, roff[m + 1] - roff[m]);
            const int fit = std::min(big, smax);
            P.batch_smem_max = smax;
            int bigatoms = 0;
            for (int m = 0; m < nm; ++m) bigatoms = std::max(bigatoms, mols[m]->n);
            if (bigatoms > kStageAtoms)
                throw std::runtime_error("batch: molecules of at most " + std::to_string(kStageAtoms) + " atoms");
            // the two-stage path for larger molecules holds its first s = nr - smax columns
            // (rows c..nr) and later the trailing block in turn; both must fit the budget
            if (big > smax) {
                const long long sp = big - smax;
                if (sp * (big + 1) - sp * (sp - 1) / 2 > budget)
                    throw std::runtime_error("batch: molecule too large for the batched EEQ");
            }
            P.batch_smem = ((size_t)kStageDoubles + kStageInts / 2 +
                            (big > smax ? (size_t)budget : (size_t)fit * (fit + 3) / 2 + 2 * (size_t)(fit + 1) + 2)) *
                           8;
            P.batch_smem = std::max<size_t>(P.batch_smem, (size_t)kWarpMols * kWarpRegion * 8);
            // mixed form: FP64 lower tiles of the molecules of the tensor-core path
            if (P.batch_tc) {
                // molecules with at most kTcMaxRed unknowns: their FP64 tiles (built at full
                // occupancy by k_eeq_tc_tiles)
                std::vector<long long> o64(nm, 0);
                std::vector<int4> tl;
                long long tot = 0;
                for (int m = 0; m < nm; ++m) {
                    const int nr = roff[m + 1] - roff[m];
                    o64[m] = tot;
                    if (nr < 1 || nr > kTcMaxRed) continue;
                    const int T = (nr + 31) / 32;
                    for (int R = 0; R < T; ++R)
                        for (int C = 0; C <= R; ++C) tl.push_back(make_int4(m, R, C, 0));
                    tot += (long long)T * (T + 1) / 2 * 1024;
                }
                P.m64off.upload(o64);
                P.M64.alloc((size_t)std::max<long long>(1, tot));
                P.tc_tiles.upload(tl);
                P.n_tc_tiles = (int)tl.size();
                // work items by estimated time, longest first (measured on the 512-conformer
                // batch: a tensor-core molecule ~0.75 us per unknown, a warp item of eight
                // small FP64 molecules ~2.5x a tensor-core molecule of its largest size, the
                // FP64 block path ~2x): the long warp items no longer end the queue
                auto cost = [&](const int4& it) {
                    const int nr0 = roff[ord[it.x] + 1] - roff[ord[it.x]];   // largest of the item
                    if (it.z) return 1.9 * nr0;
                    return nr0 <= kTcMaxRed ? 0.75 * nr0 : 1.5 * nr0;
                };
                std::stable_sort(items.begin(), items.end(),
                                 [&](const int4& a, const int4& b) { return cost(a) > cost(b); });
                P.bitems.upload(items);
                P.refine.alloc(1);
                P.batch_smem = std::max<size_t>(P.batch_smem, (size_t)kTcSmemBytes);
            }
            CK(cudaFuncSetAttribute((const void*)k_eeq_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)P.batch_smem));
            int per_sm = 0, nsm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_eeq_batch, 512, P.batch_smem));
            CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P.opt.device));
            P.batch_grid = std::max(1, std::min(nm, per_sm * nsm));
        }
    }
    // ---- term lists (internal indices) ----
    {
        std::vector<int> i, j, k;
        std::vector<double> fc, th;
        for (int m = 0; m < nm; ++m)
            for (auto& a : mols[m]->angles) {
                i.push_back(P.ix(m, a.i)); j.push_back(P.ix(m, a.j)); k.push_back(P.ix(m, a.k));
                fc.push_back(a.fc); th.push_back(a.theta0);
            }
        P.na = (int)i.size();
        P.a_i.upload(i); P.a_j.upload(j); P.a_k.upload(k); P.a_fc.upload(fc); P.a_th.upload(th);
    }
    {
        std::vector<int> i, j, k, l;
        std::vector<double> V, nn, ph;
        for (int m = 0; m < nm; ++m)
            for (auto& t : mols[m]->torsions) {
                i.push_back(P.ix(m, t.i)); j.push_back(P.ix(m, t.j)); k.push_back(P.ix(m, t.k)); l.push_back(P.ix(m, t.l));
                V.push_back(t.V); nn.push_back(t.n); ph.push_back(t.phi0);
            }
        P.nt = (int)i.size();
        P.t_i.upload(i); P.t_j.upload(j); P.t_k.upload(k); P.t_l.upload(l); P.t_V.upload(V); P.t_n.upload(nn); P.t_p.upload(ph);
    }
    {
        std::vector<int> i, j, k, l;
        std::vector<double> e;
        for (int m = 0; m < nm; ++m)
            for (auto& t : mols[m]->storsions) {
                i.push_back(P.ix(m, t.i)); j.push_back(P.ix(m, t.j)); k.push_back(P.ix(m, t.k)); l.push_back(P.ix(m, t.l));
                e.push_back(t.erefhalf);
            }
        P.ns = (int)i.size();
        P.s_i.upload(i); P.s_j.upload(j); P.s_k.upload(k); P.s_l.upload(l); P.s_e.upload(e);
    }
    {
        std::vector<int> i, j, k, l, ty;
        std::vector<double> fc, om;
        for (int m = 0; m < nm; ++m)
            for (auto& t : mols[m]->inversions) {
                i.push_back(P.ix(m, t.i)); j.push_back(P.ix(m, t.j)); k.push_back(P.ix(m, t.k)); l.push_back(P.ix(m, t.l));
                ty.push_back(t.type); fc.push_back(t.fc); om.push_back(t.omega0);
            }
        P.ninv = (int)i.size();
        P.v_i.upload(i); P.v_j.upload(j); P.v_k.upload(k); P.v_l.upload(l); P.v_t.upload(ty); P.v_fc.upload(fc); P.v_om.upload(om);
    }
    {
        std::vector<int> i, j, k;
        std::vector<double> c9, r0ij, r0ik, r0jk, sc;
        for (int m = 0; m < nm; ++m) {
            const Model& M = *mols[m];
            auto r0 = [&](int a, int b) { return 0.58 * std::sqrt(3.0 * M.rcov_d3[a] * M.rcov_d3[b]) + 4.80; };
            for (auto& t : M.atm) {
                i.push_back(P.ix(m, t.i)); j.push_back(P.ix(m, t.j)); k.push_back(P.ix(m, t.k));
                c9.push_back(std::sqrt(std::fabs(t.c6ij * t.c6ik * t.c6jk)));
                r0ij.push_back(r0(t.i, t.j)); r0ik.push_back(r0(t.i, t.k)); r0jk.push_back(r0(t.j, t.k));
                sc.push_back(t.scale);
            }
        }
        P.natm = (int)i.size();
        P.at_i.upload(i); P.at_j.upload(j); P.at_k.upload(k); P.at_c9.upload(c9);
        P.at_r0ij.upload(r0ij); P.at_r0ik.upload(r0ik); P.at_r0jk.upload(r0jk); P.at_sc.upload(sc);
    }
    {
        std::vector<int> i, j, k;
        std::vector<double> c9;
        for (int m = 0; m < nm; ++m) {
            const Model& M = *mols[m];
            auto fq = [&](int a) { return std::min(std::max(1.0 - 3.0 * M.qa[a], -4.0), 4.0); };
            for (auto& t : M.batm) {
                i.push_back(P.ix(m, t.i)); j.push_back(P.ix(m, t.j)); k.push_back(P.ix(m, t.k));
                c9.push_back(fq(t.i) * fq(t.j) * fq(t.k) * t.zi * t.zj * t.zk);
            }
        }
        P.nbatm = (int)i.size();
        P.ba_i.upload(i); P.ba_j.upload(j); P.ba_k.upload(k); P.ba_c9.upload(c9);
    }
    {   // repulsion CSR, both directions
        std::vector<std::vector<std::tuple<int, double, double, unsigned char>>> rows(n);
        for (int m = 0; m < nm; ++m) {
            for (auto& r : mols[m]->rep_bonded) {
                const int a = P.ix(m, r.i), b = P.ix(m, r.j);
                rows[a].push_back({b, r.alpha, r.repab, 0});
                rows[b].push_back({a, r.alpha, r.repab, 0});
            }
            for (auto& r : mols[m]->rep_nonbonded) {
                const int a = P.ix(m, r.i), b = P.ix(m, r.j);
                rows[a].push_back({b, r.alpha, r.repab, 1});
                rows[b].push_back({a, r.alpha, r.repab, 1});
            }
        }
        std::vector<int> off{0}, jj;
        std::vector<double> al, ab;
        std::vector<unsigned char> kd;
        for (int a = 0; a < n; ++a) {
            for (auto& e : rows[a]) { jj.push_back(std::get<0>(e)); al.push_back(std::get<1>(e)); ab.push_back(std::get<2>(e)); kd.push_back(std::get<3>(e)); }
            off.push_back((int)jj.size());
        }
        P.r_off.upload(off); P.r_j.upload(jj); P.r_al.upload(al); P.r_ab.upload(ab); P.r_kind.upload(kd);
    }
    if (nm == 1) {
        upload_hbxb(*mols[0]);
    } else {   // bonds, HB and XB of every molecule (HB/XB lists stay those of the setup)
        for (const Model* M : mols)
            if (M->hb_on_device) throw std::runtime_error("upload: batches take host-detected HB lists");
        std::vector<int> bi, bj, bh, off{0}, hb;
        std::vector<double> fc, al, r0i, r0j, cki, ckj, sh, ff;
        HBHost hbt(n);
        std::vector<int> xa, xx, xb;
        std::vector<double> xpre, xrv;
        auto qs = [](double q, double st, double sf) { const double e = std::exp(st * q); return e / (e + sf); };
        for (int m = 0; m < nm; ++m) {
            const Model& M = *mols[m];
            auto X = [&](int t) { return P.ix(m, t); };
            std::map<int, std::vector<int>> byH;
            for (auto& e : M.bond_hb) byH[e.h].insert(byH[e.h].end(), e.b_atoms.begin(), e.b_atoms.end());
            for (auto& t : M.bonds) {
                bi.push_back(X(t.i)); bj.push_back(X(t.j));
                fc.push_back(t.fc); al.push_back(t.alpha); r0i.push_back(t.r0_base_i); r0j.push_back(t.r0_base_j);
                cki.push_back(t.cnfak_i); ckj.push_back(t.cnfak_j); sh.push_back(t.rabshift); ff.push_back(t.ff);
                const int H = t.nr_hb >= 1 ? t.hb_h : -1;
                bh.push_back(H >= 0 ? X(H) : -1);
                if (H >= 0) for (int x : byH[H]) hb.push_back(X(x));
                off.push_back((int)hb.size());
            }
            hbt.add(M, X);
            for (auto& t : M.xbonds) {
                xa.push_back(X(t.a)); xx.push_back(X(t.x)); xb.push_back(X(t.b));
                xpre.push_back(-qs(-t.q_b, 15.0, 0.03) * t.aci_x * qs(t.q_x, 15.0, 0.03));
                xrv.push_back(M.rvdw[t.a] + M.rvdw[t.b]);
            }
        }
        P.nb = (int)bi.size();
        P.b_i.upload(bi); P.b_j.upload(bj); P.b_h.upload(bh); P.b_off.upload(off); P.b_hb.upload(hb);
        P.b_fc.upload(fc); P.b_al.upload(al); P.b_r0i.upload(r0i); P.b_r0j.upload(r0j);
        P.b_cki.upload(cki); P.b_ckj.upload(ckj); P.b_sh.upload(sh); P.b_ff.upload(ff);
        P.upload_hb(hbt);
        P.nhb_near = P.nhb;   // batches: every HB term in FP64
        P.nxb = (int)xa.size();
        P.x_a.upload(xa); P.x_x.upload(xx); P.x_b.upload(xb); P.x_pre.upload(xpre); P.x_rv.upload(xrv);
    }
    // ---- per-step buffers ----
    P.cnraw.alloc(n); P.cn.alloc(n); P.dlog.alloc(n); P.w.alloc((size_t)n * 7); P.dw.alloc((size_t)n * 7);
    P.hg.alloc((size_t)n * K * 7); P.hdg.alloc((size_t)n * K * 7);
    P.etot.alloc(nm);
    {   // charge response only where a pair can exceed the 100 bohr Coulomb cut
        double ext = 0.0;
        if (nm == 1) {
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (const auto& p : p0) {
                const double c[3] = {p.x, p.y, p.z};
                for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], c[d]); hi[d] = std::max(hi[d], c[d]); }
            }
            for (int d = 0; d < 3; ++d) ext += (hi[d] - lo[d]) * (hi[d] - lo[d]);
        }
        P.resp_on = P.opt.exact_gradient && nm == 1 && P.nred > 0 && std::sqrt(ext) > 90.0;
        if (P.resp_on) {
            P.cfar.alloc(n); P.ures.alloc(n); P.bres.alloc(P.nred); P.xres.alloc(P.nred); P.info3.alloc(1);
        }
    }
    P.q.alloc(n); P.dEdcn.alloc(n); P.v.alloc(n); P.grad.alloc(3 * (size_t)n); P.E.alloc(16 * (size_t)nm);
    P.gout.alloc(3 * (size_t)n); P.qout.alloc(n); P.cnout.alloc(n);
    P.lda = (P.nred + 4) & ~3;   // >= nred + 1, a multiple of 4: 16-byte aligned FP32 and FP64 columns
    P.M.alloc((size_t)std::max<long long>(1, nm == 1 ? (long long)P.lda * P.nred : P.msize));
    P.bvec.alloc(std::max(1, P.nred)); P.xyz_stage.alloc(3 * (size_t)n); P.msd.alloc(2);
    P.info.alloc(nm); P.info2.alloc(1); P.status.alloc(nm); P.bad.alloc(nm);
    CK(cudaMemset(P.info.p, 0, nm * sizeof(int)));
    P.use_lu = false;
    if (nm == 1 && P.nred > 0) {
        int l1 = 0, l2 = 0;
        CS(cusolverDnDpotrf_bufferSize(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, P.M.p, P.lda, &l1));
        CS(cusolverDnDgetrf_bufferSize(P.sol, P.nred, P.nred, P.M.p, P.lda, &l2));
        P.lwork = std::max(l1, l2);
        P.work.alloc(std::max(1, P.lwork));
        P.ipiv.alloc(P.nred);
        int nsm = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P.opt.device));
        // in-house pivoted LU (indefinite matrices): one co-resident block per SM
        {
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_lu_factor, kLuThreads, 0));
            P.lu_grid = std::max(1, std::min(nsm, nsm * per_sm));
            P.lupart.alloc(2 * (size_t)P.lu_grid);
            P.lubar.alloc(2 * kBarGen);
            CK(cudaMemset(P.lubar.p, 0, 2 * kBarGen * sizeof(unsigned int)));
        }
        // persistent tiled Cholesky: task list, flags, co-resident grid
        {
            auto tasks = chol_tasks(P.nred);
            P.chol_nt = (P.nred + 1 + CB - 1) / CB;
            P.chol_ntasks = (int)tasks.size();
            P.ctasks.upload(tasks);
            P.cflags.alloc(2 + 2 * (size_t)P.chol_nt * P.chol_nt + P.chol_nt);
            P.rdiag.alloc(P.nred);
            P.ysol.alloc(P.nred);
            P.chol_smem = (2 * CB * CLD + CB) * sizeof(double);
            CK(cudaFuncSetAttribute((const void*)k_chol, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.chol_smem));
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_chol, kCholThreads, P.chol_smem));
            P.chol_grid = std::max(1, std::min(per_sm * nsm, P.chol_ntasks));
        }
        // block-Jacobi PCG: one block per fragment (blocks of <= 64 for larger ones).
        // GFNFF_PCG_BLOCK=g merges runs of consecutive fragments (neighbours in space:
        // fragments are Morton-ordered) into blocks of up to g unknowns; measured on water
        // clusters this leaves the iteration count unchanged, so it is off by default.
        P.pcg_ready = false;
        std::vector<int2> blocks;
        int blkmax = kPcgMaxBlock;
        {
            const Model& Mf0 = *mols[0];
            std::vector<int> fsz(std::max(1, Mf0.nfrag), 0);
            for (int a = 0; a < Mf0.n; ++a) ++fsz[Mf0.frag[a]];
            int big = 0;
            for (int c : fsz) big = std::max(big, c - 1);
            const char* ep = std::getenv("GFNFF_PCG_PRE");
            P.pcg_pre = big > kPcgWarpMax && !(ep && !std::strcmp(ep, "0"));
            if (P.pcg_pre) {
                blkmax = 128;
                if (const char* eb = std::getenv("GFNFF_PCG_PREBLK")) blkmax = std::max(2, std::min(512, std::atoi(eb)));
            }
        }
        {
            int group = 0;
            if (const char* e = std::getenv("GFNFF_PCG_BLOCK")) group = std::max(0, std::min(kPcgWarpMax, std::atoi(e)));
            std::vector<int> fr(n);
            const Model& M0 = *mols[0];
            for (int a = 0; a < n; ++a) fr[P.ix(0, a)] = M0.frag[a];
            int r = 0, i = 0, cur0 = 0, cur = 0;
            auto flush = [&]() {
                if (cur > 0) blocks.push_back(make_int2(cur0, cur));
                cur = 0;
            };
            while (i < n) {
                int j = i;
                while (j < n && fr[j] == fr[i]) ++j;
                const int nr = j - i - 1;   // the fragment's anchor is its first atom
                if (nr > group) {
                    flush();
                    // equal chunks of at most blkmax
                    const int nch = (nr + blkmax - 1) / blkmax, base = nr / nch, extra = nr % nch;
                    for (int c = 0, off = 0; c < nch; ++c) {
                        const int sz = base + (c < extra ? 1 : 0);
                        blocks.push_back(make_int2(r + off, sz));
                        off += sz;
                    }
                } else if (nr > 0) {
                    if (cur + nr > group) flush();
                    if (cur == 0) cur0 = r;
                    cur += nr;
                }
                r += nr;
                i = j;
            }
            flush();
            if (r != P.nred) blocks.clear();   // fragments not contiguous: no PCG
        }
        if (!blocks.empty() && P.pcg_pre) {
            // set-up-geometry inverses of every block (host Cholesky), row-major like the
            // device-computed ones
            auto A_el = [&](int a, int b) {
                if (a == b) return adg[a];
                const double dx = p0[a].x - p0[b].x, dy = p0[a].y - p0[b].y, dz = p0[a].z - p0[b].z;
                const double d2 = dx * dx + dy * dy + dz * dz, sa = alp[a] + alp[b];
                if (d2 >= 36.0 * sa) return 1.0 / std::sqrt(d2);
                const double rr = std::sqrt(d2);
                return std::erf(rr / std::sqrt(sa)) / rr;
            };
            std::vector<double> inv;
            for (auto& b : blocks) {
                const int sz = b.y;
                std::vector<double> Mb((size_t)sz * sz), Ib((size_t)sz * sz, 0.0);
                for (int i = 0; i < sz; ++i)
                    for (int j = 0; j < sz; ++j) {
                        const int k = P.h_r2a[b.x + i], ak = P.h_anchor[k];
                        const int l = P.h_r2a[b.x + j], al = P.h_anchor[l];
                        Mb[(size_t)i * sz + j] = A_el(k, l) - A_el(k, al) - A_el(ak, l) + A_el(ak, al);
                    }
                for (int i = 0; i < sz; ++i) Ib[(size_t)i * sz + i] = 1.0;
                if (!linalg::cholesky(Mb.data(), sz)) {
                    P.pcg_pre = false;   // not positive definite: inverses per launch instead
                    break;
                }
                linalg::cholesky_solve(Mb.data(), sz, Ib.data(), sz);
                inv.insert(inv.end(), Ib.begin(), Ib.end());
            }
            if (P.pcg_pre) P.pbinv.upload(inv);
            else blocks.clear();   // rebuilt below with device-sized blocks
        }
        if (blocks.empty() && !P.pcg_pre && blkmax != kPcgMaxBlock) {
            // the set-up inverses failed: fall back to per-fragment blocks of <= 64
            std::vector<int> fr(n);
            const Model& M0 = *mols[0];
            for (int a = 0; a < n; ++a) fr[P.ix(0, a)] = M0.frag[a];
            int r = 0, i = 0;
            while (i < n) {
                int j = i;
                while (j < n && fr[j] == fr[i]) ++j;
                const int nr = j - i - 1;
                for (int c = 0; c < nr; c += kPcgMaxBlock)
                    blocks.push_back(make_int2(r + c, std::min(kPcgMaxBlock, nr - c)));
                r += nr;
                i = j;
            }
            if (r != P.nred) blocks.clear();
        }
        if (!blocks.empty()) {
            // rows per grid block: whole preconditioner blocks, about nred / nsm rows each
            std::vector<int4> part;
            std::vector<long long> boff;
            long long bo = 0;
            for (auto& b : blocks) { boff.push_back(bo); bo += (long long)b.y * b.y; }
            // the lower-triangle form from 4096 unknowns (the matrix leaves L2), and for chains
            // with set-up block inverses from 1024: its tiled product balances work by tiles, so
            // every SM takes part even where large preconditioner blocks, owned whole, would
            // load a few blocks with most rows (Gly50 + 1500 waters: 1.45 -> 0.69 ms)
            const char* esym = std::getenv("GFNFF_PCG_SYM");
            const bool lower = esym ? std::strcmp(esym, "0") != 0
                                    : (P.nred >= 4096 || (P.pcg_pre && P.nred >= 1024));
            const int G = lower ? nsm : std::max(1, std::min(nsm, (int)blocks.size()));
            size_t bk = 0;
            int maxrows = 1;
            long long maxinv = 1;
            for (int g = 0; g < G; ++g) {
                const int target = (int)(((long long)P.nred * (g + 1)) / G);
                const int b0 = (int)bk, r0 = bk < blocks.size() ? blocks[bk].x : P.nred;
                while (bk < blocks.size() && (blocks[bk].x + blocks[bk].y <= target || g == G - 1)) ++bk;
                const int r1 = bk < blocks.size() ? blocks[bk].x : P.nred;
                part.push_back(make_int4(r0, r1, b0, (int)bk));
                maxrows = std::max(maxrows, r1 - r0);
                maxinv = std::max(maxinv, (bk < blocks.size() ? boff[bk] : bo) - (b0 < (int)blocks.size() ? boff[b0] : bo));
            }
            // p (n), Gauss-Jordan scratch, x/r/z/Mp of the owned rows, owned block inverses
            if (P.pcg_pre) maxinv = 0;      // inverses applied from global memory
            maxinv = (maxinv + 1) & ~1ll;   // keeps the int4 row records behind it 16-byte aligned
            const size_t smem =
                ((size_t)((P.nred + 1) & ~1) + kPcgMaxBlock * (kPcgMaxBlock + 1) + 4 * (size_t)maxrows + maxinv) *
                    sizeof(double) +
                (size_t)maxrows * sizeof(int4);
            if (smem <= 220 * 1024) {
                std::vector<int> rblk(P.nred);
                for (size_t q = 0; q < blocks.size(); ++q)
                    for (int r = 0; r < blocks[q].y; ++r) rblk[blocks[q].x + r] = (int)q;
                P.pblocks.upload(blocks); P.pboff.upload(boff); P.ppart.upload(part); P.prblk.upload(rblk);
                P.px.alloc(P.nred); P.pz.alloc(P.nred);
                P.pcg_maxrows = maxrows;
                P.pcg_maxinv = (int)maxinv;
                {
                    P.pcg_lower = lower;
                    const char* ef = std::getenv("GFNFF_PCG_F32");
                    P.pcg_f32 = P.pcg_lower && P.opt.precision == 1 && ef && !std::strcmp(ef, "1");
                    // mixed form, lower-triangle systems: FP32-matrix CG inside FP64 refinement
                    // (k_pcg_ir; GFNFF_PCG_IR=0: the FP64 classic PCG at the absolute bar)
                    const char* eir = std::getenv("GFNFF_PCG_IR");
                    P.pcg_ir = P.pcg_lower && P.opt.precision == 1 && !P.pcg_f32 && !(eir && !std::strcmp(eir, "0"));
                    if (P.pcg_f32 || P.pcg_ir) P.Mf.alloc((size_t)P.lda * P.nred);
                    if (P.pcg_ir) {
                        const size_t n4 = (size_t)((P.nred + 3) & ~3);
                        P.p32.alloc(2 * n4);
                        CK(cudaMemset(P.p32.p, 0, 2 * n4 * sizeof(float)));   // the tails past n stay 0
                        P.pcg_tmap = tmap_f32_tiles(P.Mf.p, P.nred, P.lda);
                    }
                    const char* ec = std::getenv("GFNFF_PCG_COLS");
                    P.pcg_cols = (ec && !std::strcmp(ec, "8")) ? 2 : 1;
                    std::vector<int2> tl;
                    for (int i0 = 0; i0 < P.nred; i0 += kPcgT)
                        for (int j0 = 0; j0 <= i0; j0 += kPcgT) tl.push_back(make_int2(i0, j0));
                    P.ptiles.upload(tl);
                    P.pcg_ntiles = (int)tl.size();
                    P.pyA.alloc(P.nred);
                    CK(cudaMemset(P.pyA.p, 0, (size_t)P.nred * sizeof(double)));
                }
                P.ppartial.alloc(8 * (size_t)G); P.pbar.alloc(2 * kBarGen); P.piters.alloc(2); P.pwarm.alloc(2);
                P.pz2.alloc(P.nred);
                CK(cudaMemset(P.pwarm.p, 0, 2 * sizeof(int)));
                CK(cudaMemset(P.pbar.p, 0, 2 * kBarGen * sizeof(unsigned int)));
                CK(cudaMemset(P.piters.p, 0, 2 * sizeof(int)));
                P.pcg_grid = G;
                P.pcg_smem = smem;
                CK(cudaFuncSetAttribute((const void*)k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                int per_sm = 0;
                CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_pcg, kPcgThreads, smem));
                P.pcg_ready = per_sm >= 1;
                if (P.pcg_ir) {   // one more owned-row vector (the inner correction d), even-sized
                    // and the region of the replicated vector is the larger of the FP64 vector
                    // and the FP32 direction with two staging halves of a tile
                    P.pcg_smem_ir = smem + (size_t)((maxrows + 1) & ~1) * sizeof(double) +
                                    (size_t)(pcg_ir_pregion(P.nred) - ((P.nred + 1) & ~1)) * sizeof(double);
                    int ps = 0;
                    const void* kir = (const void*)k_pcg_ir;
                    if (P.pcg_smem_ir <= 220 * 1024) {
                        CK(cudaFuncSetAttribute(kir, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.pcg_smem_ir));
                        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, kir, kPcgThreads, P.pcg_smem_ir));
                    }
                    P.pcg_ir = ps >= 1;
                }
                // the pipelined form keeps ten owned-row vectors instead of four
                P.pcg_smem_pipe = smem + 6 * (size_t)maxrows * sizeof(double);
                const char* pe = std::getenv("GFNFF_PCG");
                // default: pipelined for L2-resident matrices (latency-bound); the tiled product
                // of large ones measured faster in the classic form
                P.pcg_pipe = pe ? std::strcmp(pe, "classic") != 0 : !P.pcg_lower;
                P.pcg_pipe = P.pcg_pipe && P.pcg_smem_pipe <= 220 * 1024;
                {
                    const char* er = std::getenv("GFNFF_PCG_RES");
                    const int nt64 = (P.nred + 63) / 64;
                    std::vector<int2> rt;
                    for (int i0 = 0; i0 < nt64; ++i0)
                        for (int j0 = 0; j0 <= i0; ++j0) rt.push_back(make_int2(64 * i0, 64 * j0));
                    int bigblk = 0;
                    for (auto& b : blocks) bigblk = std::max(bigblk, b.y);
                    P.pcg_res_ntiles = (int)rt.size();
                    P.pcg_res_ntl = (P.pcg_res_ntiles + G - 1) / G;
                    P.pcg_res_gscratch = bigblk > kPcgWarpMax ? 1 : 0;
                    P.pcg_smem_res = ((size_t)((P.nred + 1) & ~1) + (size_t)P.pcg_res_ntl * 64 * 65 +
                                      (P.pcg_res_gscratch ? (size_t)kPcgMaxBlock * (kPcgMaxBlock + 1) : 0) +
                                      10 * (size_t)maxrows + maxinv) * sizeof(double) +
                                     (size_t)maxrows * sizeof(int4);
                    P.pcg_res = er && !std::strcmp(er, "1") && P.pcg_pipe && !P.pcg_lower &&
                                P.pcg_res_ntl <= 5 && P.pcg_smem_res <= 200 * 1024;
                    if (P.pcg_res) {
                        P.prtiles.upload(rt);
                        CK(cudaFuncSetAttribute((const void*)k_pcg_res, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)P.pcg_smem_res));
                        int rs = 0;
                        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rs, (const void*)k_pcg_res, kPcgPipeThreads,
                                                                         P.pcg_smem_res));
                        P.pcg_res = rs >= 1;
                    }
                }
                if (P.pcg_pipe) {
                    CK(cudaFuncSetAttribute((const void*)k_pcg_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)P.pcg_smem_pipe));
                    int ps = 0;
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, (const void*)k_pcg_pipe, kPcgPipeThreads,
                                                                     P.pcg_smem_pipe));
                    P.pcg_pipe = ps >= 1;
                }
            }
        }
    }
    CK(cudaDeviceSynchronize());
    // The reduced EEQ matrix is indefinite for some systems (hydrogen has a negative
    // hardness); curcuma then falls back from its Cholesky to an LU solve
    // (eeq_solver.cpp:1448-2086).  Probe once at the setup geometry and keep the
    // choice for this molecule; the host entry point switches later if a geometry
    // turns it.
    P.upload_alpb(solv ? *solv : AlpbModel());
    if (P.alpb_on) P.pcg_res = false;   // its in-kernel matrix build has no Born term
    const bool graphs_setting = P.graphs_ok;
    P.graphs_ok = false;   // probes below run direct (their buffers are temporary)
    P.pcg_warm = false;    // and PCG probes start from zero
    if (nm == 1 && P.nred > 0) {
        DBuf<double> x;
        std::vector<double> h(mols[0]->xyz_setup);
        x.upload(h);
        // the probe factors with the in-house tiled Cholesky (k_chol: NOT_SPD on a pivot <= 0)
        P.solver = Impl::SOLVE_TILED;
        enqueue(x.p, true);
        int st = 0;
        fetch(nullptr, nullptr, &st, nullptr);
        if (st == GFNFF_NOT_SPD) P.use_lu = true;
        // Solver: GFNFF_EEQ_SOLVER=library|tiled|pcg|batched forces one; otherwise the fastest
        // of the in-house ones (tiled, pcg, batched) over three evaluations at the setup
        // geometry.  cuSOLVER ("library") is an explicit opt-in only.
        if (!P.use_lu) {
            const char* env = std::getenv("GFNFF_EEQ_SOLVER");
            std::vector<int> cand;
            if (env && !std::strcmp(env, "library")) cand = {Impl::SOLVE_LIBRARY};
            else if (env && !std::strcmp(env, "tiled")) cand = {Impl::SOLVE_TILED};
            else if (env && !std::strcmp(env, "pcg") && P.pcg_ready) cand = {Impl::SOLVE_PCG};
            else if (env && !std::strcmp(env, "batched") && P.batch_ready && !P.resp_on && !P.alpb_on)
                cand = {Impl::SOLVE_BATCH};
            else {
                cand = {Impl::SOLVE_TILED};
                if (P.pcg_ready) cand.push_back(Impl::SOLVE_PCG);
                // the batched kernel keeps no factor for the charge-response solve
                // (nor the solvent's Born matrix: it builds its matrix from the atoms)
                if (P.batch_ready && !P.resp_on && !P.alpb_on) cand.push_back(Impl::SOLVE_BATCH);
            }
            if (cand.size() == 1) {
                P.solver = cand[0];
            } else {
                cudaEvent_t e0, e1;
                CK(cudaEventCreate(&e0));
                CK(cudaEventCreate(&e1));
                float best = 1e30f;
                int pick = Impl::SOLVE_TILED;
                for (int c : cand) {
                    P.solver = c;
                    if (c == Impl::SOLVE_PCG) P.pcg_max_iter = 200;
                    enqueue(x.p, true);
                    fetch(nullptr, nullptr, &st, nullptr);
                    if (st != GFNFF_OK) continue;
                    if (c == Impl::SOLVE_PCG) {
                        int it = 0;
                        CK(cudaMemcpy(&it, P.piters.p, sizeof(int), cudaMemcpyDeviceToHost));
                        P.pcg_max_iter = std::min(500, 4 * it + 20);
                    }
                    CK(cudaEventRecord(e0, P.stream));
                    for (int rep = 0; rep < 3; ++rep) enqueue(x.p, true);
                    CK(cudaEventRecord(e1, P.stream));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    fetch(nullptr, nullptr, &st, nullptr);
                    if (st == GFNFF_OK && ms < best) { best = ms; pick = c; }
                }
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                P.solver = pick;
            }
        }
    }
    tune_pairs(mols);
    P.graphs_ok = graphs_setting;
    // from here on PCG starts from the previous step's solution (GFNFF_PCG_WARM=0: from zero)
    const char* warm_env = std::getenv("GFNFF_PCG_WARM");
    P.pcg_warm = !(warm_env && !std::strcmp(warm_env, "0"));
}

// Tile-shape autotuner of the Coulomb + D4 pair kernel.  Candidates: k_pairs_sym with 32- or
// 64-atom tiles (a block is one warp or two; the tile edge is the atom block width and the
// partners a warp takes per step), the 64-atom tiles also at 10 blocks per SM (96 registers)
// instead of 8, and both directions by rows (k_pairs).  After one evaluation at the set-up
// geometry (valid charges and weights in the buffers), each candidate runs once untimed and
// three times between CUDA events on the handle's stream (both terms, PART = both); the
// fastest is kept.  The pick is cached per (device, batch or single molecule, size bucket
// floor(log2 N)) for the process, so further handles of similar systems skip the timing.
// GFNFF_PAIRS_TUNE=0, GFNFF_PAIRS=rows and GFNFF_PAIRS_OCC=1 keep the untuned choice;
// GFNFF_PAIRS_VARIANT=sym32|sym64|sym64_occ10|rows forces one.
void Engine::tune_pairs(const std::vector<const Model*>& mols)
{
    Impl& P = *p_;
    const char* et = std::getenv("GFNFF_PAIRS_TUNE");
    const char* pe = std::getenv("GFNFF_PAIRS");
    const char* po = std::getenv("GFNFF_PAIRS_OCC");
    if (const char* ev = std::getenv("GFNFF_PAIRS_VARIANT")) {   // forced: sym32|sym64|sym64_occ10|rows
        const char* names[4] = {"sym32", "sym64", "sym64_occ10", "rows"};
        for (int v = 0; v < 4; ++v)
            if (!std::strcmp(ev, names[v])) {
                P.pair_variant = v;
                P.pairs_sym = v != Impl::PAIRS_ROWS;
            }
        return;
    }
    if ((et && !std::strcmp(et, "0")) || pe || po || P.n < 2) return;
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, int> cache;
    int bucket = 0;
    while ((2 << bucket) <= P.n) ++bucket;
    const auto key = std::make_tuple(P.opt.device, P.nmol > 1 ? 1 : 0, bucket);
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) {
            P.pair_variant = it->second;
            P.pairs_sym = P.pair_variant != Impl::PAIRS_ROWS;
            return;
        }
    }
    std::vector<double> h;
    for (const Model* m : mols) h.insert(h.end(), m->xyz_setup.begin(), m->xyz_setup.end());
    DBuf<double> x;
    x.upload(h);
    enqueue(x.p, true);
    View V = P.view();
    const dim3 tgrid(nblk(P.n, kTile), P.nsplit);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int pick = P.pair_variant;
    for (int v = 0; v < 4; ++v) {
        auto run = [&]() {
            if (v == Impl::PAIRS_ROWS) k_pairs<double><<<tgrid, kTile, 0, P.stream>>>(V, P.nsplit);
            else P.launch_pairs_sym<kPairBoth>(v, V, P.stream);
        };
        run();
        CK(cudaEventRecord(e0, P.stream));
        for (int r = 0; r < 3; ++r) run();
        CK(cudaEventRecord(e1, P.stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        P.pair_ms[v] = ms / 3.f;
        if (ms < best) {
            best = ms;
            pick = v;
        }
    }
    CK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P.pair_variant = pick;
    P.pairs_sym = pick != Impl::PAIRS_ROWS;
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = pick;
}

const char* Engine::pair_kernel_name() const
{
    switch (p_->pair_variant) {
    case Impl::PAIRS_SYM32: return "sym32";
    case Impl::PAIRS_SYM64_OCC: return "sym64_occ10";
    case Impl::PAIRS_ROWS: return "rows";
    default: return "sym64";
    }
}

bool Engine::switch_to_lu()
{
    if (p_->use_lu || p_->nred == 0 || p_->nmol != 1) return false;
    p_->drop_graphs();
    p_->use_lu = true;
    return true;
}

bool Engine::switch_to_direct()
{
    if (p_->nmol != 1) return false;
    if (p_->solver != Impl::SOLVE_PCG && !(p_->solver == Impl::SOLVE_BATCH && p_->batch_tc)) return false;
    p_->drop_graphs();
    p_->solver = Impl::SOLVE_TILED;   // the in-house FP64 Cholesky
    return true;
}

const char* Engine::solver_name() const
{
    if (p_->nmol != 1) return "batched";
    if (p_->use_lu) return "lu";
    switch (p_->solver) {
    case Impl::SOLVE_PCG: return "pcg";
    case Impl::SOLVE_TILED: return "tiled";
    case Impl::SOLVE_BATCH: return "batched";
    default: return "library";
    }
}

int Engine::eeq_fp64_products()
{
    if (p_->nmol != 1 || p_->use_lu || p_->solver != Impl::SOLVE_PCG || !p_->pcg_ir) return -1;
    int v[2] = {0, 0};
    CK(cudaStreamSynchronize(p_->stream));
    CK(cudaMemcpy(v, p_->piters.p, sizeof(v), cudaMemcpyDeviceToHost));
    return v[1];
}

int Engine::eeq_iterations()
{
    const bool batched = p_->nmol != 1 || (!p_->use_lu && p_->solver == Impl::SOLVE_BATCH);
    if (batched && p_->batch_tc) {   // refinement corrections of the tensor-core path
        int it = 0;
        CK(cudaStreamSynchronize(p_->stream));
        CK(cudaMemcpy(&it, p_->refine.p, sizeof(int), cudaMemcpyDeviceToHost));
        return it;
    }
    if (p_->nmol != 1 || p_->use_lu || p_->solver != Impl::SOLVE_PCG) return 0;
    int it = 0;
    CK(cudaStreamSynchronize(p_->stream));
    CK(cudaMemcpy(&it, p_->piters.p, sizeof(int), cudaMemcpyDeviceToHost));
    return it;
}

// One evaluation is ~20 kernels and memsets; replaying them as a CUDA graph removes the
// per-launch host overhead.  A graph is captured per (coordinate buffer, energy buffer,
// unit) combination and replayed while the model and the solver choice stay the same;
// phase timing (events between phases) and GFNFF_GRAPHS=0 use direct launches, and a
// capture that fails falls back to them for good.
// kernel nodes of a captured graph whose host stub lies in this shared object (library
// kernels, e.g. cuSOLVER's, are not counted)
static void own_marker() {}
static int own_kernel_nodes(cudaGraph_t g)
{
    Dl_info self{};
    if (!dladdr((void*)&own_marker, &self) || !self.dli_fname) return -1;
    size_t nn = 0;
    if (cudaGraphGetNodes(g, nullptr, &nn) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn && cudaGraphGetNodes(g, nodes.data(), &nn) != cudaSuccess) return -1;
    int k = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp{};
        // nodes of kernels from another runtime instance (cuSOLVER links its own) are not
        // known to this one: the query fails for them, and its error must not stay pending
        if (cudaGraphKernelNodeGetParams(nd, &kp) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        Dl_info di{};
        if (dladdr(kp.func, &di) && di.dli_fname && !std::strcmp(di.dli_fname, self.dli_fname)) ++k;
    }
    cudaGetLastError();
    return k;
}

int Engine::kernels_per_evaluation() const
{
    // the positions kernel is launched before the replayed graph
    return p_->graph && p_->graph_kernels >= 0 ? p_->graph_kernels + 1 : -1;
}

void Engine::enqueue(const double* d_xyz, bool bohr, double* d_energies)
{
    Impl& P = *p_;
    launch_positions(d_xyz, bohr);
    if (P.timing || !P.graphs_ok) {   // phase events cannot be timed inside a graph
        launch_body();
    } else {
        if (!P.graph) {
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(P.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                try {
                    launch_body();
                } catch (const std::exception&) {
                    ok = false;
                }
                const cudaError_t e = cudaStreamEndCapture(P.stream, &graph);
                ok = ok && e == cudaSuccess && graph;
                if (ok) P.graph_kernels = own_kernel_nodes(graph);
                if (ok) ok = cudaGraphInstantiate(&P.graph, graph, 0) == cudaSuccess;
                if (graph) cudaGraphDestroy(graph);
            }
            if (!ok) {
                cudaGetLastError();   // clear the capture error, stay with direct launches
                P.graph = nullptr;
                P.graphs_ok = false;
            }
        }
        if (P.graph) CK(cudaGraphLaunch(P.graph, P.stream));
        else launch_body();
    }
    if (d_energies)
        CK(cudaMemcpyAsync(d_energies, P.etot.p, (size_t)P.nmol * sizeof(double), cudaMemcpyDeviceToDevice, P.stream));
    P.mark(12);
    CK(cudaGetLastError());
}

// geometry in: caller order -> internal order, the HB refresh metric (direct launches;
// the only part of an evaluation that touches the caller's coordinate buffer)
void Engine::launch_positions(const double* d_xyz, bool bohr)
{
    Impl& P = *p_;
    P.mark(0);
    CK(cudaMemsetAsync(P.msd.p, 0, 2 * sizeof(double), P.stream));
    k_positions<<<nblk(P.n), kBlock, 0, P.stream>>>(P.n, P.perm.p, d_xyz, bohr ? 1.0 : kAngToBohr, P.pos.p,
                                                   P.hbref.p, P.msd.p, P.cnl_on ? P.cnl_ref.p : nullptr,
                                                   0.25 * Impl::kCnSkin * Impl::kCnSkin, P.cnl_bad.p, P.toporef.p);
}

// everything after the positions, reading and writing engine buffers only, so that it
// can be captured once as a graph; molecule totals go to etot
void Engine::launch_body()
{
    Impl& P = *p_;
    cudaStream_t s = P.stream;
    const int n = P.n;
    View V = P.view();
    const dim3 tgrid(nblk(n, kTile), P.nsplit);
    // mixed form: FP32 arithmetic in the CN erf counting and the weak hydrogen bonds; FP64
    // everywhere else (per-pair float<->double conversions cost more than FP32 saves in
    // the pair and CN-chain kernels) and in every accumulation
    const bool mixed = P.opt.precision == 1;
    CK(cudaMemsetAsync(P.grad.p, 0, 3 * (size_t)n * sizeof(double), s));
    CK(cudaMemsetAsync(P.dEdcn.p, 0, (size_t)n * sizeof(double), s));
    CK(cudaMemsetAsync(P.cnraw.p, 0, (size_t)n * sizeof(double), s));
    CK(cudaMemsetAsync(P.E.p, 0, 16 * (size_t)P.nmol * sizeof(double), s));
    CK(cudaMemsetAsync(P.bad.p, 0, (size_t)P.nmol * sizeof(int), s));
    if (P.resp_on) CK(cudaMemsetAsync(P.cfar.p, 0, (size_t)n * sizeof(double), s));
    // terms without a charge dependence: on the side stream when forking, else in phase order
    const bool fork = P.side && !P.timing;
    cudaStream_t s2 = fork ? P.side : s;
    auto hb_rep_terms = [&]() {
    if (P.nhb) {
        HBSoA H{P.nhb, P.h_rec.p, P.h_qh.p, P.h_qa.p, P.h_bas.p, P.h_aci.p, P.h_rvdw.p, P.h_zlp.p,
                P.h_pc.p, P.h_nfl.p, P.h_adjo.p, P.h_adj.p};
        const int split = mixed ? P.nhb_near : P.nhb;
        if (V.cell.on) {
            if (split > 0) k_hbonds<double, true><<<nblk(split), kBlock, 0, s2>>>(V, H, 0, split);
            if (P.nhb > split) k_hbonds<float, true><<<nblk(P.nhb - split), kBlock, 0, s2>>>(V, H, split, P.nhb);
        } else {
            if (split > 0) k_hbonds<double><<<nblk(split), kBlock, 0, s2>>>(V, H, 0, split);
            if (P.nhb > split) k_hbonds<float><<<nblk(P.nhb - split), kBlock, 0, s2>>>(V, H, split, P.nhb);
        }
    }
    if (P.nxb) k_xbonds<<<nblk(P.nxb), kBlock, 0, s2>>>(V, XBSoA{P.nxb, P.x_a.p, P.x_x.p, P.x_b.p, P.x_pre.p, P.x_rv.p});
    P.mark(8);
    k_repulsion<double><<<nblk((long)n * 32), kBlock, 0, s2>>>(V, P.r_off.p, P.r_j.p, P.r_al.p, P.r_ab.p, P.r_kind.p);
    P.mark(9);
    };
    auto bonded_terms = [&]() {
    if (P.nb) {
        BondSoA B{P.nb, P.b_i.p, P.b_j.p, P.b_h.p, P.b_off.p, P.b_hb.p, P.b_fc.p, P.b_al.p,
                  P.b_r0i.p, P.b_r0j.p, P.b_cki.p, P.b_ckj.p, P.b_sh.p, P.b_ff.p};
        k_bonds<<<nblk((long)P.nb * 32), kBlock, 0, s2>>>(V, B);
    }
    if (P.na) k_angles<<<nblk(P.na), kBlock, 0, s2>>>(V, AngleSoA{P.na, P.a_i.p, P.a_j.p, P.a_k.p, P.a_fc.p, P.a_th.p});
    if (P.nt) k_torsions<<<nblk(P.nt), kBlock, 0, s2>>>(V, TorsSoA{P.nt, P.t_i.p, P.t_j.p, P.t_k.p, P.t_l.p, P.t_V.p, P.t_n.p, P.t_p.p}, 0);
    if (P.ns) k_torsions<<<nblk(P.ns), kBlock, 0, s2>>>(V, TorsSoA{P.ns, P.s_i.p, P.s_j.p, P.s_k.p, P.s_l.p, P.s_e.p, nullptr, nullptr}, 1);
    if (P.ninv) k_inversions<<<nblk(P.ninv), kBlock, 0, s2>>>(V, InvSoA{P.ninv, P.v_i.p, P.v_j.p, P.v_k.p, P.v_l.p, P.v_t.p, P.v_fc.p, P.v_om.p});
    if (P.natm) k_atm<<<nblk(P.natm), kBlock, 0, s2>>>(V, TripSoA{P.natm, P.at_i.p, P.at_j.p, P.at_k.p, P.at_c9.p, P.at_r0ij.p, P.at_r0ik.p, P.at_r0jk.p, P.at_sc.p});
    if (P.nbatm) k_batm<<<nblk(P.nbatm), kBlock, 0, s2>>>(V, TripSoA{P.nbatm, P.ba_i.p, P.ba_j.p, P.ba_k.p, P.ba_c9.p, nullptr, nullptr, nullptr, nullptr});
    };
    // The side terms fork right before the EEQ solve and are issued after the solver's
    // launch: the latency-bound cooperative PCG takes its SM slots first and the side
    // kernels fill what it leaves (k_pcg_pipe uses half of an SM's registers); the batched
    // EEQ kernel's blocks leave their SMs one by one when the work queue runs dry, while the
    // largest molecules still factor, and the side kernels take those SMs.
    // (GFNFF_SIDE_EARLY=1: fork at the start of the evaluation instead.)
    // Coulomb + D4 pairs by tile pairs (each pair once); PART selects the terms
    auto pairs_sym = [&](auto part, cudaStream_t st) {
        constexpr int PT = decltype(part)::value;
        P.template launch_pairs_sym<PT>(P.pair_variant, V, st);
    };
    // split unless the solver is the classic PCG, whose cooperative grid fills every SM:
    // then nothing runs beside it, and the split pass costs more than it hides
    const bool full_sm_solver = P.nmol == 1 && !P.use_lu && P.solver == Impl::SOLVE_PCG && !P.pcg_pipe;
    const bool split = fork && P.pairs_sym && P.pairs_split > 0 && (P.pairs_split == 2 || !full_sm_solver);
    // own stream for batches and direct solvers (512 conformers: 0.98 -> 0.93 ms); beside
    // the pipelined PCG it slows the solver's barriers, so there it queues on the side stream
    // (1000 waters: 0.469 ms there, 0.524 ms on its own stream)
    const bool pcg_single = P.nmol == 1 && !P.use_lu && P.solver == Impl::SOLVE_PCG;
    cudaStream_t sd = split && P.side_d4 && !pcg_single ? P.side_d4 : s2;
    auto d4_pairs = [&]() {   // after ev_fork1 (the CN weights exist)
        if (!split) return;
        if (sd != s2) CK(cudaStreamWaitEvent(sd, P.ev_fork1, 0));
        pairs_sym(std::integral_constant<int, kPairD4>{}, sd);
        if (sd != s2) CK(cudaEventRecord(P.ev_join_d4, sd));
    };
    const bool early = fork && P.side_early;
    if (early) {
        CK(cudaEventRecord(P.ev_fork0, s));
        CK(cudaStreamWaitEvent(s2, P.ev_fork0, 0));
        hb_rep_terms();
    }
    auto side_after = [&]() {
        if (!fork || early) return;
        CK(cudaStreamWaitEvent(s2, P.ev_fork1, 0));
        d4_pairs();
        hb_rep_terms();
        bonded_terms();
        CK(cudaEventRecord(P.ev_join, s2));
    };
    P.mark(1);
    if (P.box_cull) k_boxes<<<nblk(n, kTile), kTile, 0, s>>>(n, P.pos.p, P.boxlo.p, P.boxhi.p);
    if (P.cnl_on) {
        (mixed ? k_cn_nl<float> : k_cn_nl<double>)<<<nblk((long)n * 32), kBlock, 0, s>>>(V, P.cnl_off.p, P.cnl_j.p,
                                                                                         P.cnl_bad.p);
        (mixed ? k_cn<float> : k_cn<double>)<<<tgrid, kTile, 0, s>>>(V, P.nsplit, P.cnl_bad.p);
    } else {
        (mixed ? k_cn<float> : k_cn<double>)<<<tgrid, kTile, 0, s>>>(V, P.nsplit, nullptr);
    }
    P.mark(2);
    k_d4_weights<<<nblk(n), kBlock, 0, s>>>(V);
    if (early) {
        CK(cudaEventRecord(P.ev_fork1, s));
        CK(cudaStreamWaitEvent(s2, P.ev_fork1, 0));
        d4_pairs();
        bonded_terms();
        CK(cudaEventRecord(P.ev_join, s2));
    }
    if (P.alpb_on) P.alpb_pre(s);   // Born radii, surfaces, shape: the Born matrix of the EEQ
    // EEQ
    P.mark(3);
    if (P.nmol == 1 && !(P.solver == Impl::SOLVE_BATCH && !P.use_lu)) {
        const int sv = P.use_lu ? -1 : P.solver;
        const bool full = sv == -1 || (sv == Impl::SOLVE_PCG && !P.pcg_lower);
        const bool aug = sv == Impl::SOLVE_TILED;
        if (P.nred > 0) {
            const long long nt = (P.nred + kMT - 1) / kMT;
            const unsigned nb = (unsigned)(nt * (nt + 1) / 2);
            if (sv == Impl::SOLVE_PCG && P.pcg_res)
                ;   // the resident PCG builds its tiles itself
            else if (sv == Impl::SOLVE_PCG && P.pcg_f32)
                (P.alpb_on ? k_eeq_M_tiles<float, true> : k_eeq_M_tiles<float, false>)<<<nb, 256, 0, s>>>(
                    V, P.red2atom.p, P.anchor.p, P.Mf.p, P.lda, 0, nullptr);
            else
                (P.alpb_on ? k_eeq_M_tiles<double, true> : k_eeq_M_tiles<double, false>)<<<nb, 256, 0, s>>>(
                    V, P.red2atom.p, P.anchor.p, P.M.p, P.lda, full ? 1 : 0,
                    sv == Impl::SOLVE_PCG && P.pcg_ir ? P.Mf.p : nullptr);
        }
        P.mark(4);
        if (P.nred > 0)
            k_eeq_rhs<<<nblk(P.nred), kBlock, 0, s>>>(V, P.red2atom.p, P.anchor.p, P.qlist.p, P.nq, P.q0.p, P.bvec.p,
                                                      aug ? P.M.p + P.nred : nullptr, P.lda);
        P.mark(5);
        if (fork && !early) CK(cudaEventRecord(P.ev_fork1, s));
        if (P.nred > 0) {
            if (sv == Impl::SOLVE_TILED) {
                P.chol_launch();
            } else if (sv == Impl::SOLVE_PCG) {
                P.pcg_launch(P.bvec.p, P.px.p, P.info.p, 0);
            } else if (sv == Impl::SOLVE_LIBRARY) {
                CS(cusolverDnDpotrf(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, P.M.p, P.lda, P.work.p, P.lwork, P.info.p));
                CS(cusolverDnDpotrs(P.sol, CUBLAS_FILL_MODE_LOWER, P.nred, 1, P.M.p, P.lda, P.bvec.p, P.nred, P.info2.p));
            } else {   // indefinite: in-house pivoted LU, b eliminated along, then U x = y
                CK(cudaMemsetAsync(P.lubar.p, 0, sizeof(unsigned int), s));
                LUArgs L{P.M.p, P.lda, P.nred, P.bvec.p, P.ipiv.p, P.info.p, P.lupart.p, P.lubar.p};
                void* args[] = {&L};
                CK(cudaLaunchCooperativeKernel((const void*)k_lu_factor, dim3(P.lu_grid), dim3(kLuThreads), args, 0, s));
                k_lu_back<<<1, 1024, 0, s>>>(P.M.p, P.lda, P.nred, P.bvec.p, P.info.p);
            }
        }
        side_after();
    } else {
        P.mark(4);
        P.mark(5);
        CK(cudaMemsetAsync(P.bnext.p, 0, sizeof(int), s));
        if (fork && !early) CK(cudaEventRecord(P.ev_fork1, s));   // single molecule, batched solver
        EEQBatch B{P.roff.p, P.moff.p, P.border.p, P.bitems.p, P.nbitems, P.bnext.p, P.batch_smem_max, P.red2atom.p,
                   P.anchor.p, P.qlist.p, P.nq, P.q0.p, P.M.p, P.bvec.p, P.info.p,
                   P.batch_tc ? 1 : 0, P.M64.p, P.m64off.p, kRefineTol, P.refine.p};
        if (P.batch_tc) {
            CK(cudaMemsetAsync(P.refine.p, 0, sizeof(int), s));
            if (P.n_tc_tiles) k_eeq_tc_tiles<<<P.n_tc_tiles, 256, 0, s>>>(V, B, P.tc_tiles.p);
        }
        k_eeq_batch<<<P.batch_grid, 512, P.batch_smem, s>>>(V, B);
        side_after();
    }
    const double* ysol = P.bvec.p;
    if (P.nmol == 1 && !P.use_lu && P.solver == Impl::SOLVE_TILED) ysol = P.ysol.p;
    if (P.nmol == 1 && !P.use_lu && P.solver == Impl::SOLVE_PCG) ysol = P.px.p;
    k_eeq_expand<<<nblk((long)P.nfrag * 32), kBlock, 0, s>>>(P.nfrag, P.q0.p, P.atom2red.p, P.frag_off.p,
                                                              P.frag_atoms.p, ysol, P.q.p);
    P.mark(6);
    if (!fork) {
        bonded_terms();
        P.mark(7);
        hb_rep_terms();
    }
    if (split) pairs_sym(std::integral_constant<int, kPairCoul>{}, s);
    else if (P.pairs_sym) pairs_sym(std::integral_constant<int, kPairBoth>{}, s);
    else k_pairs<double><<<tgrid, kTile, 0, s>>>(V, P.nsplit);
    if (P.resp_on) {
        // u = B M^-1 B^T w with the factor (or the iteration) of this step's EEQ matrix
        k_resp_rhs<<<nblk(P.nred), kBlock, 0, s>>>(V, P.red2atom.p, P.anchor.p, P.bres.p);
        const double* y = P.bres.p;
        if (P.use_lu) {
            k_lu_solve_rhs<<<1, 1024, 0, s>>>(P.M.p, P.lda, P.nred, P.ipiv.p, P.bres.p, P.info.p);
        } else if (P.solver == Impl::SOLVE_PCG) {
            P.pcg_launch(P.bres.p, P.xres.p, P.info3.p, 1);
            k_merge_info<<<1, 1, 0, s>>>(P.info.p, P.info3.p);
            y = P.xres.p;
        } else {   // the Cholesky factor (the tiled kernel, or cuSOLVER when asked for) is in M
            k_chol_solve_rhs<<<1, 1024, 0, s>>>(P.M.p, P.lda, P.nred, P.bres.p, P.info.p);
        }
        k_eeq_expand<<<nblk((long)P.nfrag * 32), kBlock, 0, s>>>(P.nfrag, nullptr, P.atom2red.p, P.frag_off.p,
                                                                  P.frag_atoms.p, y, P.ures.p);
        k_resp_pairs<<<tgrid, kTile, 0, s>>>(V, P.nsplit);
    }
    if (fork) CK(cudaStreamWaitEvent(s, P.ev_join, 0));
    if (split && sd != s2) CK(cudaStreamWaitEvent(s, P.ev_join_d4, 0));
    P.mark(10);
    k_post<<<nblk(n), kBlock, 0, s>>>(V);
    if (P.cnl_on) {
        k_cn_chain_nl<<<nblk((long)n * 32), kBlock, 0, s>>>(V, P.cnl_off.p, P.cnl_j.p, P.cnl_bad.p);
        k_cn_chain<double><<<tgrid, kTile, 0, s>>>(V, P.nsplit, P.cnl_bad.p);
    } else {
        k_cn_chain<double><<<tgrid, kTile, 0, s>>>(V, P.nsplit, nullptr);
    }
    if (P.alpb_on) P.alpb_post(s);   // solvation energy and gradient at the solved charges
    P.mark(11);
    k_outputs<<<nblk(n), kBlock, 0, s>>>(V, P.gout.p, P.qout.p, P.cnout.p, P.bad.p);
    k_finish<<<nblk(P.nmol), kBlock, 0, s>>>(V, (P.nred > 0 || P.nmol > 1) ? P.info.p : nullptr, P.bad.p, P.e0.p,
                                             P.etot.p);
}

const double* Engine::d_terms() const { return p_->E.p; }
const double* Engine::d_grad() const { return p_->gout.p; }
const double* Engine::d_charges() const { return p_->qout.p; }
const double* Engine::d_cn() const { return p_->cnout.p; }
const int* Engine::d_status() const { return p_->status.p; }
const double* Engine::d_hb_msd() const { return p_->msd.p; }
double* Engine::d_xyz_scratch() { return p_->xyz_stage.p; }
void* Engine::stream() const { return (void*)p_->stream; }
int Engine::natoms() const { return p_->n; }
int Engine::nmol() const { return p_->nmol; }
void Engine::sync() { CK(cudaStreamSynchronize(p_->stream)); }

void Engine::fetch(double* terms, double* grad, int* status, double* hb_msd)
{
    Impl& P = *p_;
    if (terms) CK(cudaMemcpyAsync(terms, P.E.p, kNumTerms * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (grad) CK(cudaMemcpyAsync(grad, P.gout.p, 3 * (size_t)P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (status) CK(cudaMemcpyAsync(status, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    if (hb_msd) CK(cudaMemcpyAsync(hb_msd, P.msd.p, sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (P.cnl_on) CK(cudaMemcpyAsync(P.cnl_bad_host, P.cnl_bad.p, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
}

void Engine::fetch_batch(double* terms16, double* grad, int* status)
{
    Impl& P = *p_;
    if (terms16) CK(cudaMemcpyAsync(terms16, P.E.p, 16 * (size_t)P.nmol * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (grad) CK(cudaMemcpyAsync(grad, P.gout.p, 3 * (size_t)P.n * sizeof(double), cudaMemcpyDeviceToHost, P.stream));
    if (status) CK(cudaMemcpyAsync(status, P.status.p, (size_t)P.nmol * sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    if (P.cnl_on) CK(cudaMemcpyAsync(P.cnl_bad_host, P.cnl_bad.p, sizeof(int), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
}

std::vector<int> Engine::device_dispersion_pairs()
{
    Impl& P = *p_;
    if (P.n > 65535) throw std::runtime_error("device_dispersion_pairs: at most 65535 atoms");
    DBuf<unsigned long long> cnt;
    cnt.alloc(1);
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), P.stream));
    dim3 g(nblk(P.n), P.n);
    k_disp_count<<<g, kBlock, 0, P.stream>>>(P.n, P.pos0.p, P.jr.p, cnt.p, nullptr, 0);
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, cnt.p, sizeof(c), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
    DBuf<int2> out;
    out.alloc(c);
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), P.stream));
    k_disp_count<<<g, kBlock, 0, P.stream>>>(P.n, P.pos0.p, P.jr.p, cnt.p, out.p, c);
    std::vector<int2> h(c);
    if (c) CK(cudaMemcpyAsync(h.data(), out.p, c * sizeof(int2), cudaMemcpyDeviceToHost, P.stream));
    CK(cudaStreamSynchronize(P.stream));
    for (auto& p : h) {
        const int a = P.h_perm[p.x], b = P.h_perm[p.y];
        p = make_int2(std::min(a, b), std::max(a, b));
    }
    std::sort(h.begin(), h.end(), [](int2 a, int2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
    std::vector<int> v;
    v.reserve(2 * c);
    for (auto& p : h) { v.push_back(p.x); v.push_back(p.y); }
    return v;
}

bool Engine::cn_list_stale(bool read_now)
{
    Impl& P = *p_;
    if (!P.cnl_on) return false;
    if (read_now) {
        CK(cudaStreamSynchronize(P.stream));
        CK(cudaMemcpy(P.cnl_bad_host, P.cnl_bad.p, sizeof(int), cudaMemcpyDeviceToHost));
    }
    return *P.cnl_bad_host != 0;
}

void Engine::refresh_cn_list()
{
    Impl& P = *p_;
    if (!P.cnl_on) return;
    CK(cudaStreamSynchronize(P.stream));
    P.drop_graphs();   // the list buffers are reallocated
    const char* ecl = std::getenv("GFNFF_CN_LIST");
    if (ecl && !std::strcmp(ecl, "host")) {
        std::vector<double4> p(P.n);
        CK(cudaMemcpy(p.data(), P.pos.p, (size_t)P.n * sizeof(double4), cudaMemcpyDeviceToHost));
        std::vector<int2> jr(P.n);
        CK(cudaMemcpy(jr.data(), P.jr.p, (size_t)P.n * sizeof(int2), cudaMemcpyDeviceToHost));
        P.build_cn_list(p, jr);
    } else {
        P.build_cn_list_device(P.pos.p);
    }
}

// EEQ parameters of a refreshed topology with the same fragments: copied into the existing
// buffers, so that captured graphs stay valid
void Engine::update_eeq_parameters(const Model& m)
{
    Impl& P = *p_;
    if (P.nmol != 1 || m.n != P.n) throw std::runtime_error("update_eeq_parameters: single molecule of the same size");
    std::vector<double> chi(P.n), cnf(P.n), gam(P.n), alp(P.n), adg(P.n), qa(P.n);
    for (int a = 0; a < m.n; ++a) {
        const int s = P.ix(0, a);
        chi[s] = m.chi_base[a]; cnf[s] = m.cnf[a]; gam[s] = m.gam[a]; alp[s] = m.alpeeq[a];
        adg[s] = m.gam[a] + 0.797884560802866 / std::sqrt(m.alpeeq[a]);
        qa[s] = m.qa[a];
    }
    CK(cudaStreamSynchronize(P.stream));
    const size_t b = (size_t)P.n * sizeof(double);
    CK(cudaMemcpy(P.chi_base.p, chi.data(), b, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.cnf.p, cnf.data(), b, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.gam.p, gam.data(), b, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.alpeeq.p, alp.data(), b, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.adiag.p, adg.data(), b, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(P.qa.p, qa.data(), b, cudaMemcpyHostToDevice));
    P.hbd.topo = nullptr;   // the HB detection's topology inputs follow the new topology
}

void Engine::set_cell(const double* cell_bohr)
{
    p_->drop_graphs();   // captured graphs hold the view, cell included
    Cell& c = p_->cell;
    c = Cell{};
    if (!cell_bohr) return;
    // columns a, b, c: h[3*col + row] = component row of lattice vector col
    for (int k = 0; k < 9; ++k) c.h[k] = cell_bohr[k];
    auto H = [&](int r, int col) { return c.h[3 * col + r]; };
    const double det = H(0, 0) * (H(1, 1) * H(2, 2) - H(1, 2) * H(2, 1)) - H(0, 1) * (H(1, 0) * H(2, 2) - H(1, 2) * H(2, 0)) +
                       H(0, 2) * (H(1, 0) * H(2, 1) - H(1, 1) * H(2, 0));
    if (!(std::fabs(det) > 1e-12)) throw std::runtime_error("set_cell: singular cell");
    // inverse = adjugate / det; the cyclic cofactor form carries the signs
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) {
            const int r1 = (col + 1) % 3, r2 = (col + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
            c.hi[3 * col + r] = (H(r1, c1) * H(r2, c2) - H(r1, c2) * H(r2, c1)) / det;
        }
    c.on = 1;
}

void Engine::set_topo_reference(const double* xyz_bohr)
{
    Impl& P = *p_;
    std::vector<double4> r(P.n);
    for (int s = 0; s < P.n; ++s) {
        const int o = P.h_perm[s];
        r[s] = make_double4(xyz_bohr[3 * o], xyz_bohr[3 * o + 1], xyz_bohr[3 * o + 2], 0.0);
    }
    P.toporef.upload(r);
}

void Engine::set_hb_reference(const double* xyz_bohr)
{
    Impl& P = *p_;
    std::vector<double4> r(P.n);
    for (int s = 0; s < P.n; ++s) {
        const int o = P.h_perm[s];
        r[s] = make_double4(xyz_bohr[3 * o], xyz_bohr[3 * o + 1], xyz_bohr[3 * o + 2], 0.0);
    }
    P.hbref.upload(r);
}

}  // namespace gfnff
