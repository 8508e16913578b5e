// GFN-FF setup, part 1: bond graph, fragments, coordination numbers, hybridisation,
// pi systems, rings, Phase-1 (topological) EEQ charges and their corrections, and the
// Hueckel pi bond orders.  Each function cites the curcuma routine it restates
// (paths relative to src/core/energy_calculators/).
#include "setup_internal.h"
#include "topo_cache.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>
#include <queue>
#include <set>
#include <stack>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace gfnff {
namespace detail {

using namespace gfnff_tables;

double dist_bohr(const Ctx& c, int i, int j)
{
    const double dx = c.xb[3 * i] - c.xb[3 * j];
    const double dy = c.xb[3 * i + 1] - c.xb[3 * j + 1];
    const double dz = c.xb[3 * i + 2] - c.xb[3 * j + 2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

double dist2_bohr(const Ctx& c, int i, int j)
{
    const double dx = c.xb[3 * i] - c.xb[3 * j];
    const double dy = c.xb[3 * i + 1] - c.xb[3 * j + 1];
    const double dz = c.xb[3 * i + 2] - c.xb[3 * j + 2];
    return dx * dx + dy * dy + dz * dz;
}

// ---------------------------------------------------------------------------------
// Uniform-grid neighbour search used by every O(N^2) "all pairs within r" scan of the
// setup.  It enumerates exactly the pairs with squared distance <= r2 (or < r2 when
// strict), so results equal a brute-force double loop.
// ---------------------------------------------------------------------------------
namespace {
struct PairGrid {
    double lo[3] = {0, 0, 0}, cell = 1.0;
    int nc[3] = {1, 1, 1};
    std::vector<int> head, next, cid;
};

PairGrid build_pair_grid(const Ctx& c, double rcut)
{
    const int n = c.n;
    PairGrid g;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], c.xb[3 * i + d]);
            hi[d] = std::max(hi[d], c.xb[3 * i + d]);
        }
    g.cell = rcut * 1.0001 + 1e-9;
    for (int d = 0; d < 3; ++d) {
        g.lo[d] = lo[d];
        g.nc[d] = std::max(1, (int)std::floor((hi[d] - lo[d]) / g.cell) + 1);
    }
    g.head.assign((size_t)g.nc[0] * g.nc[1] * g.nc[2], -1);
    g.next.assign(n, -1);
    g.cid.resize(n);
    for (int i = n - 1; i >= 0; --i) {
        int cx = std::min(g.nc[0] - 1, (int)((c.xb[3 * i] - g.lo[0]) / g.cell));
        int cy = std::min(g.nc[1] - 1, (int)((c.xb[3 * i + 1] - g.lo[1]) / g.cell));
        int cz = std::min(g.nc[2] - 1, (int)((c.xb[3 * i + 2] - g.lo[2]) / g.cell));
        int id = (cz * g.nc[1] + cy) * g.nc[0] + cx;
        g.cid[i] = id;
        g.next[i] = g.head[id];
        g.head[id] = i;
    }
    return g;
}

// the partners j > i of row i within the cut, from the 27 cells around i's
template <class F>
void grid_row(const Ctx& c, const PairGrid& g, int i, double r2, bool strict, F&& f)
{
    const int id = g.cid[i];
    const int cx = id % g.nc[0], cy = (id / g.nc[0]) % g.nc[1], cz = id / (g.nc[0] * g.nc[1]);
    for (int dz = -1; dz <= 1; ++dz) {
        const int z = cz + dz;
        if (z < 0 || z >= g.nc[2]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = cy + dy;
            if (y < 0 || y >= g.nc[1]) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = cx + dx;
                if (x < 0 || x >= g.nc[0]) continue;
                for (int j = g.head[(z * g.nc[1] + y) * g.nc[0] + x]; j >= 0; j = g.next[j]) {
                    if (j <= i) continue;
                    const double d2 = dist2_bohr(c, i, j);
                    if (strict ? d2 < r2 : d2 <= r2) f(i, j, d2);
                }
            }
        }
    }
}
}  // namespace

void pairs_within(const Ctx& c, double rcut, bool strict,
                  const std::function<void(int, int, double)>& fn)
{
    const int n = c.n;
    const double r2 = rcut * rcut;
    if (n < 600) {
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) {
                const double d2 = dist2_bohr(c, i, j);
                if (strict ? d2 < r2 : d2 <= r2) fn(i, j, d2);
            }
        return;
    }
    const PairGrid g = build_pair_grid(c, rcut);
    for (int i = 0; i < n; ++i) grid_row(c, g, i, r2, strict, fn);
}

int setup_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void pairs_within_rows(const Ctx& c, double rcut, bool strict,
                       const std::function<void(int, int, int, double)>& fn)
{
    const int n = c.n;
    const double r2 = rcut * rcut;
    PairGrid g;
    const bool grid = n >= 600;
    if (grid) g = build_pair_grid(c, rcut);
#pragma omp parallel
    {
#ifdef _OPENMP
        const int t = omp_get_thread_num();
#else
        const int t = 0;
#endif
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            if (grid) {
                grid_row(c, g, i, r2, strict, [&](int a, int b, double d2) { fn(t, a, b, d2); });
            } else {
                for (int j = i + 1; j < n; ++j) {
                    const double d2 = dist2_bohr(c, i, j);
                    if (strict ? d2 < r2 : d2 <= r2) fn(t, i, j, d2);
                }
            }
        }
    }
}

// cn_calculator.cpp:115-177 (threshold form, default 1600 bohr^2, kn=-7.5, cnmax=4.4).
// Each atom's partners are gathered from the neighbouring cells of a grid, sorted and summed
// in ascending order (the j-loop's order), atoms in parallel; no pair list is stored.  Of the
// ~1300 partners within 40 bohr in a condensed system only those closer than 1.9 rc have a
// nonzero term; the others are dropped before the sort.
std::vector<double> cn_threshold(const Ctx& c, double threshold)
{
    const int n = c.n;
    std::vector<double> cn(n, 0.0);
    const double kn = -7.5, cnmax = 4.4;
    const double rcut = std::sqrt(threshold) + 1e-6;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], c.xb[3 * i + d]);
            hi[d] = std::max(hi[d], c.xb[3 * i + d]);
        }
    const double cell = rcut * 1.0001 + 1e-9;
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = std::max(1, (int)std::floor((hi[d] - lo[d]) / cell) + 1);
    std::vector<int> head((size_t)nc[0] * nc[1] * nc[2], -1), next(n, -1), cid(n);
    for (int i = n - 1; i >= 0; --i) {
        int cx = std::min(nc[0] - 1, (int)((c.xb[3 * i] - lo[0]) / cell));
        int cy = std::min(nc[1] - 1, (int)((c.xb[3 * i + 1] - lo[1]) / cell));
        int cz = std::min(nc[2] - 1, (int)((c.xb[3 * i + 2] - lo[2]) / cell));
        const int id = (cz * nc[1] + cy) * nc[0] + cx;
        cid[i] = id;
        next[i] = head[id];
        head[id] = i;
    }
#pragma omp parallel
    {
        std::vector<std::pair<int, double>> v;
#pragma omp for schedule(dynamic, 32)
        for (int i = 0; i < n; ++i) {
            v.clear();
            const int id = cid[i];
            const int cx = id % nc[0], cy = (id / nc[0]) % nc[1], cz = id / (nc[0] * nc[1]);
            for (int z = std::max(0, cz - 1); z <= std::min(nc[2] - 1, cz + 1); ++z)
                for (int y = std::max(0, cy - 1); y <= std::min(nc[1] - 1, cy + 1); ++y)
                    for (int x = std::max(0, cx - 1); x <= std::min(nc[0] - 1, cx + 1); ++x)
                        for (int j = head[(z * nc[1] + y) * nc[0] + x]; j >= 0; j = next[j]) {
                            if (j == i) continue;
                            const double d2 = dist2_bohr(c, std::min(i, j), std::max(i, j));
                            if (d2 > threshold) continue;
                            // a partner at r >= 1.9 rc counts exactly 0 in double (erf(-7.5 * 0.9)
                            // rounds to -1), so leaving it out keeps the ordered sum bit for bit
                            const double rc = c.rcov_cn[i] + c.rcov_cn[j];
                            if (d2 >= 3.61 * rc * rc) continue;
                            v.push_back({j, d2});
                        }
            std::sort(v.begin(), v.end());
            double s = 0.0;
            for (auto& p : v) {
                const double r = std::sqrt(p.second);
                const double rc = c.rcov_cn[i] + c.rcov_cn[p.first];
                const double dr = (r - rc) / rc;
                s += 0.5 * (1.0 + std::erf(kn * dr));
            }
            cn[i] = std::log(1.0 + std::exp(cnmax)) - std::log(1.0 + std::exp(cnmax - s));
        }
    }
    return cn;
}

// ff_methods/gfnff_method.cpp:940-1000 (getCachedBondList)
void build_bond_graph(Ctx& c)
{
    const int n = c.n;
    std::vector<double> rc(n), ft(n);
    double rmax = 0.0;
    for (int i = 0; i < n; ++i) {
        rc[i] = covalent_radii[c.Z[i] - 1] * kAngToBohr;
        ft[i] = fat[c.Z[i]];
        rmax = std::max(rmax, rc[i] * ft[i]);
    }
    const double rcut = 1.3 * 2.0 * rmax * 1.2 + 1e-6;
    std::vector<std::pair<int, int>> bl;
    pairs_within(c, rcut, false, [&](int i, int j, double) {
        const double d = dist_bohr(c, i, j);
        const double thr = 1.3 * (rc[i] + rc[j]) * ft[i] * ft[j];
        if (d < thr) bl.push_back({i, j});
    });
    std::sort(bl.begin(), bl.end());
    c.m.topo_bonds = bl;
    c.m.adj.assign(n, {});
    for (auto& b : bl) {
        c.m.adj[b.first].push_back(b.second);
        c.m.adj[b.second].push_back(b.first);
    }
    c.bondset.clear();
    for (auto& b : bl) c.bondset.insert(key(b.first, b.second));
}

// gfnff_method.cpp:8772-8812 (detectMolecularFragments, BFS)
void detect_fragments(Ctx& c)
{
    const int n = c.n;
    std::vector<int> fl(n, 0);
    int nf = 0;
    for (int i = 0; i < n; ++i) {
        if (fl[i]) continue;
        ++nf;
        std::queue<int> q;
        q.push(i);
        fl[i] = nf;
        while (!q.empty()) {
            int a = q.front();
            q.pop();
            for (int b : c.m.adj[a])
                if (!fl[b]) { fl[b] = nf; q.push(b); }
        }
    }
    c.m.nfrag = nf;
    c.m.frag.resize(n);
    for (int i = 0; i < n; ++i) c.m.frag[i] = fl[i] - 1;
    c.m.qfrag.assign(nf, 0.0);
    if (nf == 1) c.m.qfrag[0] = (double)c.m.charge;
}

// gfnff_method.cpp:6446-6586 (determineHybridization)
void determine_hybridization(Ctx& c)
{
    const int n = c.n;
    c.m.hyb.assign(n, 3);
    for (int i = 0; i < n; ++i) {
        const int z = c.Z[i];
        const auto& nb = c.m.adj[i];
        std::vector<std::array<double, 3>> bv;
        for (int j : nb) {
            double v[3] = {c.xb[3 * j] - c.xb[3 * i], c.xb[3 * j + 1] - c.xb[3 * i + 1],
                           c.xb[3 * j + 2] - c.xb[3 * i + 2]};
            const double r = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            bv.push_back({v[0] / r, v[1] / r, v[2] / r});
        }
        const int k = (int)nb.size();
        int h = 3;
        auto dot = [&](int a, int b) {
            return bv[a][0] * bv[b][0] + bv[a][1] * bv[b][1] + bv[a][2] * bv[b][2];
        };
        if (k == 0) {
            h = 3;
        } else if (k == 1) {
            if (z == 8 || z == 16) h = (c.m.adj[nb[0]].size() == 1) ? 1 : 2;
            else if (z == 1 || z == 9 || z == 17 || z == 35 || z == 53) h = 0;
            else h = 1;
        } else if (k == 2) {
            if (z == 8 || z == 16) h = 3;
            else if (z == 9 || z == 17 || z == 35 || z == 53) h = 1;
            else {
                const double ang = std::acos(std::max(-1.0, std::min(1.0, dot(0, 1))));
                h = (ang > 2.8) ? 1 : 2;
            }
        } else if (k == 3) {
            if (z == 7) h = 3;
            else {
                double s = 0.0;
                for (int a = 0; a < 3; ++a)
                    s += std::acos(std::max(-1.0, std::min(1.0, dot(a, (a + 1) % 3))));
                h = (s > 6.0) ? 2 : 3;
            }
        } else {
            h = 3;
        }
        c.m.hyb[i] = h;
    }
}

// gfnff_method.cpp:6588-6697 (detectPiSystems)
void detect_pi_systems(Ctx& c)
{
    const int n = c.n;
    auto cand = [](int z) { return z == 5 || z == 6 || z == 7 || z == 8 || z == 9 || z == 16 || z == 17; };
    auto hetero = [](int z) { return z == 5 || z == 7 || z == 8 || z == 9 || z == 16 || z == 17; };
    auto unsat = [&](int i) { return c.m.hyb[i] == 1 || c.m.hyb[i] == 2; };
    std::vector<std::vector<int>> pn(n);
    for (int i = 0; i < n; ++i) {
        if (!cand(c.Z[i])) continue;
        for (int j : c.m.adj[i]) {
            if (j <= i || !cand(c.Z[j])) continue;
            bool pb = (unsat(i) && unsat(j)) || (unsat(i) && hetero(c.Z[j])) ||
                      (unsat(j) && hetero(c.Z[i]));
            if (pb) { pn[i].push_back(j); pn[j].push_back(i); }
        }
    }
    c.m.pi_frag.assign(n, 0);
    std::vector<char> vis(n, 0);
    int id = 1;
    for (int s = 0; s < n; ++s) {
        if (pn[s].empty() || vis[s]) continue;
        std::stack<int> st;
        st.push(s);
        vis[s] = 1;
        while (!st.empty()) {
            int a = st.top();
            st.pop();
            c.m.pi_frag[a] = id;
            for (int b : pn[a])
                if (!vis[b]) { vis[b] = 1; st.push(b); }
        }
        ++id;
    }
}

// gfnff_method.cpp:6698-6797 (findSmallestRings, rings up to 6 atoms)
void find_rings(Ctx& c)
{
    const int n = c.n;
    const int kMax = 6;
    std::set<std::vector<int>> uniq;
    std::vector<int> path;
    for (int u = 0; u < n; ++u) {
        for (int v : c.m.adj[u]) {
            if (v <= u) continue;
            path.assign({u, v});
            std::function<void(int, int)> dfs = [&](int cur, int depth) {
                if (depth >= kMax) return;
                for (int nx : c.m.adj[cur]) {
                    if (nx == u && depth >= 2) {
                        std::vector<int> r = path;
                        std::sort(r.begin(), r.end());
                        uniq.insert(r);
                        continue;
                    }
                    if (nx == u) continue;
                    if (std::find(path.begin(), path.end(), nx) != path.end()) continue;
                    path.push_back(nx);
                    dfs(nx, depth + 1);
                    path.pop_back();
                }
            };
            dfs(v, 1);
        }
    }
    c.rings.assign(uniq.begin(), uniq.end());
    c.atom_rings.assign(n, {});
    for (int r = 0; r < (int)c.rings.size(); ++r)
        for (int a : c.rings[r]) c.atom_rings[a].push_back(r);
    c.m.ring_size.assign(n, 0);
    for (int a = 0; a < n; ++a) {
        int s = 0;
        for (int r : c.atom_rings[a]) {
            int sz = (int)c.rings[r].size();
            if (s == 0 || sz < s) s = sz;
        }
        c.m.ring_size[a] = s;
    }
}

static bool ring_has(const std::vector<int>& r, int a)
{
    return std::binary_search(r.begin(), r.end(), a);
}

// gfnff_method.cpp:6798-6838
int same_ring_size(const Ctx& c, int i, int j)
{
    int s = 0;
    for (int r : c.atom_rings[i])
        if (ring_has(c.rings[r], j)) {
            int sz = (int)c.rings[r].size();
            if (s == 0 || sz < s) s = sz;
        }
    return s;
}

// gfnff_method.cpp:6839-6869
int smallest_ring_all(const Ctx& c, int i, int j, int k, int l)
{
    int s = 0;
    for (int r : c.atom_rings[j]) {
        const auto& R = c.rings[r];
        if (ring_has(R, i) && ring_has(R, k) && ring_has(R, l)) {
            int sz = (int)R.size();
            if (s == 0 || sz < s) s = sz;
        }
    }
    return s;
}

// gfnff_method.cpp:6938-6966
int largest_ring_all(const Ctx& c, int i, int j, int k, int l)
{
    int s = 0;
    for (int r : c.atom_rings[j]) {
        const auto& R = c.rings[r];
        if (ring_has(R, i) && ring_has(R, k) && ring_has(R, l)) s = std::max(s, (int)R.size());
    }
    return s;
}

// gfnff_method.cpp:6870-6937
int smallest_ring_bend(const Ctx& c, int i, int j, int k)
{
    if (c.atom_rings[i].empty() || c.atom_rings[j].empty() || c.atom_rings[k].empty()) return 0;
    int s = 0;
    auto upd = [&](int a, int b, int d) {
        for (int r : c.atom_rings[a]) {
            const auto& R = c.rings[r];
            if (ring_has(R, b) && ring_has(R, d)) {
                int sz = (int)R.size();
                if (s == 0 || sz < s) s = sz;
            }
        }
    };
    upd(i, j, k);
    upd(j, i, k);
    upd(k, i, j);
    return s;
}

// gfnff_method.cpp:8693-8771 (BFS bond-count distances, capped at 5).  Stored sparse:
// only pairs with distance <= 5 are kept (the dense matrix holds 999 elsewhere).
void topo_distances(Ctx& c)
{
    const int n = c.n;
    c.tdist.assign(n, {});
    std::vector<int> d(n, -1), touched;
    for (int s = 0; s < n; ++s) {
        std::queue<int> q;
        q.push(s);
        d[s] = 0;
        touched.assign(1, s);
        while (!q.empty()) {
            int a = q.front();
            q.pop();
            if (d[a] >= 5) continue;
            for (int b : c.m.adj[a])
                if (d[b] < 0) { d[b] = d[a] + 1; q.push(b); touched.push_back(b); }
        }
        for (int t : touched) {
            if (t != s) c.tdist[s].push_back({t, d[t]});
            d[t] = -1;
        }
        std::sort(c.tdist[s].begin(), c.tdist[s].end());
    }
}

int topo_dist(const Ctx& c, int i, int j)
{
    if (i == j) return 0;
    const auto& v = c.tdist[i];
    auto it = std::lower_bound(v.begin(), v.end(), std::make_pair(j, -1));
    if (it != v.end() && it->first == j) return it->second;
    return 999;
}

// ---------------------------------------------------------------------------------
// EEQ helper functions (ff_methods/eeq_solver.cpp)
// ---------------------------------------------------------------------------------

// eeq_solver.cpp:4483-4516 (detectPiSystem) with the given hybridisation
std::vector<char> eeq_pi_atoms(const Ctx& c, const std::vector<int>& hyb)
{
    const int n = c.n;
    std::vector<char> pi(n, 0);
    auto el = [](int z) { return z == 6 || z == 7 || z == 8 || z == 9 || z == 16; };
    for (int i = 0; i < n; ++i) {
        if ((hyb[i] == 1 || hyb[i] == 2) && el(c.Z[i])) pi[i] = 1;
        if (hyb[i] == 3 && (c.Z[i] == 7 || c.Z[i] == 8 || c.Z[i] == 9)) {
            for (int j : c.m.adj[i])
                if (hyb[j] == 1 || hyb[j] == 2) { pi[i] = 1; break; }
        }
    }
    return pi;
}

// eeq_solver.cpp:4518-4570 (detectAmideNitrogens; keeps the index-based npiall test)
std::vector<char> eeq_amide_n(const Ctx& c, const std::vector<int>& hyb, const std::vector<char>& pi)
{
    const int n = c.n;
    std::vector<char> am(n, 0);
    int npiall = 0;
    for (int k = 0; k < n; ++k) npiall += pi[k] ? 1 : 0;
    for (int i = 0; i < n; ++i) {
        if (c.Z[i] != 7 || i >= npiall) continue;
        if (hyb[i] != 3) continue;
        int nc = 0, ic = -1;
        for (int nb : c.m.adj[i])
            if (c.Z[nb] == 6 && nb < npiall) { ++nc; ic = nb; }
        if (nc != 1) continue;
        int no = 0;
        for (int n2 : c.m.adj[ic])
            if (c.Z[n2] == 8 && n2 < npiall && c.m.adj[n2].size() == 1) ++no;
        if (no == 1) am[i] = 1;
    }
    return am;
}

// eeq_solver.cpp:4572-4603 (detectAmideHydrogens)
std::vector<char> eeq_amide_h(const Ctx& c, const std::vector<int>& hyb, const std::vector<char>& am)
{
    const int n = c.n;
    std::vector<char> ah(n, 0);
    for (int i = 0; i < n; ++i) {
        if (c.Z[i] != 1) continue;
        for (int nb : c.m.adj[i]) {
            if (c.Z[nb] == 7 && am[nb]) {
                int sp3c = 0;
                for (int n2 : c.m.adj[nb])
                    if (c.Z[n2] == 6 && hyb[n2] == 3) ++sp3c;
                if (sp3c == 1) ah[i] = 1;
                break;
            }
        }
    }
    return ah;
}

// eeq_solver.cpp:4059-4299 (calculateDxi).  The pi flags feeding the nitro term use
// the topology hybridisation.
std::vector<double> eeq_dxi(const Ctx& c)
{
    const int n = c.n;
    std::vector<double> dxi(n, 0.0);
    std::vector<char> pi = eeq_pi_atoms(c, c.m.hyb);
    for (int i = 0; i < n; ++i) {
        const int ati = c.Z[i];
        double d = 0.0;
        int nh = 0, nm = 0;
        const int nn = (int)c.m.adj[i].size();
        for (int j : c.m.adj[i]) {
            const int zj = c.Z[j];
            if (zj == 1) ++nh;
            if (zj > 20 && (zj <= 30 || (zj >= 39 && zj <= 48) || (zj >= 72 && zj <= 80))) ++nm;
        }
        if (ati == 5 && nh > 0) d += nh * 0.015;
        if (ati == 6 && nn == 2) {
            int a = c.m.adj[i][0], b = c.m.adj[i][1];
            double v1[3], v2[3];
            for (int k = 0; k < 3; ++k) {
                v1[k] = c.xb[3 * a + k] - c.xb[3 * i + k];
                v2[k] = c.xb[3 * b + k] - c.xb[3 * i + k];
            }
            double r1 = std::sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
            double r2 = std::sqrt(v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2]);
            if (r1 > 1e-10 && r2 > 1e-10) {
                double ca = (v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2]) / (r1 * r2);
                ca = std::max(-1.0, std::min(1.0, ca));
                if (std::acos(ca) * 180.0 / M_PI < 150.0) d += -0.15;
            }
        }
        if (ati == 8) {
            if (nn == 1 && pi[i]) {
                for (int j : c.m.adj[i])
                    if (c.Z[j] == 7 && pi[j]) d += 0.05;
            }
            if (nn == 1) {
                for (int j : c.m.adj[i])
                    if (c.Z[j] == 6 && c.m.adj[j].size() == 1) d += 0.15;
            }
            if (nn == 2 && nh == 2) d += -0.02;
            if (nh > 0) d += -nh * 0.005;
            if (nn > 2) d += nn * 0.005;
        }
        if (ati == 16) {
            if (nh > 0) d += -nh * 0.005;
            if (nn > 2) d += nn * 0.005;
        }
        const int grp = periodic_group[ati - 1];
        if (ati > 9 && grp == 7 && nn > 1) {
            if (nm == 0) d += -nn * 0.021;
            else d += nn * 0.05;
        }
        dxi[i] = d;
    }
    return dxi;
}

// eeq_solver.cpp:4301-4387 (calculateDgam)
std::vector<double> eeq_dgam(const Ctx& c, const std::vector<double>& qa,
                             const std::vector<char>& pi, const std::vector<char>& am)
{
    const int n = c.n;
    std::vector<double> dg(n, 0.0);
    int npiall = 0;
    for (int k = 0; k < n; ++k) npiall += pi[k] ? 1 : 0;
    for (int i = 0; i < n; ++i) {
        const int Z = c.Z[i];
        const int h = c.m.hyb[i];
        double ff = 0.0;
        if (Z == 1) ff = -0.08;
        else if (Z == 5) ff = -0.05;
        else if (Z == 6) {
            ff = -0.27;
            if (h < 3) ff = -0.45;
            if (h < 2) ff = -0.34;
        } else if (Z == 7) {
            ff = -0.13;
            if (i < npiall) ff = -0.14;
            if (am[i]) ff = -0.16;
        } else if (Z == 8) {
            ff = -0.15;
            if (h < 3) ff = -0.08;
        } else if (Z == 9) {
            ff = 0.10;
        } else if (Z > 10) {
            ff = -0.02;
            if (Z == 17) ff = -0.02;
            if (Z == 35) ff = -0.11;
            if (Z == 53) ff = -0.07;
            if (Z <= 86) {
                const int mt = metal_type[Z - 1];
                if (mt == 1) ff = -0.08;
                if (mt == 2) ff = -0.9;
                if (periodic_group[Z - 1] == 8) ff = 0.0;
            }
        }
        dg[i] = qa[i] * ff;
    }
    return dg;
}

// eeq_solver.cpp:3093-3199 (computeTopologicalDistancesSparse): Dijkstra over the
// bond graph with single-precision edge lengths (sum of covalent radii in Angstrom),
// paths longer than 12 A capped to 13 A, scaled by 1.175 and converted to bohr.
// Returns, per atom, the (atom, distance_bohr) pairs reached within the 12 A bound.
std::vector<std::vector<std::pair<int, double>>> topological_distances(const Ctx& c, double& far)
{
    const int n = c.n;
    const float kCap = 13.0f, kThr = 12.0f;
    const double kScale = 1.175, kB2A = 0.52917726;
    std::vector<float> rad(n);
    for (int i = 0; i < n; ++i) rad[i] = (float)covalent_radii[c.Z[i] - 1];
    std::vector<std::vector<std::pair<int, double>>> out(n);
    far = kScale * (double)kCap / kB2A;
#pragma omp parallel
    {
        std::vector<float> dist(n, kCap);
        std::vector<int> touched;
#pragma omp for schedule(dynamic, 16)
        for (int s = 0; s < n; ++s) {
            using E = std::pair<float, int>;
            std::priority_queue<E, std::vector<E>, std::greater<E>> pq;
            dist[s] = 0.0f;
            touched.assign(1, s);
            pq.push({0.0f, s});
            while (!pq.empty()) {
                auto [d, u] = pq.top();
                pq.pop();
                if (d > dist[u]) continue;
                if (d > kThr) continue;
                for (int v : c.m.adj[u]) {
                    const float w = rad[u] + rad[v];
                    const float nd = d + w;
                    if (nd < dist[v]) {
                        if (dist[v] == kCap) touched.push_back(v);
                        dist[v] = nd;
                        pq.push({nd, v});
                    }
                }
            }
            for (int t : touched) {
                const float r = dist[t];
                const double val = (r > kThr) ? (double)kCap : (double)r;
                if (t != s) out[s].push_back({t, kScale * val / kB2A});
                dist[t] = kCap;
            }
            std::sort(out[s].begin(), out[s].end());
        }
    }
    return out;
}

// Phase-1 (topological) EEQ, eeq_solver.cpp:2684-3004 (calculateTopologyCharges).
// The matrix element of every pair farther apart than the 12 A path bound is the same
// constant erf(gamma*R)/R with R = 1.175*13/0.52917726 bohr; for all GFN-FF elements
// gamma*R > 6.9 so erf(gamma*R) == 1 exactly and that part of A is the rank-one term
// (1/R) 1 1^T.  Because the fragment constraints fix 1^T q = sum(qfrag), that term
// only shifts the right-hand side, and the system separates into one small constrained
// solve per fragment (same solution as the dense augmented system).  A dense path is
// kept for the rare case the constant does not round to 1/R.
std::vector<double> phase1_charges(const Ctx& c, const std::vector<double>& qfrag,
                                   const std::vector<double>& dxi, bool* ok)
{
    const int n = c.n;
    const double TSQRT2PI = 0.797884560802866;
    double far;
    auto td = topological_distances(c, far);
    std::vector<double> chi(n), gam(n), alp(n);
    for (int i = 0; i < n; ++i) {
        const int z = c.Z[i];
        double nb = std::min((double)c.m.adj[i].size(), 4.4);
        chi[i] = -chi_eeq[z - 1] + dxi[i] + cnf_eeq[z - 1] * std::sqrt(nb);
        gam[i] = gam_eeq[z - 1];
        alp[i] = alpha_eeq[z - 1] * alpha_eeq[z - 1];
    }
    bool rank_one;
    {
        // the largest alpha pair gives the smallest gamma*R; if that rounds erf to 1,
        // every far pair does
        double amax = 0.0;
        for (int i = 0; i < n; ++i) amax = std::max(amax, alp[i]);
        const double g = 1.0 / std::sqrt(amax + amax);
        rank_one = (std::erf(g * far) == 1.0);
    }
    const double cfar = 1.0 / far;
    std::vector<double> q(n, 0.0);
    *ok = true;
    if (!rank_one || c.m.nfrag == 1) {
        // dense augmented solve, A_ij = erf(gamma_ij r_ij)/r_ij with gamma = 1/sqrt(a_i+a_j)
        std::vector<double> A((size_t)n * n, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            A[(size_t)i * n + i] = gam[i] + TSQRT2PI / std::sqrt(alp[i]);
            size_t p = 0;
            const auto& row = td[i];
            for (int j = 0; j < i; ++j) {
                double r = far;
                while (p < row.size() && row[p].first < j) ++p;
                if (p < row.size() && row[p].first == j) r = row[p].second;
                const double gij = 1.0 / std::sqrt(alp[i] + alp[j]);
                A[(size_t)i * n + j] = std::erf(gij * r) / r;
            }
        }
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < i; ++j) A[(size_t)j * n + i] = A[(size_t)i * n + j];
        *ok = linalg::eeq_schur_solve(A.data(), n, chi.data(), c.m.frag.data(), c.m.nfrag,
                                      qfrag.data(), q.data());
        return q;
    }
    // per-fragment decomposition
    double qtot = 0.0;
    for (double v : qfrag) qtot += v;
    std::vector<std::vector<int>> members(c.m.nfrag);
    for (int i = 0; i < n; ++i) members[c.m.frag[i]].push_back(i);
#pragma omp parallel for schedule(dynamic, 4)
    for (int f = 0; f < c.m.nfrag; ++f) {
        const auto& mem = members[f];
        const int m = (int)mem.size();
        std::vector<double> S((size_t)m * m, 0.0), rhs(m);
        for (int a = 0; a < m; ++a) {
            const int i = mem[a];
            S[(size_t)a * m + a] = gam[i] + TSQRT2PI / std::sqrt(alp[i]) - cfar;
            rhs[a] = chi[i] - cfar * qtot;
        }
        for (int a = 0; a < m; ++a) {
            const int i = mem[a];
            for (auto& p : td[i]) {
                const int j = p.first;
                auto it = std::lower_bound(mem.begin(), mem.end(), j);
                const int b = (int)(it - mem.begin());
                const double gij = 1.0 / std::sqrt(alp[i] + alp[j]);
                S[(size_t)a * m + b] = std::erf(gij * p.second) / p.second - cfar;
            }
        }
        std::vector<int> fr(m, 0);
        double qf = qfrag[f];
        std::vector<double> qq(m);
        bool good = linalg::eeq_schur_solve(S.data(), m, rhs.data(), fr.data(), 1, &qf, qq.data());
        if (!good) {
#pragma omp critical
            *ok = false;
        }
        for (int a = 0; a < m; ++a) q[mem[a]] = qq[a];
    }
    return q;
}

// Energy of the Phase-1 style EEQ model used to place the charge of a charged
// two-fragment system (gfnff_method.cpp:7505-7555, calculateEEQEnergy).
double eeq_energy_geometric(const Ctx& c, const std::vector<double>& q, const std::vector<double>& cn)
{
    const int n = c.n;
    const double sqrt_2pi = 0.79788456080287;
    double e = 0.0;
    for (int i = 0; i < n; ++i) {
        const int zi = c.Z[i];
        const double ai = alpha_eeq[zi - 1] * alpha_eeq[zi - 1];
        for (int j = 0; j < i; ++j) {
            const int zj = c.Z[j];
            const double aj = alpha_eeq[zj - 1] * alpha_eeq[zj - 1];
            const double r = dist_bohr(c, i, j);
            const double g = 1.0 / std::sqrt(ai + aj);
            e += q[i] * q[j] * std::erf(g * r) / r;
        }
        const double self = gam_eeq[zi - 1] + sqrt_2pi / std::sqrt(ai);
        const double en = chi_eeq[zi - 1] + cnf_eeq[zi - 1] * std::sqrt(cn[i]);
        e += -q[i] * en + 0.5 * q[i] * q[i] * self;
    }
    return e;
}

// ---------------------------------------------------------------------------------
// Hueckel pi bond orders, ff_methods/huckel_solver.cpp:20-230
// ---------------------------------------------------------------------------------
static int pi_electrons(int z, int hyb)
{
    switch (z) {
        case 5: return hyb == 1 ? 1 : 0;
        case 6: return 1;
        case 7: return hyb <= 2 ? 1 : (hyb == 3 ? 2 : 0);
        case 8: return hyb == 1 ? 1 : (hyb == 2 ? 1 : (hyb == 3 ? 2 : 0));
        case 9: return hyb != 1 ? 2 : 3;
        case 16: return hyb == 1 ? 1 : (hyb == 2 ? 1 : (hyb == 3 ? 2 : 0));
        case 17: return hyb == 0 ? 2 : (hyb == 1 ? 3 : 0);
        default: return 0;
    }
}

static std::vector<double> fermi_occ(const std::vector<double>& e, int nel, double temp)
{
    const int no = (int)e.size();
    std::vector<double> occ(no, 0.0);
    const double boltz_ev = 8.617333262e-5;
    if (temp < 1.0) {
        for (int i = 0; i < nel && i < no; ++i) occ[i] = 1.0;
        return occ;
    }
    const double bkt = boltz_ev * temp;
    const int ihomo = std::min(nel, no) - 1;
    const int ilumo = std::min(nel, no - 1);
    double ef = 0.5 * (e[ihomo] + e[ilumo]);
    const double target = (double)nel;
    for (int cyc = 0; cyc < 200; ++cyc) {
        double tot = 0.0, der = 0.0;
        for (int i = 0; i < no; ++i) {
            const double x = (e[i] - ef) / bkt;
            double f = 0.0, fd = 0.0;
            if (x < 50.0) {
                const double ex = std::exp(x);
                f = 1.0 / (ex + 1.0);
                fd = ex / (bkt * (ex + 1.0) * (ex + 1.0));
            }
            occ[i] = f;
            tot += f;
            der += fd;
        }
        ef += (target - tot) / der;
        if (std::fabs(target - tot) < 1e-9) break;
    }
    return occ;
}

void huckel_bond_orders(Ctx& c, const std::vector<int>& pis_charge)
{
    const int n = c.n;
    static const double hdiag[18] = {0.0, 0.0, 0.0, 0.0, 0.0, -0.5, 0.0, 0.14, -0.38, -0.29,
                                     0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -0.30, -0.30};
    static const double hoff[18] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.66, 1.1, 0.23,
                                    0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.6, 1.0};
    const double hiter = 0.700, htriple = 1.45, hueckelp3 = -0.24, pilpf = 0.530;
    const int maxhiter = 5;
    const double conv = 1e-4, ftemp = 4000.0, h2ev = 27.2113957;
    c.pibo.clear();
    std::set<int> ids;
    for (int f : c.m.pi_frag) if (f > 0) ids.insert(f);
    for (int pis : ids) {
        std::vector<int> atoms, map(n, -1), pel(n, 0);
        int nel = 0;
        for (int k = 0; k < n; ++k)
            if (c.m.pi_frag[k] == pis) {
                map[k] = (int)atoms.size();
                atoms.push_back(k);
                int e = pi_electrons(c.Z[k], c.m.hyb[k]);
                pel[k] = e;
                nel += e;
                if (pel[k] > 2) pel[k] = 2;
            }
        const int np = (int)atoms.size();
        if (pis < (int)pis_charge.size()) nel -= pis_charge[pis];
        if (np < 2 || nel < 1) continue;
        std::vector<double> P((size_t)np * np, 2.0 / 3.0);
        double Eold = 0.0;
        for (int it = 0; it < maxhiter; ++it) {
            std::vector<double> H((size_t)np * np, 0.0);
            for (int a = 0; a < np; ++a) {
                const int k = atoms[a];
                const int Z = c.Z[k];
                const double hd = Z < 18 ? hdiag[Z] : 0.0;
                H[(size_t)a * np + a] = hd + c.m.qa[k] * hueckelp3 - (double)(pel[k] - 1) * pilpf;
            }
            for (auto& b : c.m.topo_bonds) {
                const int ia = map[b.first], ja = map[b.second];
                if (ia < 0 || ja < 0) continue;
                const int zi = c.Z[b.first], zj = c.Z[b.second];
                const double hi = zi < 18 ? hoff[zi] : 0.0, hj = zj < 18 ? hoff[zj] : 0.0;
                double beta = std::sqrt(hi * hj);
                beta -= 1.0e-9 * dist_bohr(c, b.first, b.second);
                double damp = hiter;
                if (c.m.hyb[b.first] == 1) damp *= htriple;
                if (c.m.hyb[b.second] == 1) damp *= htriple;
                const double hij = -beta * (1.0 - damp * (2.0 / 3.0 - P[(size_t)ja * np + ia]));
                H[(size_t)ja * np + ia] = hij;
                H[(size_t)ia * np + ja] = hij;
            }
            std::vector<double> ev, V;
            linalg::sym_eig(H, np, ev, V);
            for (double& e : ev) e *= 0.1 * h2ev;
            std::vector<double> occ = fermi_occ(ev, nel / 2, ftemp);
            for (double& o : occ) o *= 2.0;
            const int ih = nel / 2;
            if (ih > 0 && ih < np && std::fabs(occ[ih - 1] - occ[ih]) < 1e-4) {
                std::fill(occ.begin(), occ.end(), 0.0);
                for (int i = 0; i < nel / 2; ++i) occ[i] = 2.0;
            }
            double Enew = 0.0;
            for (int i = 0; i < np; ++i) Enew += occ[i] * ev[i];
            std::vector<double> Pn((size_t)np * np, 0.0);
            for (int a = 0; a < np; ++a)
                for (int b = 0; b < np; ++b) {
                    double s = 0.0;
                    for (int k = 0; k < np; ++k) s += V[(size_t)a * np + k] * occ[k] * V[(size_t)b * np + k];
                    Pn[(size_t)a * np + b] = s;
                }
            P.swap(Pn);
            if (std::fabs(Enew - Eold) < conv) break;
            Eold = Enew;
        }
        for (auto& b : c.m.topo_bonds) {
            const int ia = map[b.first], ja = map[b.second];
            if (ia >= 0 && ja >= 0) c.pibo[key(b.first, b.second)] = P[(size_t)ja * np + ia];
        }
    }
}

double pibo_of(const Ctx& c, int i, int j)
{
    auto it = c.pibo.find(key(i, j));
    return it == c.pibo.end() ? 0.0 : it->second;
}

// gfnff_method.cpp:4021-4098 (classifyBondType)
int classify_bond(const Ctx& c, int a, int b, int hi, int hj)
{
    int bt = 1;
    if (hi == 2 && hj == 2) bt = 2;
    const int zi = c.Z[a], zj = c.Z[b];
    if ((hi == 3 && hj == 2 && zi == 7) || (hj == 3 && hi == 2 && zj == 7)) bt = 2;
    if (hi == 1 || hj == 1) bt = 3;
    auto hal = [](int z) { return z == 9 || z == 17 || z == 35 || z == 53 || z == 85; };
    if ((hal(zi) || zi == 1) && hi == 1) bt = 3;
    if ((hal(zj) || zj == 1) && hj == 1) bt = 3;
    if (hi == 5 || hj == 5) bt = 4;
    if (c.is_metal[a] || c.is_metal[b]) bt = 5;
    if (c.is_metal[a] && c.is_metal[b]) bt = 7;
    return bt;
}

// The topology block of gfnff_method.cpp:8813-9557 (calculateTopologyInfo).
void compute_topology(Ctx& c)
{
    const int n = c.n;
    c.is_metal.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        const int z = c.Z[i];
        c.is_metal[i] = (z >= 21 && z <= 30) || (z >= 39 && z <= 48) || (z >= 57 && z <= 80);
    }
    build_bond_graph(c);
    detect_fragments(c);
    c.m.cn_setup = cn_threshold(c, 1600.0);
    determine_hybridization(c);
    detect_pi_systems(c);
    find_rings(c);

    c.m.rings = c.rings;

    // Topology cache (gfnff_method.cpp:8973-9040): on a fingerprint match the Phase-1
    // results (charges, fragment charges, dxi, dgam, alpeeq, amide-H flags) come from the
    // file and Phase 1, 1A, 1B and 1C are skipped.
    TopoCache tc;
    bool hit = c.topo_cache && read_topology_cache(c.topo_cache, topology_fingerprint(c.m.Z, c.m.topo_bonds), n, tc);
    if (hit && tc.has_qfrag && (int)tc.qfrag.size() != c.m.nfrag) hit = false;
    c.m.topo_cache_hit = hit;
    std::vector<double> dxi, dgam;
    std::vector<char> ah;
    if (hit) {
        dxi = tc.dxi;
        c.m.qa = tc.qa;
        if (tc.has_qfrag) c.m.qfrag = tc.qfrag;
        c.m.alpeeq = tc.alpeeq;
        dgam = tc.dgam;
        ah = tc.has_amide_h ? tc.amide_h : std::vector<char>(n, 0);
    } else {
        // Phase-1 charges (with the charged two-fragment placement rule, :8990-9035)
        dxi = eeq_dxi(c);
        bool ok = true;
        const double qc = (double)c.m.charge;
        if (c.m.nfrag == 2 && c.m.charge != 0) {
            std::vector<double> qA = {qc, 0.0}, qB = {0.0, qc};
            bool oka, okb;
            auto qa = phase1_charges(c, qA, dxi, &oka);
            auto qb = phase1_charges(c, qB, dxi, &okb);
            double ea = oka ? eeq_energy_geometric(c, qa, c.m.cn_setup) : 1e300;
            double eb = okb ? eeq_energy_geometric(c, qb, c.m.cn_setup) : 1e300;
            if (ea <= eb) { c.m.qfrag = qA; c.m.qa = qa; ok = oka; }
            else { c.m.qfrag = qB; c.m.qa = qb; ok = okb; }
        } else {
            if (c.m.nfrag > 2 && c.m.charge != 0) {
                c.m.qfrag.assign(c.m.nfrag, 0.0);
                c.m.qfrag[0] = qc;
            }
            c.m.qa = phase1_charges(c, c.m.qfrag, dxi, &ok);
        }
        if (!ok) throw std::runtime_error("Phase-1 EEQ solve failed");

        // alpeeq (gfnff_method.cpp:11182-11276)
        c.m.alpeeq.resize(n);
        for (int i = 0; i < n; ++i) {
            const int z = c.Z[i];
            const double ab = alpha_eeq[z - 1];
            double ff = 0.0;
            if (z == 6) ff = 0.09;
            else if (z == 7) ff = -0.21;
            else {
                const int g = periodic_group[z - 1];
                if (g == 6) ff = -0.03;
                else if (g == 7) ff = 0.50;
                else if (metal_type[z - 1] > 0) {
                    if (metal_type[z - 1] == 2) ff = -0.1;
                    else if (metal_type[z - 1] == 1) ff = 0.3;
                }
            }
            c.m.alpeeq[i] = std::pow(ab + ff * c.m.qa[i], 2);
        }
        // dgam, amide H (eeq_solver.cpp:4389-4425)
        std::vector<char> pi = eeq_pi_atoms(c, c.m.hyb);
        std::vector<char> am = eeq_amide_n(c, c.m.hyb, pi);
        ah = eeq_amide_h(c, c.m.hyb, am);
        dgam = eeq_dgam(c, c.m.qa, pi, am);
    }
    c.m.chi_base.resize(n);
    c.m.gam.resize(n);
    c.m.cnf.resize(n);
    for (int i = 0; i < n; ++i) {
        const int z = c.Z[i];
        double chi = -chi_eeq[z - 1] + dxi[i];
        if (ah[i]) chi -= 0.02;
        c.m.chi_base[i] = chi;
        c.m.gam[i] = gam_eeq[z - 1] + dgam[i];
        c.m.cnf[i] = cnf_eeq[z - 1];
    }
    c.m.dxi = dxi;
    c.m.dgam = dgam;
    c.m.amide_h = ah;

    // pi-system charges (gfnff_method.cpp:9277-9339)
    std::vector<int> pis_charge;
    {
        std::set<int> ids;
        for (int f : c.m.pi_frag) if (f > 0) ids.insert(f);
        pis_charge.assign(ids.empty() ? 0 : (*ids.rbegin()) + 1, 0);
        auto qheavy = [&](const std::vector<double>& q) {
            std::vector<double> qh = q;
            for (int i = 0; i < n; ++i) {
                if (c.Z[i] != 1) continue;
                const int nn = (int)c.m.adj[i].size();
                if (nn == 0) continue;
                const double share = q[i] / (double)nn;
                for (int nb : c.m.adj[i]) qh[nb] += share;
                qh[i] = 0.0;
            }
            return qh;
        };
        std::vector<double> qah = qheavy(c.m.qa);
        for (int pis : ids) {
            int first = -1;
            for (int k = 0; k < n; ++k) if (c.m.pi_frag[k] == pis) { first = k; break; }
            const int f = c.m.frag[first];
            if (c.m.qfrag[f] == 0.0) continue;   // neutral solve equals the charged one
            std::vector<double> qf = c.m.qfrag;
            qf[f] = 0.0;
            bool okn;
            std::vector<double> qn = qheavy(phase1_charges(c, qf, dxi, &okn));
            double dum = 0.0;
            for (int k = 0; k < n; ++k) if (c.m.pi_frag[k] == pis) dum += qah[k] - qn[k];
            dum *= 1.1;
            pis_charge[pis] = (int)std::round(dum);
        }
    }
    huckel_bond_orders(c, pis_charge);

    // bond types per topology bond (:9376-9420)
    c.m.bond_type.resize(c.m.topo_bonds.size());
    for (size_t b = 0; b < c.m.topo_bonds.size(); ++b) {
        const int i = c.m.topo_bonds[b].first, j = c.m.topo_bonds[b].second;
        int hi = c.m.hyb[i], hj = c.m.hyb[j];
        if (hi == 3 && c.m.pi_frag[i] > 0) hi = 2;
        if (hj == 3 && c.m.pi_frag[j] > 0) hj = 2;
        int bt = classify_bond(c, i, j, hi, hj);
        if (bt == 3) {
            int bb = 3;
            if (hi == 0 || hj == 0 || hi == 3 || hj == 3) bb = 1;
            else if (hi == 2 || hj == 2) bb = 2;
            if (bb != 3 && pibo_of(c, i, j) > 0.1) bt = 2;
        }
        c.m.bond_type[b] = bt;
    }
    topo_distances(c);
}

}  // namespace detail
}  // namespace gfnff
