// Internal state shared by the setup translation units.
#pragma once

#include <cstdint>
#include <functional>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../tables/gfnff_tables.inc"
#include "linalg.h"
#include "model.h"

namespace gfnff {
namespace detail {

inline uint64_t key(int i, int j)
{
    if (i > j) std::swap(i, j);
    return ((uint64_t)(uint32_t)i << 32) | (uint32_t)j;
}

struct Ctx {
    Model& m;
    int n;
    const int* Z;
    std::vector<double> xb;    // bohr
    std::vector<double> xa;    // Angstrom (the few Angstrom-based geometric tests)
    std::vector<double> rcov_cn;
    std::vector<char> is_metal;
    std::unordered_set<uint64_t> bondset;                     // topology bonds
    std::vector<std::vector<int>> rings;                      // sorted atom sets
    std::vector<std::vector<int>> atom_rings;
    std::vector<std::vector<std::pair<int, int>>> tdist;      // (atom, bond count <= 5)
    std::unordered_map<uint64_t, double> pibo;                // pi bond orders of bonds
    const char* topo_cache = nullptr;                         // <geometry>.topo.json to consult
    explicit Ctx(Model& mm) : m(mm), n(mm.n), Z(mm.Z.data()) {}
    bool bonded(int i, int j) const { return bondset.count(key(i, j)) != 0; }
};

double dist_bohr(const Ctx& c, int i, int j);
double dist2_bohr(const Ctx& c, int i, int j);
void pairs_within(const Ctx& c, double rcut, bool strict,
                  const std::function<void(int, int, double)>& fn);
// The same pairs with the rows i split into contiguous ranges over the OpenMP threads
// (static schedule): fn(t, i, j, d2) runs on thread t (0 <= t < setup_threads()), and each
// thread sees its rows in ascending order, so per-thread collections concatenated in thread
// order are ordered by i.  fn must be safe to call concurrently for different t.
int setup_threads();
void pairs_within_rows(const Ctx& c, double rcut, bool strict,
                       const std::function<void(int, int, int, double)>& fn);
std::vector<double> cn_threshold(const Ctx& c, double threshold);
void compute_topology(Ctx& c);
int same_ring_size(const Ctx& c, int i, int j);
int smallest_ring_all(const Ctx& c, int i, int j, int k, int l);
int largest_ring_all(const Ctx& c, int i, int j, int k, int l);
int smallest_ring_bend(const Ctx& c, int i, int j, int k);
int topo_dist(const Ctx& c, int i, int j);
double pibo_of(const Ctx& c, int i, int j);

void generate_parameters(Ctx& c);
void detect_hbxb(Ctx& c, const std::vector<double>& xbohr);

}  // namespace detail
}  // namespace gfnff
