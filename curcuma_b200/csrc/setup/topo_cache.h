// Topology cache in curcuma's `<geometry>.topo.json` format (ff_methods/gfnff_method.cpp:
// 2515-2656 computeTopologyFingerprint / exportTopology, 2941-2985 the write after the
// set-up, 8973-9040 the read before Phase 1).
//
// The file is a JSON object.  On a set-up whose fingerprint (atom count, elements and the
// geometric bond list, hashed with std::hash<std::string> and written as a decimal string)
// equals the file's, the Phase-1 results are taken from it instead of being recomputed:
// topology_charges, qfrag, dxi, dgam, alpeeq and is_amide_h, the keys curcuma's cache-hit
// path reads.  The other keys (fraglist, coordination_numbers, hybridization, ring_sizes,
// pi_fragments, is_aromatic, is_metal, rings, nfrag, version, timestamp) are written for
// curcuma's exporter's layout and not read back, as in curcuma.  The fingerprint matches
// curcuma's when both sides use libstdc++'s std::hash.
#pragma once

#include <string>
#include <vector>

#include "model.h"

namespace gfnff {

// the Phase-1 data of a cache hit
struct TopoCache {
    std::vector<double> qa, qfrag, dxi, dgam, alpeeq;
    std::vector<char> amide_h;
    bool has_qfrag = false, has_amide_h = false;
};

// `<geometry file without its last extension>.topo.json` (gfnff_method.cpp:2967-2969)
std::string topology_cache_path(const std::string& geometry_file);

// curcuma's fingerprint string: "N=<n>|Z=z0,z1,...|B=i-j,..." hashed (gfnff_method.cpp:2515-2533)
std::string topology_fingerprint(const std::vector<int>& Z, const std::vector<std::pair<int, int>>& bonds);

// Reads `path`; true on a usable hit: the file parses, carries this fingerprint and the
// Phase-1 vectors have n entries (a cache that lacks one of them is treated as a miss and
// the set-up recomputes Phase 1).  A missing or unreadable file is a miss, never an error.
bool read_topology_cache(const std::string& path, const std::string& fingerprint, int n, TopoCache& out);

// Writes the cache of a completed set-up (topology, Phase-1 data and the fingerprint).
// Skipped, returning false, when the Phase-1 charges are unphysical: not finite, their sum
// more than 1 e from the molecular charge, or the fragment charges more than 0.5 e from it
// (the write guard of gfnff_method.cpp:2941-2963).  Throws std::runtime_error when the
// file cannot be written.
bool write_topology_cache(const std::string& path, const Model& m);

}  // namespace gfnff
