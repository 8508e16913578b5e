// Parameter file: the complete set-up result of one molecule (topology, parameters, term
// lists) as a versioned binary image, so that later runs on the same structure skip the
// set-up.  curcuma keeps the same idea as `<input>.param.json` (parameter caching of its
// force fields) and `<geom>.topo.json` (gfnff_method.cpp:2515-2811); this format is the
// library's own and is read only by the library build that wrote it (the record layouts
// are part of the header check).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "model.h"

namespace gfnff {
namespace {

constexpr char kMagic[8] = {'G', 'F', 'N', 'F', 'F', 'P', 'A', 'R'};
constexpr uint32_t kVersion = 1;

// record sizes in the header: a build whose term layouts differ refuses the file
uint32_t layout_hash()
{
    const uint32_t s[] = {sizeof(BondTerm), sizeof(AngleTerm), sizeof(TorsionTerm), sizeof(InversionTerm),
                          sizeof(STorsionTerm), sizeof(RepPair), sizeof(DispPair), sizeof(XBTerm),
                          sizeof(ATMTriple), sizeof(BATMTriple), sizeof(SetupOptions)};
    uint32_t h = 2166136261u;
    for (uint32_t v : s) h = (h ^ v) * 16777619u;
    return h;
}

struct Writer {
    FILE* f;
    void raw(const void* p, size_t n)
    {
        if (n && std::fwrite(p, 1, n, f) != n) throw std::runtime_error("parameter file: write failed");
    }
    template <class T>
    void val(const T& v)
    {
        static_assert(std::is_trivially_copyable<T>::value, "plain value");
        raw(&v, sizeof(T));
    }
    template <class T>
    void vec(const std::vector<T>& v)
    {
        static_assert(std::is_trivially_copyable<T>::value, "plain records");
        val<uint64_t>(v.size());
        raw(v.data(), v.size() * sizeof(T));
    }
    void vecvec(const std::vector<std::vector<int>>& v)
    {
        val<uint64_t>(v.size());
        for (auto& r : v) vec(r);
    }
    void pairs(const std::vector<std::pair<int, int>>& v)
    {
        std::vector<int> flat;
        flat.reserve(2 * v.size());
        for (auto& p : v) { flat.push_back(p.first); flat.push_back(p.second); }
        vec(flat);
    }
};

struct Reader {
    FILE* f;
    void raw(void* p, size_t n)
    {
        if (n && std::fread(p, 1, n, f) != n) throw std::runtime_error("parameter file: truncated");
    }
    template <class T>
    T val()
    {
        T v;
        raw(&v, sizeof(T));
        return v;
    }
    template <class T>
    void vec(std::vector<T>& v)
    {
        const uint64_t n = val<uint64_t>();
        if (n > (uint64_t(1) << 40) / sizeof(T)) throw std::runtime_error("parameter file: corrupt length");
        v.resize(n);
        raw(v.data(), n * sizeof(T));
    }
    void vecvec(std::vector<std::vector<int>>& v)
    {
        const uint64_t n = val<uint64_t>();
        if (n > (uint64_t(1) << 32)) throw std::runtime_error("parameter file: corrupt length");
        v.resize(n);
        for (auto& r : v) vec(r);
    }
    void pairs(std::vector<std::pair<int, int>>& v)
    {
        std::vector<int> flat;
        vec(flat);
        if (flat.size() % 2) throw std::runtime_error("parameter file: corrupt pair list");
        v.resize(flat.size() / 2);
        for (size_t k = 0; k < v.size(); ++k) v[k] = {flat[2 * k], flat[2 * k + 1]};
    }
};

// the fields in file order; the same function serves writing and reading
template <class IO>
void hb_terms(IO& io, std::vector<HBTerm>& hb);

template <>
void hb_terms(Writer& w, std::vector<HBTerm>& hb)
{
    w.val<uint64_t>(hb.size());
    for (auto& t : hb) {
        w.val(t.a); w.val(t.h); w.val(t.b); w.val(t.case_type);
        w.val(t.bas_a); w.val(t.bas_b); w.val(t.aci_a); w.val(t.aci_b);
        w.val(t.q_h); w.val(t.q_a); w.val(t.q_b); w.val(t.parent_c);
        w.vec(t.nb_b); w.vec(t.nb_c);
    }
}

template <>
void hb_terms(Reader& r, std::vector<HBTerm>& hb)
{
    const uint64_t n = r.val<uint64_t>();
    if (n > (uint64_t(1) << 34)) throw std::runtime_error("parameter file: corrupt length");
    hb.resize(n);
    for (auto& t : hb) {
        t.a = r.val<int>(); t.h = r.val<int>(); t.b = r.val<int>(); t.case_type = r.val<int>();
        t.bas_a = r.val<double>(); t.bas_b = r.val<double>(); t.aci_a = r.val<double>(); t.aci_b = r.val<double>();
        t.q_h = r.val<double>(); t.q_a = r.val<double>(); t.q_b = r.val<double>(); t.parent_c = r.val<int>();
        r.vec(t.nb_b); r.vec(t.nb_c);
    }
}

template <class IO>
void bond_hb(IO& io, std::vector<BondHB>& v);

template <>
void bond_hb(Writer& w, std::vector<BondHB>& v)
{
    w.val<uint64_t>(v.size());
    for (auto& t : v) { w.val(t.a); w.val(t.h); w.vec(t.b_atoms); }
}

template <>
void bond_hb(Reader& r, std::vector<BondHB>& v)
{
    const uint64_t n = r.val<uint64_t>();
    if (n > (uint64_t(1) << 34)) throw std::runtime_error("parameter file: corrupt length");
    v.resize(n);
    for (auto& t : v) { t.a = r.val<int>(); t.h = r.val<int>(); r.vec(t.b_atoms); }
}

template <class IO>
void body(IO& io, Model& m)
{
    io.vec(m.Z); io.vec(m.xyz_setup);
    io.vecvec(m.adj);
    io.vec(m.hyb); io.vec(m.pi_frag); io.vec(m.ring_size); io.vec(m.frag);
    io.vec(m.cn_setup); io.vec(m.qa); io.vec(m.qfrag); io.vec(m.bond_type); io.pairs(m.topo_bonds);
    io.vec(m.rcov_cn); io.vec(m.rcov_d3); io.vec(m.rvdw); io.vec(m.chi_base); io.vec(m.cnf); io.vec(m.gam);
    io.vec(m.alpeeq);
    io.vec(m.present_Z); io.vec(m.slot); io.vec(m.nref); io.vec(m.refcn); io.vec(m.c6ref); io.vec(m.w_setup);
    io.vec(m.zeta); io.vec(m.sqrt_zr4r2);
    io.vec(m.bonds); io.vec(m.angles); io.vec(m.torsions); io.vec(m.inversions); io.vec(m.storsions);
    io.vec(m.rep_bonded); io.vec(m.rep_nonbonded); io.vec(m.disp);
    hb_terms(io, m.hbonds);
    io.vec(m.xbonds); io.vec(m.atm); io.vec(m.batm);
    bond_hb(io, m.bond_hb);
}

}  // namespace

void save_parameters(const Model& m, const char* path)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) throw std::runtime_error(std::string("parameter file: cannot create ") + path);
    try {
        Writer w{f};
        w.raw(kMagic, sizeof(kMagic));
        w.val(kVersion); w.val(layout_hash());
        w.val(m.n); w.val(m.nfrag); w.val(m.charge); w.val(m.n_primary_torsions); w.val(m.e0);
        w.val<int>(m.nonbonded_rep_all_pairs ? 1 : 0);
        w.val(m.opt);
        body(w, const_cast<Model&>(m));   // body() only reads the model when writing
        if (std::fclose(f) != 0) throw std::runtime_error("parameter file: write failed");
    } catch (...) {
        std::fclose(f);
        std::remove(path);
        throw;
    }
}

Model load_parameters(const char* path)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("parameter file: cannot open ") + path);
    Model m;
    try {
        Reader r{f};
        char magic[8];
        r.raw(magic, sizeof(magic));
        if (std::memcmp(magic, kMagic, sizeof(kMagic)) != 0) throw std::runtime_error("not a parameter file");
        if (r.val<uint32_t>() != kVersion) throw std::runtime_error("parameter file: unsupported version");
        if (r.val<uint32_t>() != layout_hash()) throw std::runtime_error("parameter file: written by another build");
        m.n = r.val<int>(); m.nfrag = r.val<int>(); m.charge = r.val<int>(); m.n_primary_torsions = r.val<int>();
        m.e0 = r.val<double>();
        m.nonbonded_rep_all_pairs = r.val<int>() != 0;
        m.opt = r.val<SetupOptions>();
        body(r, m);
        if (std::fgetc(f) != EOF) throw std::runtime_error("parameter file: trailing data");
        std::fclose(f);
    } catch (...) {
        std::fclose(f);
        throw;
    }
    const size_t n = (size_t)m.n;
    if (m.n <= 0 || m.Z.size() != n || m.xyz_setup.size() != 3 * n || m.frag.size() != n || m.qa.size() != n ||
        m.slot.size() != n || m.nfrag <= 0)
        throw std::runtime_error("parameter file: inconsistent sizes");
    return m;
}

}  // namespace gfnff
