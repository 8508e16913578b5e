// Topology cache in curcuma's `<geometry>.topo.json` format: fingerprint, JSON writer and a
// small JSON reader (objects, arrays, numbers, strings, literals) for the keys the cache-hit
// path consumes.
#include "topo_cache.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <stdexcept>

#include "../tables/gfnff_tables.inc"

namespace gfnff {

namespace {

// ---- reader ---------------------------------------------------------------------------
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    const JVal* get(const char* k) const
    {
        for (const auto& kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class Reader {
public:
    explicit Reader(const std::string& s) : s_(s) {}
    bool parse(JVal& v)
    {
        if (!value(v, 0)) return false;
        ws();
        return p_ == s_.size();
    }

private:
    const std::string& s_;
    size_t p_ = 0;
    void ws()
    {
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) ++p_;
    }
    bool lit(const char* w)
    {
        const size_t l = std::strlen(w);
        if (s_.compare(p_, l, w) != 0) return false;
        p_ += l;
        return true;
    }
    bool string(std::string& out)
    {
        if (p_ >= s_.size() || s_[p_] != '"') return false;
        ++p_;
        out.clear();
        while (p_ < s_.size()) {
            const char ch = s_[p_++];
            if (ch == '"') return true;
            if (ch != '\\') { out.push_back(ch); continue; }
            if (p_ >= s_.size()) return false;
            const char e = s_[p_++];
            switch (e) {
                case '"': case '\\': case '/': out.push_back(e); break;
                case 'b': out.push_back('\b'); break;
                case 'f': out.push_back('\f'); break;
                case 'n': out.push_back('\n'); break;
                case 'r': out.push_back('\r'); break;
                case 't': out.push_back('\t'); break;
                case 'u': {
                    if (p_ + 4 > s_.size()) return false;
                    unsigned cp = (unsigned)std::strtoul(s_.substr(p_, 4).c_str(), nullptr, 16);
                    p_ += 4;
                    // code points of the basic plane as UTF-8 (no key of the cache needs more)
                    if (cp < 0x80) out.push_back((char)cp);
                    else if (cp < 0x800) { out.push_back((char)(0xC0 | (cp >> 6))); out.push_back((char)(0x80 | (cp & 0x3F))); }
                    else {
                        out.push_back((char)(0xE0 | (cp >> 12)));
                        out.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
                        out.push_back((char)(0x80 | (cp & 0x3F)));
                    }
                    break;
                }
                default: return false;
            }
        }
        return false;
    }
    bool value(JVal& v, int depth)
    {
        if (depth > 64) return false;
        ws();
        if (p_ >= s_.size()) return false;
        const char ch = s_[p_];
        if (ch == '{') {
            ++p_;
            v.kind = JVal::Obj;
            ws();
            if (p_ < s_.size() && s_[p_] == '}') { ++p_; return true; }
            while (true) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (p_ >= s_.size() || s_[p_] != ':') return false;
                ++p_;
                v.obj.emplace_back(std::move(k), JVal());
                if (!value(v.obj.back().second, depth + 1)) return false;
                ws();
                if (p_ < s_.size() && s_[p_] == ',') { ++p_; continue; }
                if (p_ < s_.size() && s_[p_] == '}') { ++p_; return true; }
                return false;
            }
        }
        if (ch == '[') {
            ++p_;
            v.kind = JVal::Arr;
            ws();
            if (p_ < s_.size() && s_[p_] == ']') { ++p_; return true; }
            while (true) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), depth + 1)) return false;
                ws();
                if (p_ < s_.size() && s_[p_] == ',') { ++p_; continue; }
                if (p_ < s_.size() && s_[p_] == ']') { ++p_; return true; }
                return false;
            }
        }
        if (ch == '"') { v.kind = JVal::Str; return string(v.str); }
        if (lit("true")) { v.kind = JVal::Bool; v.num = 1.0; return true; }
        if (lit("false")) { v.kind = JVal::Bool; v.num = 0.0; return true; }
        if (lit("null")) { v.kind = JVal::Null; return true; }
        const char* b = s_.c_str() + p_;
        char* e = nullptr;
        v.num = std::strtod(b, &e);
        if (e == b) return false;
        v.kind = JVal::Num;
        p_ += (size_t)(e - b);
        return true;
    }
};

bool numbers(const JVal* v, int n, std::vector<double>& out)
{
    if (!v || v->kind != JVal::Arr || (int)v->arr.size() != n) return false;
    out.resize(n);
    for (int i = 0; i < n; ++i) {
        const JVal& e = v->arr[i];
        if (e.kind != JVal::Num && e.kind != JVal::Bool) return false;
        out[i] = e.num;
    }
    return true;
}

// ---- writer ---------------------------------------------------------------------------
void put_num(std::ostream& o, double x)
{
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", x);
    o << buf;
}

template <class T, class F>
void put_array(std::ostream& o, const char* key, const std::vector<T>& v, F&& fmt, bool last = false)
{
    o << "  \"" << key << "\": [";
    for (size_t i = 0; i < v.size(); ++i) {
        if (i) o << ", ";
        fmt(o, v[i]);
    }
    o << "]" << (last ? "\n" : ",\n");
}

}  // namespace

std::string topology_cache_path(const std::string& geometry_file)
{
    const size_t dot = geometry_file.find_last_of('.');
    return (dot != std::string::npos ? geometry_file.substr(0, dot) : geometry_file) + ".topo.json";
}

std::string topology_fingerprint(const std::vector<int>& Z, const std::vector<std::pair<int, int>>& bonds)
{
    std::string s = "N=" + std::to_string(Z.size()) + "|Z=";
    for (size_t i = 0; i < Z.size(); ++i) {
        if (i) s += ',';
        s += std::to_string(Z[i]);
    }
    s += "|B=";
    for (size_t b = 0; b < bonds.size(); ++b) {
        if (b) s += ',';
        s += std::to_string(bonds[b].first) + "-" + std::to_string(bonds[b].second);
    }
    return std::to_string(std::hash<std::string>{}(s));
}

bool read_topology_cache(const std::string& path, const std::string& fingerprint, int n, TopoCache& out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    JVal root;
    if (!Reader(text).parse(root) || root.kind != JVal::Obj) return false;
    const JVal* fp = root.get("fingerprint");
    if (!fp || fp->kind != JVal::Str || fp->str != fingerprint) return false;
    TopoCache c;
    if (!numbers(root.get("topology_charges"), n, c.qa)) return false;
    if (!numbers(root.get("dxi"), n, c.dxi)) return false;
    if (!numbers(root.get("dgam"), n, c.dgam)) return false;
    if (!numbers(root.get("alpeeq"), n, c.alpeeq)) return false;
    if (const JVal* q = root.get("qfrag")) {
        if (q->kind != JVal::Arr) return false;
        if (!numbers(q, (int)q->arr.size(), c.qfrag)) return false;
        c.has_qfrag = true;
    }
    if (const JVal* a = root.get("is_amide_h")) {
        std::vector<double> fl;
        if (!numbers(a, n, fl)) return false;
        c.amide_h.resize(n);
        for (int i = 0; i < n; ++i) c.amide_h[i] = fl[i] != 0.0;
        c.has_amide_h = true;
    }
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(c.qa[i]) || !std::isfinite(c.dxi[i]) || !std::isfinite(c.dgam[i]) ||
            !std::isfinite(c.alpeeq[i]))
            return false;
    out = std::move(c);
    return true;
}

bool write_topology_cache(const std::string& path, const Model& m)
{
    const int n = m.n;
    if ((int)m.qa.size() != n || (int)m.dxi.size() != n || (int)m.dgam.size() != n) return false;
    double qs = 0.0, fs = 0.0;
    for (double q : m.qa) {
        if (!std::isfinite(q)) return false;
        qs += q;
    }
    for (double q : m.qfrag) fs += q;
    if (std::fabs(qs - m.charge) >= 1.0) return false;
    if (!m.qfrag.empty() && std::fabs(fs - m.charge) >= 0.5) return false;

    std::ostringstream o;
    auto num = [](std::ostream& s, double x) { put_num(s, x); };
    auto intf = [](std::ostream& s, int x) { s << x; };
    o << "{\n  \"version\": 1,\n  \"nfrag\": " << m.nfrag << ",\n";
    std::vector<int> fl(n), metal(n), arom(n, 0), amide(n);
    for (int i = 0; i < n; ++i) {
        fl[i] = m.frag[i] + 1;   // curcuma numbers fragments from 1
        const int z = m.Z[i];
        metal[i] = (z >= 1 && z <= 86 && gfnff_tables::metal_type[z - 1] > 0) ? 1 : 0;
        amide[i] = (i < (int)m.amide_h.size() && m.amide_h[i]) ? 1 : 0;
    }
    put_array(o, "fraglist", fl, intf);
    put_array(o, "qfrag", m.qfrag, num);
    put_array(o, "topology_charges", m.qa, num);
    put_array(o, "coordination_numbers", m.cn_setup, num);
    put_array(o, "hybridization", m.hyb, intf);
    put_array(o, "ring_sizes", m.ring_size, intf);
    put_array(o, "pi_fragments", m.pi_frag, intf);
    put_array(o, "is_aromatic", arom, intf);   // curcuma's set-up leaves every flag false
    put_array(o, "is_metal", metal, intf);
    o << "  \"rings\": [";
    for (size_t r = 0; r < m.rings.size(); ++r) {
        o << (r ? ", [" : "[");
        for (size_t k = 0; k < m.rings[r].size(); ++k) o << (k ? ", " : "") << m.rings[r][k];
        o << "]";
    }
    o << "],\n";
    put_array(o, "is_amide_h", amide, intf);
    put_array(o, "dxi", m.dxi, num);
    put_array(o, "alpeeq", m.alpeeq, num);
    put_array(o, "dgam", m.dgam, num);
    o << "  \"timestamp\": " << (long long)std::chrono::system_clock::now().time_since_epoch().count() << ",\n";
    o << "  \"fingerprint\": \"" << topology_fingerprint(m.Z, m.topo_bonds) << "\"\n}\n";

    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) throw std::runtime_error("topology cache: cannot write " + path);
    f << o.str();
    f.close();
    if (!f.good()) throw std::runtime_error("topology cache: cannot write " + path);
    return true;
}

}  // namespace gfnff
