// pdf_files.cpp -- netlist and vector files, and the text dumps of the
// reference's debug logs.
//
// The reference reads circuits with Circuit::read_bench / Circuit::load and
// vectors with get_vector_dim / read_vectors (main.cu:128-156), all in its
// util/ submodule, which is not part of the reference snapshot.  The formats
// here are therefore this library's own:
//
//  * ISCAS .bench: `INPUT(n)`, `OUTPUT(n)`, `n = TYPE(a, b, ...)`, `#`
//    comments.  Flip-flops are cut for full scan: the output of `q = DFF(d)`
//    becomes a primary input and d a primary output.  Levels are the longest
//    distance from an input; within a level, gates keep file order.
//  * levelized text (`pdf-level 1`): one line per gate in id order,
//    `id level TYPE po nfi fan-ins... nfo fan-outs...`; round-trips every
//    field of a pdf_netlist, fan-out order included.
//  * vectors: one vector per line, one 0/1 character per primary input
//    (whitespace ignored, `#` comments).
//
// The dumps follow the text layout of debugSimulationOutput
// (simkernel.cuh:250-295), debugMarkOutput (markkernel.cuh:357-394) and
// debugMergeOutput (mergekernel.cuh:269-284).
#include <algorithm>
#include <cctype>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <new>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "pdf.h"
#include "pdf_internal.h"

namespace {

void put_msg(char *msg, size_t len, const char *fmt, ...) {
    if (!msg || !len) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, len, fmt, ap);
    va_end(ap);
}

const char *kTypeNames[PDF_NTYPES] = {"UNKN", "INPT", "AND", "NAND", "OR",   "NOR",
                                      "XOR",  "XNOR", "BUFF", "NOT", "FROM", "DFF"};

int type_code(std::string s) {
    for (auto &ch : s) ch = (char)std::toupper((unsigned char)ch);
    if (s == "BUF") return PDF_BUFF;
    if (s == "INPUT") return PDF_INPT;
    for (int t = 0; t < PDF_NTYPES; t++)
        if (s == kTypeNames[t]) return t;
    return -1;
}

std::string trim(const std::string &s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) a++;
    while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

std::string strip_comment(const std::string &s) {
    const size_t h = s.find('#');
    return h == std::string::npos ? s : s.substr(0, h);
}

// A netlist given as gates with fan-in lists (any order); levelizes it, orders
// gates by (level, input order) and builds the edge array with fan-outs as the
// transpose ordered by consumer id and fan-in position.
struct RawGate {
    int type;
    uint8_t po;
    std::vector<uint32_t> fin;
};

pdf_status build_levelized(const std::vector<RawGate> &raw, pdf_netbuf **out, char *msg, size_t len) {
    const uint32_t n = (uint32_t)raw.size();
    if (n == 0) {
        put_msg(msg, len, "no gates");
        return PDF_EINVAL;
    }
    std::vector<uint32_t> level(n, 0), indeg(n, 0), order;
    std::vector<std::vector<uint32_t>> users(n);
    for (uint32_t g = 0; g < n; g++)
        for (uint32_t f : raw[g].fin) {
            users[f].push_back(g);
            indeg[g]++;
        }
    // Kahn's algorithm: a gate's level is 1 + the highest level of its fan-ins
    order.reserve(n);
    for (uint32_t g = 0; g < n; g++)
        if (indeg[g] == 0) order.push_back(g);
    for (size_t k = 0; k < order.size(); k++) {
        const uint32_t g = order[k];
        for (uint32_t u : users[g]) {
            level[u] = std::max(level[u], level[g] + 1);
            if (--indeg[u] == 0) order.push_back(u);
        }
    }
    if (order.size() != n) {
        put_msg(msg, len, "combinational loop (%u gates on or after a cycle)", n - (uint32_t)order.size());
        return PDF_EINVAL;
    }
    for (uint32_t g = 0; g < n; g++)
        if ((raw[g].type == PDF_INPT) != (level[g] == 0)) {
            put_msg(msg, len, "gate %u: a gate without fan-ins that is not an input", g);
            return PDF_EINVAL;
        }
    uint32_t L = 0;
    for (uint32_t g = 0; g < n; g++) L = std::max(L, level[g] + 1);
    // new id: by level, then by input order (stable)
    std::vector<uint32_t> perm(n), id(n);
    for (uint32_t g = 0; g < n; g++) perm[g] = g;
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return level[a] < level[b]; });
    for (uint32_t k = 0; k < n; k++) id[perm[k]] = k;

    pdf_netbuf *b = new (std::nothrow) pdf_netbuf();
    if (!b) return PDF_ENOMEM;
    try {
        b->n_gates = n;
        b->n_levels = L;
        b->level_offsets.assign(L + 1, 0);
        for (uint32_t g = 0; g < n; g++) b->level_offsets[level[g] + 1]++;
        for (uint32_t l = 0; l < L; l++) b->level_offsets[l + 1] += b->level_offsets[l];
        b->type.resize(n);
        b->po.resize(n);
        b->nfi.resize(n);
        b->nfo.assign(n, 0);
        b->edge_offset.resize(n);
        std::vector<std::vector<uint32_t>> fo(n);
        for (uint32_t k = 0; k < n; k++) {
            const RawGate &r = raw[perm[k]];
            b->type[k] = (uint8_t)r.type;
            b->po[k] = r.po;
            b->nfi[k] = (uint32_t)r.fin.size();
            for (uint32_t f : r.fin) fo[id[f]].push_back(k);
        }
        uint64_t e = 0;
        for (uint32_t k = 0; k < n; k++) {
            b->nfo[k] = (uint32_t)fo[k].size();
            b->edge_offset[k] = e;
            e += b->nfi[k] + b->nfo[k];
        }
        b->edges.resize(e);
        for (uint32_t k = 0; k < n; k++) {
            uint64_t o = b->edge_offset[k];
            for (uint32_t f : raw[perm[k]].fin) b->edges[o++] = id[f];
            for (uint32_t u : fo[k]) b->edges[o++] = u;
        }
    } catch (const std::bad_alloc &) {
        delete b;
        return PDF_ENOMEM;
    }
    pdf_netlist view;
    pdf_netbuf_view(b, &view);
    const pdf_status st = pdf_netlist_check(&view, msg, len);
    if (st != PDF_OK) {
        delete b;
        return st;
    }
    *out = b;
    return PDF_OK;
}

// `name = TYPE(args)` or `KEY(name)`; returns false on a malformed line.
bool split_call(const std::string &s, std::string &head, std::vector<std::string> &args) {
    const size_t l = s.find('('), r = s.rfind(')');
    if (l == std::string::npos || r == std::string::npos || r < l || !trim(s.substr(r + 1)).empty()) return false;
    head = trim(s.substr(0, l));
    args.clear();
    std::string inner = s.substr(l + 1, r - l - 1), cur;
    std::stringstream ss(inner);
    while (std::getline(ss, cur, ',')) args.push_back(trim(cur));
    if (args.size() == 1 && args[0].empty()) args.clear();
    for (auto &a : args)
        if (a.empty()) return false;
    // getline drops an empty last field ("a,"): every comma must separate two
    if (!args.empty() && (size_t)std::count(inner.begin(), inner.end(), ',') + 1 != args.size()) return false;
    return !head.empty();
}

}  // namespace

extern "C" pdf_status pdf_read_bench(const char *path, uint32_t flags, pdf_netbuf **out, char *msg,
                                     size_t msg_len) {
    if (!path || !out || (flags & ~(uint32_t)PDF_BENCH_BRANCHES)) return PDF_EINVAL;
    *out = nullptr;
    std::ifstream in(path);
    if (!in) {
        put_msg(msg, msg_len, "cannot open %s", path);
        return PDF_EINVAL;
    }
    struct Def {
        int type;
        std::vector<std::string> args;
        uint64_t line;
    };
    std::vector<std::string> names;                // net names in first-definition order
    std::unordered_map<std::string, uint32_t> net;  // name -> index into names / defs
    std::vector<Def> defs;
    std::vector<uint8_t> is_out;
    std::vector<uint64_t> out_line;
    auto intern = [&](const std::string &nm) {
        auto it = net.find(nm);
        if (it != net.end()) return it->second;
        const uint32_t k = (uint32_t)names.size();
        net.emplace(nm, k);
        names.push_back(nm);
        defs.push_back({-1, {}, 0});
        is_out.push_back(0);
        out_line.push_back(0);
        return k;
    };
    std::string line;
    uint64_t ln = 0;
    try {
        while (std::getline(in, line)) {
            ln++;
            const std::string s = trim(strip_comment(line));
            if (s.empty()) continue;
            std::string head;
            std::vector<std::string> args;
            const size_t eq = s.find('=');
            if (eq == std::string::npos) {
                if (!split_call(s, head, args) || args.size() != 1) {
                    put_msg(msg, msg_len, "%s:%llu: expected INPUT(name) or OUTPUT(name)", path,
                            (unsigned long long)ln);
                    return PDF_EINVAL;
                }
                std::string key = head;
                for (auto &ch : key) ch = (char)std::toupper((unsigned char)ch);
                const uint32_t k = intern(args[0]);
                if (key == "INPUT") {
                    if (defs[k].type != -1) {
                        put_msg(msg, msg_len, "%s:%llu: %s defined twice", path, (unsigned long long)ln,
                                args[0].c_str());
                        return PDF_EINVAL;
                    }
                    defs[k] = {PDF_INPT, {}, ln};
                } else if (key == "OUTPUT") {
                    is_out[k] = 1;
                    if (!out_line[k]) out_line[k] = ln;
                } else {
                    put_msg(msg, msg_len, "%s:%llu: unknown keyword %s", path, (unsigned long long)ln, head.c_str());
                    return PDF_EINVAL;
                }
                continue;
            }
            const std::string lhs = trim(s.substr(0, eq));
            if (lhs.empty() || !split_call(s.substr(eq + 1), head, args)) {
                put_msg(msg, msg_len, "%s:%llu: expected name = TYPE(inputs)", path, (unsigned long long)ln);
                return PDF_EINVAL;
            }
            const int t = type_code(head);
            if (t < 0 || t == PDF_INPT || t == PDF_UNKN) {
                put_msg(msg, msg_len, "%s:%llu: unknown gate type %s", path, (unsigned long long)ln, head.c_str());
                return PDF_EINVAL;
            }
            const bool one = t == PDF_NOT || t == PDF_BUFF || t == PDF_FROM || t == PDF_DFF;
            if (args.empty() || args.size() > 255 || (one && args.size() != 1)) {
                put_msg(msg, msg_len, "%s:%llu: %s takes %s inputs, got %zu", path, (unsigned long long)ln,
                        head.c_str(), one ? "exactly 1" : "1 to 255", args.size());
                return PDF_EINVAL;
            }
            const uint32_t k = intern(lhs);
            if (defs[k].type != -1) {
                put_msg(msg, msg_len, "%s:%llu: %s defined twice", path, (unsigned long long)ln, lhs.c_str());
                return PDF_EINVAL;
            }
            for (const auto &a : args) intern(a);
            defs[k] = {t, args, ln};
        }
        for (uint32_t k = 0; k < names.size(); k++)
            if (defs[k].type == -1) {
                put_msg(msg, msg_len, "%s: net %s is used but never defined", path, names[k].c_str());
                return PDF_EINVAL;
            }
        // gates: inputs first (file order), then flip-flop outputs cut for
        // full scan, then the rest; the order only breaks ties within a level
        std::vector<uint32_t> gate_of(names.size());
        std::vector<RawGate> raw;
        raw.reserve(names.size());
        std::vector<uint32_t> seq(names.size());
        for (uint32_t k = 0; k < names.size(); k++) seq[k] = k;
        auto rank = [&](uint32_t k) { return defs[k].type == PDF_INPT ? 0 : defs[k].type == PDF_DFF ? 1 : 2; };
        std::stable_sort(seq.begin(), seq.end(), [&](uint32_t a, uint32_t b) {
            if (rank(a) != rank(b)) return rank(a) < rank(b);
            return defs[a].line < defs[b].line;
        });
        std::vector<uint8_t> pseudo_po(names.size(), 0);
        for (uint32_t k : seq) {
            gate_of[k] = (uint32_t)raw.size();
            raw.push_back({defs[k].type == PDF_DFF ? PDF_INPT : defs[k].type, is_out[k], {}});
            if (defs[k].type == PDF_DFF) pseudo_po[net[defs[k].args[0]]] = 1;
        }
        for (uint32_t k = 0; k < names.size(); k++) {
            RawGate &r = raw[gate_of[k]];
            if (pseudo_po[k]) r.po = 1;
            if (defs[k].type == PDF_DFF || defs[k].type == PDF_INPT) continue;
            for (const auto &a : defs[k].args) r.fin.push_back(gate_of[net[a]]);
        }
        if (flags & PDF_BENCH_BRANCHES) {
            // a FROM gate per fan-out branch of every stem read more than once
            std::vector<uint32_t> reads(raw.size(), 0);
            for (const auto &r : raw)
                for (uint32_t f : r.fin) reads[f]++;
            const uint32_t n0 = (uint32_t)raw.size();
            for (uint32_t g = 0; g < n0; g++)
                for (uint32_t j = 0; j < raw[g].fin.size(); j++) {
                    const uint32_t f = raw[g].fin[j];
                    if (reads[f] < 2) continue;
                    raw[g].fin[j] = (uint32_t)raw.size();
                    raw.push_back({PDF_FROM, 0, {f}});
                }
        }
        if (raw.size() >= 0x7FFFFFFFull) return PDF_ENOTSUP;
        return build_levelized(raw, out, msg, msg_len);
    } catch (const std::bad_alloc &) {
        return PDF_ENOMEM;
    }
}

extern "C" pdf_status pdf_write_bench(const pdf_netlist *nl, const char *path) {
    if (!nl || !path) return PDF_EINVAL;
    pdf_status st = pdf_netlist_check(nl, nullptr, 0);
    if (st != PDF_OK) return st;
    std::ofstream o(path);
    if (!o) return PDF_EINVAL;
    const uint32_t G = nl->n_gates, npi = nl->level_offsets[1];
    o << "# " << G << " gates, " << nl->n_levels << " levels\n";
    for (uint32_t g = 0; g < npi; g++) o << "INPUT(g" << g << ")\n";
    for (uint32_t g = 0; g < G; g++)
        if (nl->po[g]) o << "OUTPUT(g" << g << ")\n";
    for (uint32_t g = npi; g < G; g++) {
        o << "g" << g << " = " << kTypeNames[nl->type[g]] << "(";
        for (uint32_t j = 0; j < nl->nfi[g]; j++) o << (j ? ", " : "") << "g" << nl->edges[nl->edge_offset[g] + j];
        o << ")\n";
    }
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_write_level(const pdf_netlist *nl, const char *path) {
    if (!nl || !path) return PDF_EINVAL;
    pdf_status st = pdf_netlist_check(nl, nullptr, 0);
    if (st != PDF_OK) return st;
    std::ofstream o(path);
    if (!o) return PDF_EINVAL;
    o << "pdf-level 1\n" << nl->n_gates << " " << nl->n_levels << "\n";
    for (uint32_t l = 0; l < nl->n_levels; l++)
        for (uint32_t g = nl->level_offsets[l]; g < nl->level_offsets[l + 1]; g++) {
            const uint64_t e = nl->edge_offset[g];
            o << g << " " << l << " " << kTypeNames[nl->type[g]] << " " << (int)nl->po[g] << " " << nl->nfi[g];
            for (uint32_t j = 0; j < nl->nfi[g]; j++) o << " " << nl->edges[e + j];
            o << " " << nl->nfo[g];
            for (uint32_t k = 0; k < nl->nfo[g]; k++) o << " " << nl->edges[e + nl->nfi[g] + k];
            o << "\n";
        }
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_read_level(const char *path, pdf_netbuf **out, char *msg, size_t msg_len) {
    if (!path || !out) return PDF_EINVAL;
    *out = nullptr;
    std::ifstream in(path);
    if (!in) {
        put_msg(msg, msg_len, "cannot open %s", path);
        return PDF_EINVAL;
    }
    std::string line;
    uint64_t ln = 0;
    auto next_line = [&](std::string &s) {
        while (std::getline(in, line)) {
            ln++;
            s = trim(strip_comment(line));
            if (!s.empty()) return true;
        }
        return false;
    };
    auto fail = [&](const char *what) {
        put_msg(msg, msg_len, "%s:%llu: %s", path, (unsigned long long)ln, what);
        return PDF_EINVAL;
    };
    std::string s;
    if (!next_line(s) || s != "pdf-level 1") return fail("expected the header 'pdf-level 1'");
    unsigned long long G = 0, L = 0;
    if (!next_line(s)) return fail("expected 'n_gates n_levels'");
    {
        std::istringstream ss(s);
        std::string extra;
        if (!(ss >> G >> L) || (ss >> extra) || G == 0 || L == 0 || G >= 0x7FFFFFFFull || L > G)
            return fail("expected 'n_gates n_levels'");
    }
    pdf_netbuf *b = new (std::nothrow) pdf_netbuf();
    if (!b) return PDF_ENOMEM;
    try {
        b->n_gates = (uint32_t)G;
        b->n_levels = (uint32_t)L;
        b->level_offsets.assign(L + 1, 0);
        b->type.resize(G);
        b->po.resize(G);
        b->nfi.resize(G);
        b->nfo.resize(G);
        b->edge_offset.resize(G);
        uint32_t prev_level = 0;
        for (unsigned long long g = 0; g < G; g++) {
            if (!next_line(s)) {
                delete b;
                return fail("fewer gate lines than n_gates");
            }
            std::istringstream ss(s);
            unsigned long long id, lvl, nfi, nfo, po;
            std::string tname, extra;
            if (!(ss >> id >> lvl >> tname >> po >> nfi) || id != g || lvl >= L || lvl < prev_level || po > 1 ||
                nfi > 255 || type_code(tname) < 0) {
                delete b;
                return fail("bad gate line (id level TYPE po nfi fan-ins... nfo fan-outs...)");
            }
            prev_level = (uint32_t)lvl;
            b->level_offsets[lvl + 1]++;
            b->type[g] = (uint8_t)type_code(tname);
            b->po[g] = (uint8_t)po;
            b->nfi[g] = (uint32_t)nfi;
            b->edge_offset[g] = b->edges.size();
            for (unsigned long long j = 0; j < nfi; j++) {
                unsigned long long f;
                if (!(ss >> f) || f >= G) {
                    delete b;
                    return fail("bad fan-in id");
                }
                b->edges.push_back((uint32_t)f);
            }
            if (!(ss >> nfo) || nfo >= 0xFFFFFFFFull) {
                delete b;
                return fail("missing fan-out count");
            }
            b->nfo[g] = (uint32_t)nfo;
            for (unsigned long long k = 0; k < nfo; k++) {
                unsigned long long f;
                if (!(ss >> f) || f >= G) {
                    delete b;
                    return fail("bad fan-out id");
                }
                b->edges.push_back((uint32_t)f);
            }
            if (ss >> extra) {
                delete b;
                return fail("trailing fields on a gate line");
            }
        }
        if (next_line(s)) {
            delete b;
            return fail("more gate lines than n_gates");
        }
        for (uint32_t l = 0; l < L; l++) b->level_offsets[l + 1] += b->level_offsets[l];
    } catch (const std::bad_alloc &) {
        delete b;
        return PDF_ENOMEM;
    }
    pdf_netlist view;
    pdf_netbuf_view(b, &view);
    const pdf_status st = pdf_netlist_check(&view, msg, msg_len);
    if (st != PDF_OK) {
        delete b;
        return st;
    }
    *out = b;
    return PDF_OK;
}

namespace {

// Calls fn(row index, digits) for each vector line; returns the line number of
// the first malformed line, or 0.
template <class F>
uint64_t scan_vectors(std::ifstream &in, F fn) {
    std::string line, digits;
    uint64_t ln = 0, row = 0;
    while (std::getline(in, line)) {
        ln++;
        digits.clear();
        for (char ch : strip_comment(line)) {
            if (ch == '0' || ch == '1')
                digits.push_back(ch);
            else if (!std::isspace((unsigned char)ch))
                return ln;
        }
        if (digits.empty()) continue;
        if (!fn(row++, digits)) return ln;
    }
    return 0;
}

}  // namespace

extern "C" pdf_status pdf_vectors_dim(const char *path, uint64_t *n_vec, uint32_t *width) {
    if (!path || !n_vec || !width) return PDF_EINVAL;
    *n_vec = 0;
    *width = 0;
    std::ifstream in(path);
    if (!in) return PDF_EINVAL;
    uint64_t n = 0;
    size_t w = 0;
    const uint64_t bad = scan_vectors(in, [&](uint64_t, const std::string &d) {
        if (n == 0) w = d.size();
        n++;
        return d.size() == w && w < 0xFFFFFFFFull;
    });
    if (bad || n == 0) return PDF_EINVAL;
    *n_vec = n;
    *width = (uint32_t)w;
    return PDF_OK;
}

extern "C" pdf_status pdf_vectors_read(const char *path, uint32_t n_pi, uint64_t n_vec, uint8_t *vec) {
    if (!path || !vec || n_pi == 0 || n_vec == 0) return PDF_EINVAL;
    std::ifstream in(path);
    if (!in) return PDF_EINVAL;
    uint64_t rows = 0;
    const uint64_t bad = scan_vectors(in, [&](uint64_t r, const std::string &d) {
        if (d.size() != n_pi || r >= n_vec) return false;
        for (uint32_t i = 0; i < n_pi; i++) vec[(uint64_t)i * n_vec + r] = (uint8_t)(d[i] - '0');
        rows = r + 1;
        return true;
    });
    return (bad || rows != n_vec) ? PDF_EINVAL : PDF_OK;
}

namespace {

// Header line of the per-gate dumps (simkernel.cuh:256-261).
void dump_header(std::ofstream &o, uint32_t n_gates) {
    o << "Gate:     " << "\t";
    for (uint32_t i = 0; i < n_gates; i++) o << std::setw(4) << i << " ";
    o << "\n";
}

inline uint32_t bit_at(const uint32_t *row, uint64_t p) { return (row[p >> 5] >> (p & 31)) & 1u; }

// Decimal digits of the 128-bit value hi:lo.
std::string u128_decimal(uint64_t hi, uint64_t lo) {
    unsigned __int128 v = ((unsigned __int128)hi << 64) | lo;
    std::string d;
    do {
        d.insert(d.begin(), char('0' + (int)(v % 10)));
        v /= 10;
    } while (v);
    return d;
}

}  // namespace

extern "C" pdf_status pdf_dump_sim(const char *path, const uint32_t *sim_v, const uint32_t *sim_t,
                                   uint32_t n_gates, uint64_t n_pairs, uint64_t ld, uint64_t pair_base,
                                   int append) {
    if (!path || !sim_v || !sim_t || !n_gates || ld < (n_pairs + 31) / 32) return PDF_EINVAL;
    std::ofstream o(path, append ? std::ios::out | std::ios::app : std::ios::out);
    if (!o) return PDF_EINVAL;
    if (!append) dump_header(o, n_gates);
    static const char *code[4] = {"S0 ", "S1 ", "T0 ", "T1 "};
    for (uint64_t p = 0; p < n_pairs; p++) {
        o << "Vector " << p + pair_base << ":\t";
        for (uint32_t g = 0; g < n_gates; g++) {
            const uint64_t r = (uint64_t)g * ld;
            o << std::setw(5) << code[bit_at(sim_v + r, p) | (bit_at(sim_t + r, p) << 1)];
        }
        o << "\n";
    }
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_dump_mark(const char *path, const uint32_t *mark, uint32_t n_gates, uint64_t n_pairs,
                                    uint64_t ld, uint64_t pair_base, int append) {
    if (!path || !mark || !n_gates || ld < (n_pairs + 31) / 32) return PDF_EINVAL;
    std::ofstream o(path, append ? std::ios::out | std::ios::app : std::ios::out);
    if (!o) return PDF_EINVAL;
    if (!append) dump_header(o, n_gates);
    for (uint64_t p = 0; p < n_pairs; p++) {
        o << "Vector " << p + pair_base << ":\t";
        for (uint32_t g = 0; g < n_gates; g++) o << std::setw(4) << (bit_at(mark + (uint64_t)g * ld, p) ? "Y" : "N") << " ";
        o << "\n";
    }
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_dump_cover(const char *path, const uint64_t *counts, uint32_t n_pi, uint64_t n_pairs,
                                     uint64_t pair_base, int append) {
    if (!path || !counts || !n_pi) return PDF_EINVAL;
    std::ofstream o(path, append ? std::ios::out | std::ios::app : std::ios::out);
    if (!o) return PDF_EINVAL;
    if (!append) dump_header(o, n_pi);  // the primary inputs are gates 0 .. n_pi - 1
    for (uint64_t p = 0; p < n_pairs; p++) {
        o << "Vector " << p + pair_base << ":\t";
        for (uint32_t i = 0; i < n_pi; i++) {
            const uint64_t *c = counts + ((uint64_t)i * n_pairs + p) * 2;
            o << std::setw(4) << u128_decimal(c[1], c[0]) << " ";
        }
        o << "\n";
    }
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_dump_merge(const char *path, const uint32_t *first_x, const uint32_t *first_y,
                                     uint32_t n_gates) {
    if (!path || !first_x || !first_y) return PDF_EINVAL;
    std::ofstream o(path);
    if (!o) return PDF_EINVAL;
    // the reference keeps the ids in an int2 (mergekernel.cuh:271-279)
    for (uint32_t g = 0; g < n_gates; g++)
        o << "Gate " << g << ":\t" << std::setw(4) << (int32_t)first_x[g] << "," << (int32_t)first_y[g] << " "
          << "\n";
    return o.good() ? PDF_OK : PDF_EINVAL;
}

extern "C" pdf_status pdf_dump_segments(const char *path, const uint32_t *gates, uint32_t seg_len,
                                        uint64_t n_segments, const uint32_t *first_x, const uint32_t *first_y) {
    if (!path || !gates || !first_x || !first_y || seg_len == 0) return PDF_EINVAL;
    std::ofstream o(path);
    if (!o) return PDF_EINVAL;
    for (uint64_t s = 0; s < n_segments; s++) {
        o << "Segment " << s << "(";
        for (uint32_t j = 0; j < seg_len; j++) o << gates[s * seg_len + j] << (j + 1 < seg_len ? "," : "");
        o << "): " << (int32_t)first_x[s] << "," << (int32_t)first_y[s] << " " << "\n";
    }
    return o.good() ? PDF_OK : PDF_EINVAL;
}
