// pdf_gen.cpp -- seeded synthetic levelized netlists and vector pairs.
//
// The reference ships no circuits (its Makefile test target points at
// ../data/c17.level, outside the repository, Makefile:16-18), so every
// workload here is generated: splitmix64 seeds xoshiro256**, the netlist and
// the pairs use separate streams, and the same seed always gives the same
// bytes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "pdf.h"
#include "pdf_internal.h"

namespace {

inline uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Xoshiro256 {
    uint64_t s[4];
    explicit Xoshiro256(uint64_t seed) {
        uint64_t x = seed;
        for (auto &v : s) v = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

// Draw from a discrete distribution given its cumulative table.
uint32_t draw_cdf(Xoshiro256 &r, const std::vector<double> &cdf) {
    const double u = r.uniform() * cdf.back();
    return (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
}

}  // namespace

extern "C" pdf_status pdf_gen_netlist(const pdf_gen_params *p, pdf_netbuf **out) {
    if (!p || !out) return PDF_EINVAL;
    *out = nullptr;
    const uint32_t G = p->n_gates, NPI = p->n_pi, D = p->depth;
    if (NPI == 0 || D == 0 || G < NPI + D) return PDF_EINVAL;
    if (p->fanin_min == 0 || p->fanin_max < p->fanin_min || p->fanin_max > 255) return PDF_EINVAL;
    if (p->n_po > G - NPI) return PDF_EINVAL;
    uint32_t mask = p->type_mask;
    if (mask == 0)
        mask = (1u << PDF_AND) | (1u << PDF_NAND) | (1u << PDF_OR) | (1u << PDF_NOR) |
               (1u << PDF_XOR) | (1u << PDF_XNOR) | (1u << PDF_NOT) | (1u << PDF_BUFF);
    if (mask & ((1u << PDF_INPT) | (1u << PDF_UNKN)) || (mask >> PDF_NTYPES)) return PDF_EINVAL;
    std::vector<uint8_t> types;
    for (int t = 0; t < PDF_NTYPES; t++)
        if (mask & (1u << t)) types.push_back((uint8_t)t);

    pdf_netbuf *b = new (std::nothrow) pdf_netbuf();
    if (!b) return PDF_ENOMEM;
    try {
        Xoshiro256 rng(p->seed);
        const uint32_t L = D + 1;
        b->n_gates = G;
        b->n_levels = L;
        b->level_offsets.resize(L + 1);
        b->level_offsets[0] = 0;
        b->level_offsets[1] = NPI;
        const uint32_t rest = G - NPI;
        for (uint32_t l = 1; l <= D; l++) {
            const uint32_t w = rest / D + ((l - 1) < rest % D ? 1 : 0);
            b->level_offsets[l + 1] = b->level_offsets[l] + w;
        }
        std::vector<uint32_t> level_of(G);
        for (uint32_t l = 0; l < L; l++)
            for (uint32_t g = b->level_offsets[l]; g < b->level_offsets[l + 1]; g++) level_of[g] = l;

        // Fan-out weights: a source is picked with probability proportional to
        // its weight.  Exp(1) weights give a geometric fan-out law (a Poisson
        // count with an exponentially distributed rate); Zipf weights give a
        // power-law tail.
        std::vector<double> weight(G);
        const uint32_t fo_max = p->fanout_max ? p->fanout_max : 0xFFFFFFu;
        std::vector<double> zipf_cdf;
        if (p->fanout_dist == 1) {
            const uint32_t K = p->fanout_max ? p->fanout_max : 256;
            zipf_cdf.resize(K);
            double acc = 0;
            for (uint32_t k = 1; k <= K; k++) zipf_cdf[k - 1] = (acc += std::pow((double)k, -p->zipf_s));
        }
        for (uint32_t g = 0; g < G; g++)
            weight[g] = p->fanout_dist == 1 ? (double)(draw_cdf(rng, zipf_cdf) + 1)
                                            : -std::log(1.0 - rng.uniform()) + 1e-9;
        // Per-level cumulative weights for weighted source picks.
        std::vector<double> cum(G);
        for (uint32_t l = 0; l < L; l++) {
            double acc = 0;
            for (uint32_t g = b->level_offsets[l]; g < b->level_offsets[l + 1]; g++) cum[g] = (acc += weight[g]);
        }
        std::vector<uint32_t> nfo(G, 0);
        auto pick = [&](uint32_t l) -> uint32_t {
            const uint32_t lo = b->level_offsets[l], hi = b->level_offsets[l + 1];
            const double total = cum[hi - 1];
            for (int attempt = 0; attempt < 64; attempt++) {
                const double u = rng.uniform() * total;
                uint32_t g = (uint32_t)(std::upper_bound(cum.begin() + lo, cum.begin() + hi, u) - cum.begin());
                if (g >= hi) g = hi - 1;
                if (nfo[g] < fo_max) return g;
            }
            for (uint32_t g = lo; g < hi; g++)
                if (nfo[g] < fo_max) return g;
            return lo + rng.below(hi - lo);  // every gate is full: exceed the cap
        };

        b->type.assign(G, PDF_INPT);
        b->po.assign(G, 0);
        b->nfi.assign(G, 0);
        std::vector<std::vector<uint32_t>> fin(G);
        for (uint32_t g = NPI; g < G; g++) {
            const uint32_t l = level_of[g];
            const uint8_t t = types[rng.below((uint32_t)types.size())];
            b->type[g] = t;
            uint32_t n = 1;
            if (t >= PDF_AND && t <= PDF_XNOR) n = p->fanin_min + rng.below(p->fanin_max - p->fanin_min + 1);
            auto &f = fin[g];
            f.reserve(n);
            // one fan-in from the level just below, so the depth is exact
            f.push_back(pick(l - 1));
            for (uint32_t j = 1; j < n; j++) {
                uint32_t src = 0;
                for (int attempt = 0; attempt < 16; attempt++) {
                    uint32_t d = 1;
                    while (d < l && (rng.next() & 1)) d++;  // P(d) = 2^-d, clamped
                    src = pick(l - d);
                    if (std::find(f.begin(), f.end(), src) == f.end()) break;
                }
                f.push_back(src);
            }
            // the level l-1 fan-in takes a random position among the fan-ins
            std::swap(f[0], f[rng.below((uint32_t)f.size())]);
            for (uint32_t s : f) nfo[s]++;
            b->nfi[g] = (uint32_t)f.size();
        }
        // Primary outputs: drawn from the sinks (gates above the inputs with no
        // fan-out); if there are too few sinks, the rest are drawn from the
        // other gates above the inputs.
        std::vector<uint32_t> sinks, others;
        for (uint32_t g = NPI; g < G; g++) (nfo[g] == 0 ? sinks : others).push_back(g);
        auto shuffle = [&](std::vector<uint32_t> &v) {
            for (size_t i = v.size(); i > 1; i--) std::swap(v[i - 1], v[rng.below((uint32_t)i)]);
        };
        shuffle(sinks);
        shuffle(others);
        uint32_t placed = 0;
        for (uint32_t g : sinks) {
            if (placed == p->n_po) break;
            b->po[g] = 1;
            placed++;
        }
        for (uint32_t g : others) {
            if (placed == p->n_po) break;
            b->po[g] = 1;
            placed++;
        }
        // CSR: fan-ins, then fan-outs (in consumer order).
        b->nfo = nfo;
        b->edge_offset.resize(G);
        uint64_t off = 0;
        for (uint32_t g = 0; g < G; g++) {
            b->edge_offset[g] = off;
            off += (uint64_t)b->nfi[g] + nfo[g];
        }
        b->edges.resize(off);
        std::vector<uint32_t> fill(G, 0);
        for (uint32_t g = 0; g < G; g++) {
            for (uint32_t j = 0; j < b->nfi[g]; j++) {
                const uint32_t s = fin[g][j];
                b->edges[b->edge_offset[g] + j] = s;
                b->edges[b->edge_offset[s] + b->nfi[s] + fill[s]++] = g;
            }
        }
    } catch (const std::bad_alloc &) {
        delete b;
        return PDF_ENOMEM;
    }
    *out = b;
    return PDF_OK;
}

extern "C" pdf_status pdf_netbuf_from(const pdf_netlist *nl, pdf_netbuf **out) {
    if (!nl || !out) return PDF_EINVAL;
    *out = nullptr;
    pdf_netbuf *b = new (std::nothrow) pdf_netbuf();
    if (!b) return PDF_ENOMEM;
    try {
        const uint32_t G = nl->n_gates;
        b->n_gates = G;
        b->n_levels = nl->n_levels;
        b->level_offsets.assign(nl->level_offsets, nl->level_offsets + nl->n_levels + 1);
        b->type.assign(nl->type, nl->type + G);
        b->po.assign(nl->po, nl->po + G);
        b->nfi.assign(nl->nfi, nl->nfi + G);
        b->nfo.assign(nl->nfo, nl->nfo + G);
        b->edge_offset.assign(nl->edge_offset, nl->edge_offset + G);
        b->edges.assign(nl->edges, nl->edges + nl->n_edges);
    } catch (const std::bad_alloc &) {
        delete b;
        return PDF_ENOMEM;
    }
    *out = b;
    return PDF_OK;
}

extern "C" void pdf_netbuf_view(const pdf_netbuf *b, pdf_netlist *v) {
    if (!b || !v) return;
    v->n_gates = b->n_gates;
    v->n_levels = b->n_levels;
    v->level_offsets = b->level_offsets.data();
    v->type = b->type.data();
    v->po = b->po.data();
    v->nfi = b->nfi.data();
    v->nfo = b->nfo.data();
    v->edge_offset = b->edge_offset.data();
    v->edges = b->edges.data();
    v->n_edges = b->edges.size();
}

extern "C" void pdf_netbuf_free(pdf_netbuf *b) { delete b; }

// Each PI row has its own stream (seeded from the seed and the row), and the
// words of a row alternate v, t, so a prefix of the pairs does not depend on
// how many pairs are drawn.
extern "C" pdf_status pdf_gen_pairs(uint64_t seed, uint32_t n_pi, uint64_t n_pairs, uint64_t ld,
                                    uint32_t *v, uint32_t *t) {
    const uint64_t W = (n_pairs + 31) / 32;
    if (!v || !t || ld < W) return PDF_EINVAL;
    for (uint32_t i = 0; i < n_pi; i++) {
        uint64_t x = seed ^ (0xD1B54A32D192ED03ull * (i + 1));
        Xoshiro256 r(splitmix64(x));
        uint32_t *vr = v + (uint64_t)i * ld, *tr = t + (uint64_t)i * ld;
        for (uint64_t w = 0; w < W; w += 1) {
            const uint64_t a = r.next();
            vr[w] = (uint32_t)a;
            tr[w] = (uint32_t)(a >> 32);
        }
        if (n_pairs % 32) {
            const uint32_t keep = (1u << (n_pairs % 32)) - 1;
            vr[W - 1] &= keep;
            tr[W - 1] &= keep;
        }
        for (uint64_t w = W; w < ld; w++) vr[w] = tr[w] = 0;
    }
    return PDF_OK;
}

extern "C" pdf_status pdf_pairs_from_vectors(const uint8_t *vec, uint32_t n_pi, uint64_t n_vec,
                                             uint64_t ld, uint32_t *v, uint32_t *t) {
    const uint64_t W = (n_vec + 31) / 32;
    if (!vec || !v || !t || ld < W || n_vec == 0) return PDF_EINVAL;
    for (uint32_t i = 0; i < n_pi; i++) {
        const uint8_t *row = vec + (uint64_t)i * n_vec;
        uint32_t *vr = v + (uint64_t)i * ld, *tr = t + (uint64_t)i * ld;
        std::memset(vr, 0, ld * 4);
        std::memset(tr, 0, ld * 4);
        for (uint64_t p = 0; p < n_vec; p++) {
            const uint32_t v1 = row[p] & 1, v2 = row[p + 1 < n_vec ? p + 1 : 0] & 1;
            vr[p / 32] |= v2 << (p % 32);
            tr[p / 32] |= (v1 ^ v2) << (p % 32);
        }
    }
    return PDF_OK;
}
