/*
 * pdf_oracle.c -- CPU oracle (test infrastructure only; see pdf_oracle.h).
 *
 * Restates the reference's algorithm one byte per (gate, pair), like the
 * reference's GPU_Data rows.  Each function cites the reference lines it
 * follows (lordofhyphens/gpu-path-delay-coverage).  The only deliberate
 * departures, all documented at the function:
 *   - merge takes the minimum over every pair of the chunk (the reference's
 *     kernSegmentReduce2 only visits the first 1056 words of a chunk,
 *     mergekernel.cuh:125-130; it is exact for chunks of <= 4224 pairs);
 *   - path counts are exact 128-bit integers (the reference packs 16-bit
 *     h and c per (net, pair), coverkernel.cuh:41-43, and sums in uint32,
 *     coverkernel.cuh:82-101); they agree wherever the reference does not
 *     overflow.
 */
#include "pdf_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;
static const u128 U128_MAX = ~(u128)0;

/* ---- lookup tables: the reference's constants (simkernel.cuh:158-165) ---- */

static const uint8_t LUT_AND2[16] = {0, 0, 0, 0, 0, 1, 2, 3, 0, 2, 2, 0, 0, 3, 0, 3};
static const uint8_t LUT_NAND2[16] = {1, 1, 1, 1, 1, 0, 3, 2, 1, 3, 3, 1, 1, 2, 1, 2};
static const uint8_t LUT_OR2[16] = {0, 1, 2, 3, 1, 1, 1, 1, 2, 1, 2, 1, 3, 1, 1, 3};
static const uint8_t LUT_NOR2[16] = {1, 0, 3, 2, 0, 0, 0, 0, 3, 0, 3, 0, 2, 0, 0, 2};
static const uint8_t LUT_XOR2[16] = {0, 1, 2, 3, 1, 0, 3, 2, 2, 3, 0, 1, 3, 2, 1, 0};
static const uint8_t LUT_XNOR2[16] = {1, 0, 3, 2, 0, 1, 2, 3, 3, 2, 1, 0, 2, 3, 0, 1};
static const uint8_t LUT_STABLE[4] = {0, 2, 3, 1}; /* [v2 * 2 + v1] */
static const uint8_t LUT_NOT[4] = {1, 0, 3, 2};

/* Sensitisation tables (markkernel.cuh:36-37), indexed by type - 2. */
static const uint16_t SENS_NR[6] = {0x2A00, 0x2A00, 0x5100, 0x5100, 0x0000, 0x0000};
static const uint16_t SENS_R[6] = {0x2200, 0x2200, 0x1100, 0x1100, 0x0000, 0x0000};
/* FIXED modes (no reference counterpart), same LUT_16 layout, bit on*4+off:
 * textbook robust (on c->nc: side steady nc; on nc->c: side final nc; XOR:
 * side steady) and non-robust (side final nc; XOR: any side). */
static const uint16_t SENS_FIXED_R[6] = {0x2A00, 0x2A00, 0x5100, 0x5100, 0x3300, 0x3300};
static const uint16_t SENS_FIXED_NR[6] = {0xAA00, 0xAA00, 0x5500, 0x5500, 0xFF00, 0xFF00};

/* tex2D(lut, val, r) on a 4x4 array = lut[r * 4 + val] (simkernel.cuh:51-56). */
uint8_t pdfo_lut2(int type, uint8_t val, uint8_t r) {
    const int i = (r & 3) * 4 + (val & 3);
    switch (type) {
        case PDF_XOR: return LUT_XOR2[i];
        case PDF_XNOR: return LUT_XNOR2[i];
        case PDF_OR: return LUT_OR2[i];
        case PDF_NOR: return LUT_NOR2[i];
        case PDF_AND: return LUT_AND2[i];
        case PDF_NAND: return LUT_NAND2[i];
        default: return 0;
    }
}

/* tex2D(stableLUT, v1, v2) (simkernel.cuh:121-124). */
uint8_t pdfo_stable(uint8_t v1, uint8_t v2) { return LUT_STABLE[(v2 & 1) * 2 + (v1 & 1)]; }

/* tex1D(notLUT, v) (simkernel.cuh:137-140). */
uint8_t pdfo_not(uint8_t v) { return LUT_NOT[v & 3]; }

/* LUT_16(LUT[type - 2], on, off) (markkernel.cuh:39-41,49). */
int pdfo_sens(int mark_mode, int type, uint8_t on, uint8_t off) {
    if (type < PDF_AND || type > PDF_XNOR) return 0;
    const uint16_t *tab = mark_mode == PDF_MARK_ROBUST          ? SENS_R
                          : mark_mode == PDF_MARK_FIXED_ROBUST    ? SENS_FIXED_R
                          : mark_mode == PDF_MARK_FIXED_NONROBUST ? SENS_FIXED_NR
                                                                  : SENS_NR;
    const uint16_t t = tab[type - 2];
    return (t >> (((on & 3) << 2) + (off & 3))) & 1;
}

/* The coalesce_t overload of simLUT (simkernel.cuh:62-95): XOR and XNOR fall
 * through to `packed = 0`, so they yield S0 (kernSimulateP1 uses this
 * overload, :146). */
static inline uint8_t sim_lut_coalesced(int type, uint8_t val, uint8_t r) {
    switch (type) {
        case PDF_OR:
        case PDF_NOR:
        case PDF_AND:
        case PDF_NAND: return pdfo_lut2(type, val, r);
        default: return 0;
    }
}

static inline uint32_t fanin(const pdf_netlist *nl, uint32_t g, uint32_t j) {
    return nl->edges[nl->edge_offset[g] + j];
}
static inline uint32_t fanout(const pdf_netlist *nl, uint32_t g, uint32_t k) {
    return nl->edges[nl->edge_offset[g] + nl->nfi[g] + k];
}

static int nthreads(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

/* Split [0, n) into `parts` contiguous ranges aligned to 64 pairs. */
static void part_range(uint64_t n, int parts, int i, uint64_t *lo, uint64_t *hi) {
    uint64_t blocks = (n + 63) / 64;
    uint64_t per = (blocks + parts - 1) / parts;
    uint64_t a = per * i * 64, b = per * (i + 1) * 64;
    if (a > n) a = n;
    if (b > n) b = n;
    *lo = a;
    *hi = b;
}

/*
 * One gate of kernSimulateP1 (simkernel.cuh:111-149) over pairs [p0, p1).
 * INPT rows come from `pi` (already-formed pair codes).
 */
static void sim_gate(const pdf_netlist *nl, uint32_t g, const uint8_t *pi, uint64_t n_pairs,
                     uint8_t *sim, uint64_t p0, uint64_t p1, int fixed) {
    uint8_t *row = sim + (uint64_t)g * n_pairs;
    const int type = nl->type[g];
    if (fixed && type >= PDF_AND && type <= PDF_XNOR) {
        /* FIXED: the gate's n-input function under each vector separately */
        const int inv = type == PDF_NAND || type == PDF_NOR || type == PDF_XNOR;
        for (uint64_t p = p0; p < p1; p++) {
            uint8_t v1 = 0, v2 = 0;
            for (uint32_t j = 0; j < nl->nfi[g]; j++) {
                const uint8_t c = sim[(uint64_t)fanin(nl, g, j) * n_pairs + p];
                const uint8_t b2 = c & 1, b1 = (uint8_t)(b2 ^ (c >> 1));
                if (j == 0) {
                    v1 = b1;
                    v2 = b2;
                } else if (type == PDF_AND || type == PDF_NAND) {
                    v1 &= b1;
                    v2 &= b2;
                } else if (type == PDF_OR || type == PDF_NOR) {
                    v1 |= b1;
                    v2 |= b2;
                } else {
                    v1 ^= b1;
                    v2 ^= b2;
                }
            }
            v1 ^= (uint8_t)inv;
            v2 ^= (uint8_t)inv;
            row[p] = pdfo_stable(v1, v2);
        }
        return;
    }
    switch (type) {
        case PDF_INPT: /* :112-125 */
            memcpy(row + p0, pi + (uint64_t)g * n_pairs + p0, p1 - p0);
            break;
        case PDF_DFF:
        case PDF_BUFF:
        case PDF_FROM: { /* :126-130, copy fan-in 0 */
            const uint8_t *f0 = sim + (uint64_t)fanin(nl, g, 0) * n_pairs;
            memcpy(row + p0, f0 + p0, p1 - p0);
            break;
        }
        default: { /* :131-148 */
            const uint8_t *f0 = sim + (uint64_t)fanin(nl, g, 0) * n_pairs;
            for (uint64_t p = p0; p < p1; p++) {
                uint8_t val = f0[p];
                if (type == PDF_NOT) val = pdfo_not(val);
                row[p] = val;
            }
            /* left fold of the 2-input op over the remaining fan-ins (:142-148) */
            for (uint32_t j = 1; j < nl->nfi[g]; j++) {
                const uint8_t *fj = sim + (uint64_t)fanin(nl, g, j) * n_pairs;
                for (uint64_t p = p0; p < p1; p++) row[p] = sim_lut_coalesced(type, row[p], fj[p]);
            }
        }
    }
}

int pdfo_sim(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs, uint8_t *sim,
             int threads) {
    return pdfo_sim_mode(nl, pi_codes, n_pairs, sim, PDF_MARK_DEFAULT, threads);
}

int pdfo_sim_mode(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs, uint8_t *sim,
                  int mark_mode, int threads) {
    const int fixed = mark_mode >= PDF_MARK_FIXED_ROBUST;
    const int nt = nthreads(threads);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num(), cnt = omp_get_num_threads();
#else
        const int tid = 0, cnt = 1;
#endif
        uint64_t p0, p1;
        part_range(n_pairs, cnt, tid, &p0, &p1);
        if (p0 < p1)
            for (uint32_t g = 0; g < nl->n_gates; g++) sim_gate(nl, g, pi_codes, n_pairs, sim, p0, p1, fixed);
    }
    return 0;
}

/*
 * kernSimulateP1 with the reference's own pair formation from a vector stream
 * (simkernel.cuh:115-124): pair p = stable(vec[p], vec[p + 1]); the last pair
 * takes vector 0 as its second vector.  Matches the reference exactly when
 * n_vec is a multiple of 4 (otherwise the reference reads row padding, :116-120).
 */
int pdfo_sim_vectors(const pdf_netlist *nl, const uint8_t *vec, uint64_t n_vec, uint8_t *sim,
                     int threads) {
    const uint32_t n_pi = nl->level_offsets[1];
    uint8_t *pi = (uint8_t *)malloc((size_t)n_pi * n_vec + 1);
    if (!pi) return -1;
    for (uint32_t i = 0; i < n_pi; i++)
        for (uint64_t p = 0; p < n_vec; p++) {
            const uint8_t v1 = vec[(uint64_t)i * n_vec + p];
            const uint8_t v2 = vec[(uint64_t)i * n_vec + (p + 1 < n_vec ? p + 1 : 0)];
            pi[(uint64_t)i * n_vec + p] = pdfo_stable(v1, v2);
        }
    int rc = pdfo_sim(nl, pi, n_vec, sim, threads);
    free(pi);
    return rc;
}

/*
 * kernMarkPathSegments (markkernel.cuh:215-270) over levels in order, then
 * kernRemoveInvalidMarks (markkernel.cuh:271-293) over levels in reverse
 * (gpuMarkPaths, markkernel.cuh:308-342).
 */
static void mark_forward_gate(const pdf_netlist *nl, uint32_t g, const uint8_t *sim,
                              uint64_t n_pairs, int mark_mode, uint8_t *mark, uint64_t p0,
                              uint64_t p1) {
    const uint8_t *srow = sim + (uint64_t)g * n_pairs;
    uint8_t *row = mark + (uint64_t)g * n_pairs;
    const int type = nl->type[g];
    const uint32_t nfi = nl->nfi[g];
    for (uint64_t p = p0; p < p1; p++) {
        const uint8_t trans = srow[p] > 1; /* rowCache (:230) */
        uint8_t r = 0;
        switch (type) {
            case PDF_INPT: r = trans; break; /* :234-241 */
            case PDF_FROM:
            case PDF_BUFF:
            case PDF_DFF:
            case PDF_NOT: r = mark[(uint64_t)fanin(nl, g, 0) * n_pairs + p]; break; /* :242-246 */
            case PDF_OR:
            case PDF_NOR:
            case PDF_XOR:
            case PDF_XNOR:
            case PDF_NAND:
            case PDF_AND: /* :253-261 with robust()/nonrobust() (:43-72) */
                for (uint32_t f1 = 0; f1 < nfi; f1++) {
                    /* oldmark is fan-in 0's mark for every candidate (:254); the
                     * FIXED modes take the candidate's own mark */
                    const uint32_t from = mark_mode >= PDF_MARK_FIXED_ROBUST ? f1 : 0;
                    const uint8_t oldmark = mark[(uint64_t)fanin(nl, g, from) * n_pairs + p];
                    const uint8_t on = sim[(uint64_t)fanin(nl, g, f1) * n_pairs + p];
                    uint8_t tmp = 0xFF;
                    for (uint32_t f2 = 0; f2 < nfi; f2++) {
                        if (f1 == f2) continue;
                        const uint8_t off = sim[(uint64_t)fanin(nl, g, f2) * n_pairs + p];
                        tmp = (uint8_t)(tmp && pdfo_sens(mark_mode, type, on, off));
                    }
                    tmp &= oldmark;
                    r |= tmp;
                }
                break;
            default: break;
        }
        row[p] = r & trans; /* :266-267 */
    }
}

static void prune_gate(const pdf_netlist *nl, uint32_t g, uint64_t n_pairs, uint8_t *mark,
                       uint64_t p0, uint64_t p1) {
    uint8_t *row = mark + (uint64_t)g * n_pairs;
    const uint8_t po = nl->po[g] > 0; /* :282 */
    for (uint64_t p = p0; p < p1; p++) {
        uint8_t r = po;
        for (uint32_t k = 0; k < nl->nfo[g]; k++) r |= mark[(uint64_t)fanout(nl, g, k) * n_pairs + p];
        row[p] = r & row[p]; /* :290-291 */
    }
}

int pdfo_mark(const pdf_netlist *nl, const uint8_t *sim, uint64_t n_pairs, int mark_mode,
              uint8_t *mark, int prune, int threads) {
    const int nt = nthreads(threads);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num(), cnt = omp_get_num_threads();
#else
        const int tid = 0, cnt = 1;
#endif
        uint64_t p0, p1;
        part_range(n_pairs, cnt, tid, &p0, &p1);
        if (p0 < p1) {
            for (uint32_t g = 0; g < nl->n_gates; g++)
                mark_forward_gate(nl, g, sim, n_pairs, mark_mode, mark, p0, p1);
            if (prune)
                for (uint32_t g = nl->n_gates; g-- > 0;) prune_gate(nl, g, n_pairs, mark, p0, p1);
        }
    }
    return 0;
}

/*
 * kernSegmentReduce2<1> (mergekernel.cuh:116-198) for segments of one net:
 * first_x(g) = min pair id p with mark && value-bit 0 (falling), first_y with
 * value-bit 1 (rising), folded with atomicMin into the persistent list
 * (:185-197).  Unsigned compare, 0xFFFFFFFF = none.  Every pair of the chunk is
 * visited (see the file header).
 */
int pdfo_merge(const pdf_netlist *nl, const uint8_t *sim, const uint8_t *mark, uint64_t n_pairs,
               uint64_t pair_base, uint32_t *first_x, uint32_t *first_y, int threads) {
    (void)threads;
    for (uint32_t g = 0; g < nl->n_gates; g++) {
        const uint8_t *m = mark + (uint64_t)g * n_pairs;
        const uint8_t *s = sim + (uint64_t)g * n_pairs;
        uint32_t fx = 0xFFFFFFFFu, fy = 0xFFFFFFFFu;
        for (uint64_t p = 0; p < n_pairs && (fx == 0xFFFFFFFFu || fy == 0xFFFFFFFFu); p++) {
            if (!m[p]) continue;
            const uint32_t pid = (uint32_t)(pair_base + p);
            if (s[p] & 1) {
                if (fy == 0xFFFFFFFFu) fy = pid;
            } else {
                if (fx == 0xFFFFFFFFu) fx = pid;
            }
        }
        if (fx < first_x[g]) first_x[g] = fx;
        if (fy < first_y[g]) first_y[g] = fy;
    }
    return 0;
}

static inline u128 sat_add(u128 a, u128 b, int *ovf) {
    u128 r = a + b;
    if (r < a) {
        *ovf = 1;
        return U128_MAX;
    }
    return r;
}

/*
 * kernCover<1,512> (coverkernel.cuh:171-230) over levels in reverse, then
 * kernSumSingle<512> (coverkernel.cuh:77-105) over the level-0 INPT gates.
 * Per pair p (global id pid):
 *   H = [po == 1] * m + sum_fo h(fo);  C = sum_fo c(fo)
 *   first = (pid == first_x(g)) || (pid == first_y(g))
 *   c = m ? C + (first ? H : 0) : 0;   h = (m && !first) ? H : 0;  h = 0 on INPT
 * Values saturate at 2^128 - 1.  PDF_FLAG_OVERFLOW is raised when a c value
 * saturates or the sum does: every marked net has a marked path from an input
 * (marks need fan-in 0's mark), so a saturated c means the true total is at
 * least 2^128; an h that saturates but is never credited changes nothing.
 */
static int cover_impl(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                      const uint32_t *first_x, const uint32_t *first_y, const uint8_t *first_plane,
                      uint64_t *pi_counts, uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads);

int pdfo_cover(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
               const uint32_t *first_x, const uint32_t *first_y, uint64_t *lo, uint64_t *hi,
               uint32_t *flags, int threads) {
    return cover_impl(nl, mark, n_pairs, pair_base, first_x, first_y, NULL, NULL, lo, hi, flags, threads);
}

/* pdfo_cover, also writing the c value of every primary input i for every
 * pair p to pi_counts[(i * n_pairs + p) * 2 + {0, 1}] (low, high 64 bits):
 * what debugCover prints to gpucover.log (coverkernel.cuh:44-66). */
int pdfo_cover_counts(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                      const uint32_t *first_x, const uint32_t *first_y, uint64_t *pi_counts, uint64_t *lo,
                      uint64_t *hi, uint32_t *flags, int threads) {
    return cover_impl(nl, mark, n_pairs, pair_base, first_x, first_y, NULL, pi_counts, lo, hi, flags, threads);
}

/* first_plane (segments longer than one net): byte [g][p] = 1 when pair p of
 * the chunk first-detects a segment through g; replaces the first_x/first_y
 * test (coverkernel.cuh:115-170 finds those pairs per gate). */
static int cover_impl(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                      const uint32_t *first_x, const uint32_t *first_y, const uint8_t *first_plane,
                      uint64_t *pi_counts, uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads) {
    const uint32_t G = nl->n_gates;
    const uint32_t lvl0 = nl->level_offsets[1];
    const int nt = nthreads(threads);
    u128 total = 0;
    int ovf_total = 0;
    int fail = 0;
#pragma omp parallel num_threads(nt)
    {
        u128 *h = (u128 *)malloc(sizeof(u128) * (size_t)G);
        u128 *c = (u128 *)malloc(sizeof(u128) * (size_t)G);
        u128 local = 0;
        int ovf = 0;
        if (!h || !c) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 16)
            for (int64_t pi = 0; pi < (int64_t)n_pairs; pi++) {
                const uint64_t p = (uint64_t)pi;
                const uint32_t pid = (uint32_t)(pair_base + p);
                for (uint32_t g = G; g-- > 0;) {
                    const int m = mark[(uint64_t)g * n_pairs + p] > 0; /* :194 */
                    if (!m) {
                        h[g] = 0;
                        c[g] = 0;
                        continue;
                    }
                    u128 H = nl->po[g] == 1 ? 1 : 0; /* :198-201 */
                    u128 C = 0;
                    int hovf = 0;
                    for (uint32_t k = 0; k < nl->nfo[g]; k++) { /* :204-209 */
                        const uint32_t fo = fanout(nl, g, k);
                        C = sat_add(C, c[fo], &ovf);
                        H = sat_add(H, h[fo], &hovf); /* an uncredited overflow is harmless */
                    }
                    const int first = first_plane ? first_plane[(uint64_t)g * n_pairs + p] != 0
                                                  : (first_x[g] == pid) || (first_y[g] == pid); /* :216 */
                    if (first) {
                        c[g] = sat_add(C, H, &ovf); /* :217 */
                        h[g] = 0;                    /* :219 */
                    } else {
                        c[g] = C;
                        h[g] = H;
                    }
                    /* a saturated h that gets credited shows up as a saturated c */
                    if (c[g] == U128_MAX) ovf = 1;
                    if (nl->type[g] == PDF_INPT) h[g] = 0; /* :221-223 */
                }
                for (uint32_t g = 0; g < lvl0; g++) /* kernSumSingle :83-92 */
                    if (nl->type[g] == PDF_INPT) {
                        local = sat_add(local, c[g], &ovf);
                        if (pi_counts) {
                            pi_counts[((uint64_t)g * n_pairs + p) * 2] = (uint64_t)c[g];
                            pi_counts[((uint64_t)g * n_pairs + p) * 2 + 1] = (uint64_t)(c[g] >> 64);
                        }
                    }
            }
        }
#pragma omp critical
        {
            total = sat_add(total, local, &ovf_total);
            if (ovf) ovf_total = 1;
        }
        free(h);
        free(c);
    }
    if (fail) return -1;
    u128 cur = ((u128)*hi << 64) | *lo;
    int o2 = 0;
    cur = sat_add(cur, total, &o2);
    if (ovf_total || o2) *flags |= PDF_FLAG_OVERFLOW;
    *lo = (uint64_t)cur;
    *hi = (uint64_t)(cur >> 64);
    return 0;
}

/* The chunk loop of main.cu:171-231 (segs = 1). */
int pdfo_grade(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs,
               uint64_t pair_base, int mark_mode, uint64_t chunk, uint32_t *first_x,
               uint32_t *first_y, uint8_t *sim_out, uint8_t *mark_out, uint64_t *lo,
               uint64_t *hi, uint32_t *flags, uint64_t *chunk_totals, int threads) {
    const uint32_t G = nl->n_gates;
    const uint32_t n_pi = nl->level_offsets[1];
    if (chunk == 0 || chunk > n_pairs) chunk = n_pairs ? n_pairs : 1;
    uint8_t *pi = (uint8_t *)malloc((size_t)n_pi * chunk + 1);
    uint8_t *sim = (uint8_t *)malloc((size_t)G * chunk + 1);
    uint8_t *mark = (uint8_t *)malloc((size_t)G * chunk + 1);
    if (!pi || !sim || !mark) {
        free(pi);
        free(sim);
        free(mark);
        return -1;
    }
    int rc = 0;
    uint64_t ci = 0;
    for (uint64_t start = 0; start < n_pairs; start += chunk, ci++) {
        const uint64_t K = n_pairs - start < chunk ? n_pairs - start : chunk;
        for (uint32_t i = 0; i < n_pi; i++)
            memcpy(pi + (uint64_t)i * K, pi_codes + (uint64_t)i * n_pairs + start, K);
        pdfo_sim_mode(nl, pi, K, sim, mark_mode, threads);                 /* main.cu:175 */
        pdfo_mark(nl, sim, K, mark_mode, mark, 1, threads);                /* main.cu:182 */
        pdfo_merge(nl, sim, mark, K, pair_base + start, first_x, first_y, threads); /* :185 */
        uint64_t clo = 0, chi = 0;
        uint32_t cfl = 0;
        rc = pdfo_cover(nl, mark, K, pair_base + start, first_x, first_y, &clo, &chi, &cfl,
                        threads); /* main.cu:206 */
        if (rc) break;
        if (chunk_totals) {
            chunk_totals[2 * ci] = clo;
            chunk_totals[2 * ci + 1] = chi;
        }
        u128 cur = ((u128)*hi << 64) | *lo; /* main.cu:224 */
        int o = 0;
        cur = sat_add(cur, ((u128)chi << 64) | clo, &o);
        if (o || (cfl & PDF_FLAG_OVERFLOW)) *flags |= PDF_FLAG_OVERFLOW;
        *lo = (uint64_t)cur;
        *hi = (uint64_t)(cur >> 64);
        if (sim_out || mark_out)
            for (uint32_t g = 0; g < G; g++) {
                if (sim_out)
                    memcpy(sim_out + (uint64_t)g * n_pairs + start, sim + (uint64_t)g * K, K);
                if (mark_out)
                    memcpy(mark_out + (uint64_t)g * n_pairs + start, mark + (uint64_t)g * K, K);
            }
    }
    free(pi);
    free(sim);
    free(mark);
    return rc;
}

/* ---- path segments longer than one net (main.cu:185-223, segs = N > 1) ----
 *
 * The reference builds its segment list in util/segment.cuh
 * (generateSegmentList, mergekernel.cuh:210), which its snapshot does not
 * contain.  Restated definition: a segment of length N is a directed subpath
 * of exactly N nets (g_0, ..., g_{N-1}), g_{i+1} a fan-out of g_i; listed by
 * g_0 ascending, then depth first along fan-outs in edge order.  For N = 1
 * the segments are the nets, which is the N = 1 path above. */

/* Number of segments of length N (saturates at UINT64_MAX); when out is not
 * NULL and cap >= the count, writes them as out[s * N + i]. */
uint64_t pdfo_segments(const pdf_netlist *nl, uint32_t N, uint32_t *out, uint64_t cap) {
    const uint32_t G = nl->n_gates;
    if (N == 0 || N > 8) return 0;
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * G), *nxt = (uint64_t *)malloc(sizeof(uint64_t) * G);
    if (!cnt || !nxt) {
        free(cnt);
        free(nxt);
        return UINT64_MAX;
    }
    for (uint32_t g = 0; g < G; g++) cnt[g] = 1;
    for (uint32_t k = 1; k < N; k++) {
        for (uint32_t g = 0; g < G; g++) {
            uint64_t t = 0;
            for (uint32_t j = 0; j < nl->nfo[g]; j++) {
                const uint64_t add = cnt[fanout(nl, g, j)];
                t = t + add < t ? UINT64_MAX : t + add;
            }
            nxt[g] = t;
        }
        uint64_t *tmp = cnt;
        cnt = nxt;
        nxt = tmp;
    }
    uint64_t S = 0;
    for (uint32_t g = 0; g < G; g++) S = S + cnt[g] < S ? UINT64_MAX : S + cnt[g];
    free(cnt);
    free(nxt);
    if (!out || cap < S || S == UINT64_MAX) return S;
    uint32_t path[8], idx[8];
    uint64_t s = 0;
    for (uint32_t g0 = 0; g0 < G; g0++) {
        int d = 0;
        path[0] = g0;
        idx[0] = 0;
        while (d >= 0) {
            if ((uint32_t)d == N - 1) {
                memcpy(out + s * N, path, N * sizeof(uint32_t));
                s++;
                d--;
                continue;
            }
            const uint32_t g = path[d];
            if (idx[d] < nl->nfo[g]) {
                path[d + 1] = fanout(nl, g, idx[d]++);
                idx[d + 1] = 0;
                d++;
            } else {
                d--;
            }
        }
    }
    return S;
}

/* kernSegmentReduce2<N> (mergekernel.cuh:116-198): the first pair marking every
 * net of the segment (has_marked_segment, :99-108), falling (x) or rising (y)
 * by the value of the segment's first net (:140-143), folded with min. */
int pdfo_merge_seg(const pdf_netlist *nl, const uint8_t *sim, const uint8_t *mark, uint64_t n_pairs,
                   uint64_t pair_base, uint32_t N, const uint32_t *segs, uint64_t S, uint32_t *seg_fx,
                   uint32_t *seg_fy) {
    (void)nl;
    for (uint64_t s = 0; s < S; s++) {
        const uint32_t *sg = segs + s * N;
        uint32_t fx = 0xFFFFFFFFu, fy = 0xFFFFFFFFu;
        for (uint64_t p = 0; p < n_pairs && (fx == 0xFFFFFFFFu || fy == 0xFFFFFFFFu); p++) {
            int all = 1;
            for (uint32_t i = 0; i < N && all; i++) all = mark[(uint64_t)sg[i] * n_pairs + p] != 0;
            if (!all) continue;
            const uint32_t pid = (uint32_t)(pair_base + p);
            if (sim[(uint64_t)sg[0] * n_pairs + p] & 1) {
                if (fy == 0xFFFFFFFFu) fy = pid;
            } else if (fx == 0xFFFFFFFFu) {
                fx = pid;
            }
        }
        if (fx < seg_fx[s]) seg_fx[s] = fx;
        if (fy < seg_fy[s]) seg_fy[s] = fy;
    }
    return 0;
}

/* kernCover<N> (coverkernel.cuh:171-230): a pair is first at net g when it is
 * the first pair of some segment through g (findActiveThreads, :130-154). */
int pdfo_cover_seg(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                   uint32_t N, const uint32_t *segs, uint64_t S, const uint32_t *seg_fx, const uint32_t *seg_fy,
                   uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads) {
    uint8_t *fp = (uint8_t *)calloc((size_t)nl->n_gates * n_pairs + 1, 1);
    if (!fp) return -1;
    for (uint64_t s = 0; s < S; s++) {
        const uint32_t f[2] = {seg_fx[s], seg_fy[s]};
        for (int k = 0; k < 2; k++) {
            if (f[k] == 0xFFFFFFFFu || f[k] < pair_base || f[k] - pair_base >= n_pairs) continue;
            for (uint32_t i = 0; i < N; i++) fp[(uint64_t)segs[s * N + i] * n_pairs + (f[k] - pair_base)] = 1;
        }
    }
    const int rc = cover_impl(nl, mark, n_pairs, pair_base, NULL, NULL, fp, NULL, lo, hi, flags, threads);
    free(fp);
    return rc;
}

/* The chunk loop of main.cu:171-231 with segments of length N: sim, mark,
 * gpuMergeSegments<N>, gpuCountPaths<N> per chunk; seg_fx / seg_fy hold S
 * entries (segments as listed by pdfo_segments). */
int pdfo_grade_seg(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs, uint64_t pair_base,
                   int mark_mode, uint64_t chunk, uint32_t N, const uint32_t *segs, uint64_t S, uint32_t *seg_fx,
                   uint32_t *seg_fy, uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads) {
    const uint32_t G = nl->n_gates;
    const uint32_t n_pi = nl->level_offsets[1];
    if (chunk == 0 || chunk > n_pairs) chunk = n_pairs ? n_pairs : 1;
    uint8_t *pi = (uint8_t *)malloc((size_t)n_pi * chunk + 1);
    uint8_t *sim = (uint8_t *)malloc((size_t)G * chunk + 1);
    uint8_t *mark = (uint8_t *)malloc((size_t)G * chunk + 1);
    int rc = (!pi || !sim || !mark) ? -1 : 0;
    for (uint64_t start = 0; rc == 0 && start < n_pairs; start += chunk) {
        const uint64_t K = n_pairs - start < chunk ? n_pairs - start : chunk;
        for (uint32_t i = 0; i < n_pi; i++)
            memcpy(pi + (uint64_t)i * K, pi_codes + (uint64_t)i * n_pairs + start, K);
        pdfo_sim_mode(nl, pi, K, sim, mark_mode, threads);
        pdfo_mark(nl, sim, K, mark_mode, mark, 1, threads);
        pdfo_merge_seg(nl, sim, mark, K, pair_base + start, N, segs, S, seg_fx, seg_fy);
        uint64_t clo = 0, chi = 0;
        uint32_t cfl = 0;
        rc = pdfo_cover_seg(nl, mark, K, pair_base + start, N, segs, S, seg_fx, seg_fy, &clo, &chi, &cfl, threads);
        if (rc) break;
        u128 cur = ((u128)*hi << 64) | *lo;
        int o = 0;
        cur = sat_add(cur, ((u128)chi << 64) | clo, &o);
        if (o || (cfl & PDF_FLAG_OVERFLOW)) *flags |= PDF_FLAG_OVERFLOW;
        *lo = (uint64_t)cur;
        *hi = (uint64_t)(cur >> 64);
    }
    free(pi);
    free(sim);
    free(mark);
    return rc;
}
