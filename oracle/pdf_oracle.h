/*
 * pdf_oracle.h -- CPU oracle for the path-delay-fault grading path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, as the checker.
 *
 * A serial restatement (optionally OpenMP over pairs) of the reference's four
 * kernels with one byte per (gate, pair), exactly like the reference's
 * GPU_Data rows.  Path counts are exact 128-bit with saturation.
 *
 * Parity pinning: the reference ships no tests, fixtures or golden vectors;
 * the oracle is pinned by exhaustive known-answer tests of the reference's
 * lookup tables and by the reference's own kernels run through the harness in
 * oracle/refharness (fixtures under tests/golden/).
 */
#ifndef PDF_ORACLE_H
#define PDF_ORACLE_H

#include <stdint.h>
#include "pdf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Reference lookup tables (simkernel.cuh:158-165), indexed lut[r * 4 + val]. */
uint8_t pdfo_lut2(int type, uint8_t val, uint8_t r);
uint8_t pdfo_stable(uint8_t v1, uint8_t v2);
uint8_t pdfo_not(uint8_t v);
/* Reference sensitisation test LUT_16(LUT[type-2], on, off) (markkernel.cuh:36-41). */
int pdfo_sens(int mark_mode, int type, uint8_t on, uint8_t off);

/* Stage functions over byte arrays [n_gates][n_pairs]. */
int pdfo_sim(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs,
             uint8_t *sim, int threads);
/* pdfo_sim with the gate semantics of mark_mode (PDF_MARK_FIXED_* evaluate
 * AND..XNOR as true n-input functions; pdfo_sim is PDF_MARK_DEFAULT). */
int pdfo_sim_mode(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs,
                  uint8_t *sim, int mark_mode, int threads);
int pdfo_sim_vectors(const pdf_netlist *nl, const uint8_t *vec, uint64_t n_vec,
                     uint8_t *sim, int threads);
int pdfo_mark(const pdf_netlist *nl, const uint8_t *sim, uint64_t n_pairs, int mark_mode,
              uint8_t *mark, int prune, int threads);
int pdfo_merge(const pdf_netlist *nl, const uint8_t *sim, const uint8_t *mark,
               uint64_t n_pairs, uint64_t pair_base, uint32_t *first_x, uint32_t *first_y,
               int threads);
/* Adds the chunk's count to (*lo, *hi), sets PDF_FLAG_OVERFLOW in *flags. */
int pdfo_cover(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs,
               uint64_t pair_base, const uint32_t *first_x, const uint32_t *first_y,
               uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads);
/* pdfo_cover, also writing every primary input's count for every pair to
 * pi_counts[(i * n_pairs + p) * 2 + {0, 1}] (low, high 64 bits). */
int pdfo_cover_counts(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                      const uint32_t *first_x, const uint32_t *first_y, uint64_t *pi_counts, uint64_t *lo,
                      uint64_t *hi, uint32_t *flags, int threads);

/*
 * The reference's chunk loop (main.cu:171-231) over pi_codes [n_pi][n_pairs]:
 * for each chunk of `chunk` pairs, sim -> mark -> merge -> cover, adding into
 * (first_x, first_y, *lo, *hi, *flags).  sim_out / mark_out (optional,
 * [n_gates][n_pairs]) receive the per-(gate, pair) codes and pruned marks.
 * chunk_totals (optional) receives 2 words (lo, hi) per chunk.
 */
int pdfo_grade(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs,
               uint64_t pair_base, int mark_mode, uint64_t chunk,
               uint32_t *first_x, uint32_t *first_y, uint8_t *sim_out, uint8_t *mark_out,
               uint64_t *lo, uint64_t *hi, uint32_t *flags, uint64_t *chunk_totals,
               int threads);

/* Segments longer than one net (segs = N, 2..8): the list (count returned;
 * out[s * N + i] written when cap >= count), the merge into per-segment first
 * ids, the cover, and the chunk loop. */
uint64_t pdfo_segments(const pdf_netlist *nl, uint32_t N, uint32_t *out, uint64_t cap);
int pdfo_merge_seg(const pdf_netlist *nl, const uint8_t *sim, const uint8_t *mark, uint64_t n_pairs,
                   uint64_t pair_base, uint32_t N, const uint32_t *segs, uint64_t S, uint32_t *seg_fx,
                   uint32_t *seg_fy);
int pdfo_cover_seg(const pdf_netlist *nl, const uint8_t *mark, uint64_t n_pairs, uint64_t pair_base,
                   uint32_t N, const uint32_t *segs, uint64_t S, const uint32_t *seg_fx, const uint32_t *seg_fy,
                   uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads);
int pdfo_grade_seg(const pdf_netlist *nl, const uint8_t *pi_codes, uint64_t n_pairs, uint64_t pair_base,
                   int mark_mode, uint64_t chunk, uint32_t N, const uint32_t *segs, uint64_t S, uint32_t *seg_fx,
                   uint32_t *seg_fy, uint64_t *lo, uint64_t *hi, uint32_t *flags, int threads);

#ifdef __cplusplus
}
#endif
#endif
