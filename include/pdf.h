/*
 * pdf.h -- C ABI of the B200 path-delay-fault grader.
 *
 * The grader takes a levelized combinational netlist and a batch of two-pattern
 * vector pairs and produces, per (net, pair), a 2-bit transition code and a
 * robust path mark, per net the first pair index that marks it with a falling
 * and with a rising transition, and the exact number of covered paths.
 *
 * Every entry point returns a pdf_status and never exits or traps.  Host
 * buffers are caller-owned; device memory behind a pdf_circuit / pdf_state is
 * library-owned.  Streams are passed as `void *` (a cudaStream_t, NULL = the
 * legacy default stream) so that no CUDA or torch type appears here.
 *
 * Reference interface replaced (lordofhyphens/gpu-path-delay-coverage):
 *   gpuRunSimulation   simkernel.cuh:16,200     -> pdf_sim
 *   gpuMarkPaths       markkernel.cuh:31,295    -> pdf_mark
 *   gpuMergeSegments<1> mergekernel.cuh:200-201 -> pdf_merge
 *   gpuCountPaths<1>   coverkernel.cuh:233-235  -> pdf_cover
 *   the chunk loop     main.cu:171-231          -> pdf_grade
 *   GPU_Circuit::copy  main.cu:137              -> pdf_circuit_create
 *   dc_seglist + totals main.cu:141,169,224     -> pdf_state_*
 */
#ifndef PDF_H
#define PDF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDF_ABI_VERSION 2

typedef enum pdf_status {
    PDF_OK = 0,
    PDF_EINVAL = 1,     /* malformed argument or netlist */
    PDF_ENOMEM = 2,     /* device or host allocation failed / admission refused */
    PDF_EOVERFLOW = 3,  /* a path count does not fit in 128 bits */
    PDF_ETIMEOUT = 4,   /* a bounded device-side wait gave up */
    PDF_ECUDA = 5,      /* a CUDA runtime call failed */
    PDF_ENOTSUP = 6,    /* not supported for these options or on this device */
    PDF_EBUSY = 7,      /* resource in use (serving queue full, job still running) */
    PDF_ENODEV = 8,     /* no CUDA device */
    PDF_ELIMIT = 9      /* request larger than the fixed scratch of pdf_cover_noalloc */
} pdf_status;

/* Gate type codes.  AND..XNOR must be 2..7: the reference indexes its robust
 * sensitisation table with (type - 2) (markkernel.cuh:36-37,49). */
enum {
    PDF_UNKN = 0,
    PDF_INPT = 1,
    PDF_AND = 2,
    PDF_NAND = 3,
    PDF_OR = 4,
    PDF_NOR = 5,
    PDF_XOR = 6,
    PDF_XNOR = 7,
    PDF_BUFF = 8,
    PDF_NOT = 9,
    PDF_FROM = 10,
    PDF_DFF = 11,
    PDF_NTYPES = 12
};

/* 2-bit transition codes: bit0 = value under the second vector, bit1 = the
 * value changed (simkernel.cuh:164, markkernel.cuh:230, mergekernel.cuh:141-146).
 * T0 is a falling transition, T1 a rising one. */
enum { PDF_S0 = 0, PDF_S1 = 1, PDF_T0 = 2, PDF_T1 = 3 };

/* Result flags (pdf_totals.flags). */
#define PDF_FLAG_OVERFLOW 0x1u   /* some count exceeded 2^128 - 1; totals are saturated */

/*
 * A levelized netlist (the data contract of the reference's GPU_Circuit:
 * GPUNODE{type,nfi,nfo,offset,po} and the FIN edge array,
 * simkernel.cuh:108-145, markkernel.cuh:220-223,277, coverkernel.cuh:205).
 *
 * Gate ids are in level order: level l holds gates
 * [level_offsets[l], level_offsets[l+1]).  Level 0 holds the primary inputs
 * (type PDF_INPT) and nothing else.  Every fan-in of a gate lies on a lower
 * level.  For gate g, edges[edge_offset[g] + j] (j < nfi[g]) are its fan-ins
 * in order (fan-in 0 first) and edges[edge_offset[g] + nfi[g] + k]
 * (k < nfo[g]) its fan-outs.  The fan-out lists must be exactly the transpose
 * of the fan-in lists (as multisets).  po[g] != 0 marks a primary output.
 */
typedef struct pdf_netlist {
    uint32_t n_gates;
    uint32_t n_levels;              /* number of levels, >= 1 */
    const uint32_t *level_offsets;  /* n_levels + 1 entries */
    const uint8_t *type;            /* n_gates */
    const uint8_t *po;              /* n_gates */
    const uint32_t *nfi;            /* n_gates */
    const uint32_t *nfo;            /* n_gates */
    const uint64_t *edge_offset;    /* n_gates */
    const uint32_t *edges;
    uint64_t n_edges;               /* length of edges[] */
} pdf_netlist;

/*
 * Vector pairs as two bit-planes per primary input.  For PI i (the i-th gate
 * of level 0) and pair p, bit (p % 32) of v[i * ld + p / 32] is the value
 * under the second vector (code bit 0) and the same bit of t[] is the
 * transition flag (code bit 1).  Bits at pair indices >= n_pairs are ignored.
 */
typedef struct pdf_pairs {
    const uint32_t *v;
    const uint32_t *t;
    uint64_t n_pairs;
    uint64_t ld;        /* words per PI row, >= ceil(n_pairs / 32) */
    int on_device;      /* 1: v, t are device pointers on the circuit's device */
} pdf_pairs;

/*
 * Optional per-(net, pair) outputs, gate-major bit-planes: bit (p % 32) of
 * word [g * ld + p / 32].  sim_v / sim_t are the two code bits of the
 * simulated transition value, mark the robust mark after pruning.  Any pointer
 * may be NULL.  Bits at pair indices >= n_pairs are written as 0.
 */
typedef struct pdf_outputs {
    uint32_t *sim_v;
    uint32_t *sim_t;
    uint32_t *mark;
    uint64_t ld;        /* words per gate row, >= ceil(n_pairs / 32) */
    int on_device;
} pdf_outputs;

/* 128-bit path totals. */
typedef struct pdf_totals {
    uint64_t lo;
    uint64_t hi;
    uint64_t pairs;     /* pairs graded */
    uint32_t flags;     /* PDF_FLAG_* */
    uint32_t reserved;
} pdf_totals;

typedef struct pdf_circuit pdf_circuit;
typedef struct pdf_state pdf_state;

/* Semantics and sensitisation table.  The reference reads one of two tables
 * (markkernel.cuh:36-37, selected at :255-259 by --robust, main.cu:53); the
 * first two modes reproduce it exactly, quirks included (multi-input gates
 * as a left fold of the 2-input table, XOR/XNOR with several fan-ins S0, the
 * mark of fan-in 0 required for every on-path candidate).
 *
 * The FIXED modes have no reference counterpart: AND..XNOR are true n-input
 * functions (XOR/XNOR evaluated, NAND(a) = NOT a), and a gate is marked when
 * its output transitions and some fan-in i carries a mark and a transition
 * with every other fan-in passing the side-input table for (i, other):
 *   FIXED_ROBUST     AND/NAND: on T0 -> side S1 or T1, on T1 -> side S1
 *                    OR/NOR:   on T0 -> side S0, on T1 -> side S0 or T0
 *                    XOR/XNOR: side S0 or S1          {0x2A00,0x2A00,0x5100,0x5100,0x3300,0x3300}
 *   FIXED_NONROBUST  side final value non-controlling (S1/T1 for AND/NAND,
 *                    S0/T0 for OR/NOR), any side for XOR/XNOR
 *                                                     {0xAA00,0xAA00,0x5500,0x5500,0xFF00,0xFF00}
 * Pruning, merge and cover are the same in every mode. */
enum {
    PDF_MARK_DEFAULT = 0,          /* LUT_NR: {0x2A00,0x2A00,0x5100,0x5100,0,0} (no --robust) */
    PDF_MARK_ROBUST = 1,           /* LUT_R:  {0x2200,0x2200,0x1100,0x1100,0,0} (--robust)    */
    PDF_MARK_FIXED_ROBUST = 2,     /* textbook robust, true n-input gates */
    PDF_MARK_FIXED_NONROBUST = 3   /* textbook non-robust, true n-input gates */
};

typedef struct pdf_circuit_opts {
    int device;          /* CUDA device ordinal */
    int mark_mode;       /* PDF_MARK_* */
    uint32_t max_pairs;  /* largest batch this circuit will grade (sizes scratch); 0 = 65536 */
    uint32_t tile_words; /* words (32 pairs) per CTA column block: 1, 2, 4, 8 (a thread per gate)
                            or 32, 64, 128 (the lane kernel: a warp per gate, 1, 2 or 4 words
                            per lane, for wide levels); 0 = chosen: a lane tile when max_pairs
                            gives >= 1 1,024-pair block per SM and the levels average >= 1,024
                            gates (the one with the least modelled time), else 8 when max_pairs
                            gives >= 2 8-word CTAs per SM, else 4 */
    uint32_t threads;    /* 0 = piece capacity + 64 (lane tiles: 1,024, or 512 at 128 words);
                            else threads per CTA: 64..1024, a multiple of 32, capped at the
                            lane tile's default; from 128 up, pieces of the thread-per-gate
                            tiles then hold at most threads - 64 gates */
    uint32_t seg_len;    /* path segments of this many nets, 0 or 1 = single nets; up to 8
                            (fcount --segs N, main.cu:76-81,185-223) */
    uint32_t wait_polls; /* bound on each device-side wait of the forward kernels for its staged
                            copy: 0 = 2^24 blocking polls (the default); n > 0 = n non-blocking
                            polls, after which the call reports PDF_ETIMEOUT (small values
                            exist to test that path).  The lane kernel (tile_words 32, 64,
                            128) waits for nothing. */
    uint32_t reserved;
} pdf_circuit_opts;

typedef struct pdf_circuit_info {
    uint32_t n_gates, n_levels, n_pi, n_po;
    uint32_t max_level_width;
    uint32_t max_nfi, max_nfo;
    uint32_t tile_words, threads;
    uint64_t n_edges;
    uint64_t device_bytes;   /* netlist + plan + scratch */
    uint64_t max_pairs;
    uint32_t seg_len;        /* 1, or the segment length */
    uint32_t reserved;
    uint64_t n_segments;     /* entries of a state's first-detect arrays: n_gates, or the segments */
} pdf_circuit_info;

const char *pdf_status_string(int status);
/* The last CUDA failure behind a PDF_ECUDA / PDF_ENOMEM of this thread: the
 * CUDA error name and number and the failing call ("" if none yet). */
const char *pdf_last_error(void);
int pdf_abi_version(void);

/* Host-side fault injection, for tests of the error paths (no reference
 * counterpart).  The next `count` allocations of the given kind made by this
 * library fail as if memory were exhausted (count 0 clears it):
 * PDF_INJECT_DEVICE_ALLOC  device memory of circuits, states and workspaces;
 * PDF_INJECT_HOST_ALLOC    the pinned read-back staging of the server.
 * Process-wide; calls that then fail return PDF_ENOMEM and leave their
 * objects usable. */
enum { PDF_INJECT_DEVICE_ALLOC = 1, PDF_INJECT_HOST_ALLOC = 2 };
pdf_status pdf_test_inject(int site, uint32_t count);

/* Host-side structural check of a netlist (no device needed).  On failure a
 * one-line reason is written to msg (if msg_len > 0). */
pdf_status pdf_netlist_check(const pdf_netlist *nl, char *msg, size_t msg_len);

/* Upload a netlist to a device (GPU_Circuit::copy, main.cu:137). */
pdf_status pdf_circuit_create(const pdf_netlist *nl, const pdf_circuit_opts *opts,
                              pdf_circuit **out);
void pdf_circuit_destroy(pdf_circuit *c);
pdf_status pdf_circuit_query(const pdf_circuit *c, pdf_circuit_info *info);

/*
 * Segments (seg_len N = 2..8; the reference's --segs, with its segment list
 * from the util/segment.cuh that its snapshot lacks): every directed subpath
 * of exactly N nets (g_0, ..., g_{N-1}), g_{i+1} a fan-out of g_i, listed by
 * g_0 ascending, then depth first along fan-outs in edge order.  A segment's
 * first pair is the first pair marking all its nets, falling (x) or rising
 * (y) by the value of g_0 (mergekernel.cuh:99-198); in the cover a pair is
 * first at a net when it is the first pair of a segment through that net
 * (coverkernel.cuh:115-170).  With N = 1 the segments are the nets.  State
 * first-detect arrays then hold info.n_segments entries, one per segment.
 * Segment lists beyond 2^28 gate ids return PDF_ENOTSUP; batches, the server
 * and pdf_cover_noalloc grade single nets only (PDF_ENOTSUP).
 * pdf_circuit_segments writes the list as gates[s * N + i] (n_segments * N
 * entries; for N = 1 the identity).
 */
pdf_status pdf_circuit_segments(const pdf_circuit *c, uint32_t *gates);

/* Per-circuit first-detect state and running total: the reference keeps the
 * per-segment first pair ids in dc_seglist across chunks and the total in
 * *totals (main.cu:141,169,224; mergekernel.cuh:205-222).  first_x = first
 * pair marking the net with a falling (T0) transition, first_y = rising (T1);
 * 0xFFFFFFFF = none yet.  The arrays hold info.n_segments entries: one per
 * net (n_gates), or one per segment when seg_len > 1. */
pdf_status pdf_state_create(pdf_circuit *c, pdf_state **out);
/* A state may be destroyed before or after its circuit. */
void pdf_state_destroy(pdf_state *s);
pdf_status pdf_state_reset(pdf_state *s);
/* Synchronises with the state's last grading call. Any pointer may be NULL. */
pdf_status pdf_state_snapshot(pdf_state *s, uint32_t *first_x, uint32_t *first_y,
                              pdf_totals *totals);
pdf_status pdf_state_restore(pdf_state *s, const uint32_t *first_x,
                             const uint32_t *first_y, const pdf_totals *totals);
/* pdf_state_snapshot ordered on `stream` (the stream of the state's last
 * grading call): copies after the work queued there and waits for that
 * stream only, not for the whole device, so copies and kernels of other
 * streams (another circuit's uploads, say) do not hold it up.  (No reference
 * counterpart: the reference reads *totals after a device-wide sync,
 * main.cu:224.) */
pdf_status pdf_state_snapshot_on(pdf_state *s, uint32_t *first_x, uint32_t *first_y,
                                 pdf_totals *totals, void *stream);

/* Stream-ordered reset: clears the state on `stream` without waiting. */
pdf_status pdf_state_reset_async(pdf_state *s, void *stream);
/* Allocate now the device workspace that grading batches of up to n_pairs
 * pairs needs (otherwise allocated by the first such call). */
pdf_status pdf_state_reserve(pdf_state *s, uint64_t n_pairs);

/* Device timing of grading calls with CUDA events on the grading stream.
 * enable = 1 clears and starts recording, 0 stops.  pdf_state_profile_read
 * waits for the recorded calls and returns, summed over them, ms[0] = the
 * forward kernel (sim + mark + prune + merge), ms[1] = the cover kernels,
 * ms[2] = the whole call; *calls = calls recorded. */
pdf_status pdf_state_profile(pdf_state *s, int enable);
pdf_status pdf_state_profile_read(pdf_state *s, double *ms, uint32_t *calls);

/*
 * Grade one batch of pairs with global pair indices pair_base .. pair_base +
 * n_pairs - 1 (the chunk loop body, main.cu:171-231): simulate, mark, prune,
 * fold the first-detecting pairs into the state and add the batch's covered
 * path count to the state's total.  Batches of one state must come in
 * increasing pair order for the result to be independent of the batching.
 *
 * pdf_grade_async only enqueues work on `stream`; pdf_grade also waits and
 * returns this batch's count in *batch (may be NULL).
 */
pdf_status pdf_grade_async(pdf_circuit *c, pdf_state *s, const pdf_pairs *pairs,
                           uint64_t pair_base, const pdf_outputs *out, void *stream);
pdf_status pdf_grade(pdf_circuit *c, pdf_state *s, const pdf_pairs *pairs,
                     uint64_t pair_base, const pdf_outputs *out, pdf_totals *batch,
                     void *stream);

/*
 * The two halves of pdf_grade_async, for callers that combine first-detect
 * ids of several states between them (pairs sharded over GPUs: each rank
 * marks its own pairs, the ranks reduce first_x/first_y with an unsigned MIN,
 * then each rank counts its pairs).  pdf_grade_mark_async runs sim, mark,
 * prune and merge into the state and writes the outputs;
 * pdf_grade_cover_async counts the paths of that batch against the state's
 * current first-detect ids.  No reference counterpart: the reference is
 * single-GPU (main.cu:34).
 */
pdf_status pdf_grade_mark_async(pdf_circuit *c, pdf_state *s, const pdf_pairs *pairs,
                                uint64_t pair_base, const pdf_outputs *out, void *stream);
pdf_status pdf_grade_cover_async(pdf_circuit *c, pdf_state *s, void *stream);
/* Stream-ordered copy of the state's first-detect ids to (to_state = 0) or
 * from (to_state = 1) device buffers of info.n_segments uint32 each (n_gates
 * for single nets). */
pdf_status pdf_state_first_copy(pdf_state *s, uint32_t *first_x, uint32_t *first_y, int to_state,
                                void *stream);

/*
 * Stage calls, one per reference host function, over device buffers in the
 * pdf_outputs plane layout (gate-major, ld words per row).  They compose to
 * exactly what pdf_grade computes.
 */
/* gpuRunSimulation (simkernel.cuh:200-249): transition codes of every net. */
pdf_status pdf_sim(pdf_circuit *c, const pdf_pairs *pairs, uint32_t *sim_v,
                   uint32_t *sim_t, uint64_t ld, void *stream);
/* gpuMarkPaths (markkernel.cuh:295-355): forward robust marks, then removal of
 * marks that reach no primary output. */
pdf_status pdf_mark(pdf_circuit *c, const uint32_t *sim_v, const uint32_t *sim_t,
                    uint32_t *mark, uint64_t n_pairs, uint64_t ld, void *stream);
/* The forward marks alone, before the removal pass: the first level loop of
 * gpuMarkPaths (markkernel.cuh:297-322), dumped as gpumark-full.log (:323-324). */
pdf_status pdf_mark_forward(pdf_circuit *c, const uint32_t *sim_v, const uint32_t *sim_t,
                            uint32_t *mark, uint64_t n_pairs, uint64_t ld, void *stream);
/* gpuMergeSegments<1> (mergekernel.cuh:200-267): fold the first marking pair
 * of every net (split by transition direction) into the state. */
pdf_status pdf_merge(pdf_circuit *c, pdf_state *s, const uint32_t *sim_v,
                     const uint32_t *mark, uint64_t n_pairs, uint64_t ld,
                     uint64_t pair_base, void *stream);
/* gpuCountPaths<1> (coverkernel.cuh:233-333): count covered paths of this
 * chunk against the state's first-detect ids, add them to the state's total
 * and (synchronously) return the chunk's count in *chunk_total. */
pdf_status pdf_cover(pdf_circuit *c, pdf_state *s, const uint32_t *mark,
                     uint64_t n_pairs, uint64_t ld, uint64_t pair_base,
                     pdf_totals *chunk_total, void *stream);

/* pdf_cover that also returns, in host memory, the paths each primary input
 * credits to each pair of the chunk: counts[(i * n_pairs + p) * 2] and
 * [... + 1] are the low and high 64 bits of input i's count for pair p
 * (n_pi x n_pairs x 16 bytes).  These are the per-(input, pair) values the
 * reference writes to gpucover.log in debug builds (debugCover,
 * coverkernel.cuh:44-66,242-248), here exact; their sum is the chunk count. */
pdf_status pdf_cover_counts(pdf_circuit *c, pdf_state *s, const uint32_t *mark, uint64_t n_pairs,
                            uint64_t ld, uint64_t pair_base, uint64_t *counts, pdf_totals *chunk_total,
                            void *stream);

/*
 * pdf_cover without any allocation.  No counterpart in the reference (whose
 * gpuCountPaths allocates per chunk, coverkernel.cuh:256-275).
 *
 * For callers that may not enter the CUDA allocator while they grade: a host
 * framework that owns all device memory through its own pool, or a
 * latency-bound loop in which a cudaMalloc could synchronise the device or
 * fail under memory pressure.  The circuit is created once beforehand
 * (pdf_circuit_create allocates); this call then allocates and frees nothing.
 * Its scratch is one fixed array of 8 MiB in device memory, held by every GPU
 * that loads the library until the process exits; a chunk needs
 * 4 * (ceil(ceil(n_pairs/32)/tile_words) * ceil(n_gates/32)
 *      + ceil(n_pairs/32) + min(n_pairs, 2 * n_gates)) bytes of it plus about
 * 1 KiB, and larger requests return PDF_ELIMIT (a circuit with segments of
 * more than one net gets PDF_ENOTSUP before any size check: the fixed array
 * holds no (net, pair) set).  The caller passes the
 * pruned mark plane (as pdf_cover) and the first-detect ids as device arrays
 * of n_gates uint32 (for example copied out with pdf_state_first_copy); the
 * chunk's count is returned in *chunk_total (the call waits for it).
 * The first call on each device looks up the array's device address; make
 * that first call before any stream capture.  All calls on a device share the
 * array, so calls that overlap on the GPU race: serialise them.
 */
pdf_status pdf_cover_noalloc(pdf_circuit *c, const uint32_t *mark, uint64_t n_pairs, uint64_t ld,
                             uint64_t pair_base, const uint32_t *first_x, const uint32_t *first_y,
                             pdf_totals *chunk_total, void *stream);

/* ---- batched grading: many circuits in one pass ---- */

/*
 * A batch grades the vector pairs of many (circuit, state) jobs in one pass of
 * a few kernel launches, captured once as a CUDA graph and replayed by each
 * pdf_batch_run.  Each job's result is the same as pdf_grade of that job alone
 * (its state's first-detect ids and totals).  No reference counterpart: the
 * reference grades one circuit per process (main.cu:129-235).
 *
 * Jobs borrow their circuit and state (both must outlive the batch, and the
 * state must not be graded elsewhere meanwhile); all circuits share one
 * device, mark mode and tile width.  pairs are device planes (on_device = 1,
 * ld a multiple of the tile width, 16-byte aligned rows) that stay bound to the
 * batch: rewrite their contents between runs to grade new pairs.  With
 * PDF_BATCH_APPEND each run also advances every job's pair_base by its pair
 * count, so consecutive runs grade consecutive batches of each job's pairs
 * (as consecutive pdf_grade calls would).
 */
typedef struct pdf_batch pdf_batch;
typedef struct pdf_batch_job {
    pdf_circuit *circuit;
    pdf_state *state;
    pdf_pairs pairs;
    uint64_t pair_base; /* global id of the job's first pair in the first run */
} pdf_batch_job;
enum {
    PDF_BATCH_APPEND = 1,   /* each run advances every job's pair_base by its pair count */
    PDF_BATCH_NO_GRAPH = 2  /* launch the kernels directly instead of replaying a captured graph
                               (for batches rebuilt often, or when other host threads make
                               device-synchronising CUDA calls while a run might capture) */
};
typedef struct pdf_batch_info {
    uint32_t n_jobs, tile_words, threads, ctas;
    uint64_t gate_evals; /* per run: sum over jobs of n_gates * n_pairs */
    uint64_t device_bytes;
    uint32_t launches;   /* kernel launches per run: the forward launches, then k_batch_active,
                            the small- and large-table passes of k_batch_cover and (when a
                            circuit may spill) k_batch_cover_spill */
    uint32_t forward_launches; /* one per class of tile width and CTAs per SM */
} pdf_batch_info;
pdf_status pdf_batch_create(const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags, pdf_batch **out);
void pdf_batch_destroy(pdf_batch *b);
/* Point an existing batch at another set of jobs (same rules as
 * pdf_batch_create; same device).  Its device memory is reused when large
 * enough, so a loop whose job set changes often allocates and frees little.
 * No run of the batch may be in flight.  On failure the batch must not be
 * run until a rebind succeeds. */
pdf_status pdf_batch_rebind(pdf_batch *b, const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags);
pdf_status pdf_batch_query(const pdf_batch *b, pdf_batch_info *info);
/* One pass over every job, stream-ordered (the first call captures the graph). */
pdf_status pdf_batch_run_async(pdf_batch *b, void *stream);
/* pdf_batch_run_async, then wait; reports a device-side error of any job. */
pdf_status pdf_batch_run(pdf_batch *b, void *stream);
/* Timing of a batch's passes (no reference counterpart).  With enable != 0
 * every later run records CUDA events on the run's stream (as event nodes of
 * the captured graph) before the forward launches, after they have all
 * joined, and after the cover; pdf_batch_profile_read waits for the most
 * recent run and returns ms[0] = its forward span (every class's forward
 * launch, side by side) and ms[1] = its cover (k_batch_active + k_batch_cover).
 * Switching profiling on or off recaptures the graph at the next run. */
pdf_status pdf_batch_profile(pdf_batch *b, int enable);
pdf_status pdf_batch_profile_read(pdf_batch *b, double ms[2]);

/*
 * Autotuner of the batch's tile shape: for each candidate (tile width in words
 * of 32 pairs per CTA: 2, 4, 8; block size: the default, piece capacity + 64,
 * or 256 threads, pieces of 192 gates; base->threads, when set, fixes the
 * block size) it builds the circuits, states and pair planes of the given
 * netlists and pair counts (seeded pairs), times `reps` graph replays after a
 * warm-up, and returns the fastest options in *best (tile_words and threads;
 * the other fields copied from *base) with its milliseconds per run in
 * *best_ms.  All it allocates is freed before it returns.
 */
pdf_status pdf_batch_autotune(const pdf_netlist *const *netlists, const uint64_t *n_pairs, uint32_t n,
                              const pdf_circuit_opts *base, uint32_t reps, pdf_circuit_opts *best,
                              float *best_ms);

/* ---- serving: continuous batching of grading jobs ---- */

/*
 * A server grades jobs that arrive over time.  A job is a netlist plus all
 * its vector pairs (host planes, kept by the caller until the job is done);
 * it is graded in batches of `batch_pairs` pairs that append to the job's
 * device-resident coverage state.  Each pdf_server_step admits queued jobs
 * in arrival order while their device footprint fits `hbm_budget` (and
 * fewer than `max_jobs` are active), enqueues the next batch of every active
 * job as one batched pass (pdf_batch_*), then waits for the pass the step
 * before enqueued and retires the jobs whose pairs that pass finished
 * grading (their results stay readable).  So one pass stays in flight while
 * the caller's thread works between steps, and a job retires at the step
 * after its last batch was enqueued.  Jobs that arrive meanwhile join at the
 * next step, so work of jobs of different ages overlaps on the device.  A job's result equals pdf_grade of all its pairs in batches of
 * batch_pairs.  Per-batch latency is the time from the batch being ready
 * (submission, or the previous batch's end) to its result.  No reference
 * counterpart: the reference grades one circuit per process (main.cu).
 */
typedef struct pdf_server pdf_server;
typedef struct pdf_server_opts {
    int device;
    int mark_mode;          /* PDF_MARK_* for every job */
    uint32_t tile_words;    /* as pdf_circuit_opts.tile_words, for every job; 0 = 4 */
    uint32_t batch_pairs;   /* pairs per batch, a multiple of 32 (0 = 4096) */
    uint32_t max_jobs;      /* active jobs at most (0 = 1024) */
    uint32_t workers;       /* host threads preparing admitted jobs (0 = 4) */
    uint64_t hbm_budget;    /* bytes of device memory for active jobs (0 = half the free memory) */
} pdf_server_opts;
typedef struct pdf_server_stats {
    uint64_t jobs_done, jobs_active, jobs_queued;
    uint64_t batches;       /* job batches graded */
    uint64_t steps;         /* batched passes run */
    uint64_t gate_evals;    /* graded so far */
    double busy_s;          /* time inside pdf_server_step */
    double lat_p50_ms, lat_p99_ms, lat_max_ms; /* per-batch latency */
    uint64_t bytes_in_use;
    uint64_t launches;      /* kernel launches of the batched passes */
    double gpu_s;           /* device time of the batched passes (forward launches and cover) */
} pdf_server_stats;
pdf_status pdf_server_create(const pdf_server_opts *opts, pdf_server **out);
void pdf_server_destroy(pdf_server *srv);
/* Queue a job: v, t are host planes [n_pi][ld] of n_pairs pairs. */
pdf_status pdf_server_submit(pdf_server *srv, const pdf_netlist *nl, const uint32_t *v, const uint32_t *t,
                             uint64_t ld, uint64_t n_pairs, uint64_t *job_id);
/* One step; *retired gets the number of jobs that finished in it.  Call it
 * until every job has retired: a step with no job to grade still completes
 * the pass in flight. */
pdf_status pdf_server_step(pdf_server *srv, uint32_t *retired);
/* Result of a finished job: its total (and first-detect ids, if non-null, n_gates each).
 * PDF_EINVAL while the job is still queued or active. */
pdf_status pdf_server_result(pdf_server *srv, uint64_t job_id, pdf_totals *total, uint32_t *first_x,
                             uint32_t *first_y);
pdf_status pdf_server_query(const pdf_server *srv, pdf_server_stats *stats);

/* ---- synthetic inputs (seeded, host-side) ---- */

typedef struct pdf_gen_params {
    uint64_t seed;
    uint32_t n_gates;     /* total, including the primary inputs */
    uint32_t n_pi;
    uint32_t n_po;
    uint32_t depth;       /* levels above the inputs; n_levels = depth + 1 */
    uint32_t fanin_min;   /* for AND..XNOR; NOT/BUFF take exactly 1 */
    uint32_t fanin_max;
    uint32_t fanout_dist; /* 0 = geometric, 1 = Zipf */
    double zipf_s;
    uint32_t fanout_max;  /* cap on fan-out (0 = none) */
    uint32_t type_mask;   /* bit per gate code drawn uniformly; 0 = AND..XNOR,NOT,BUFF */
    uint32_t reserved[4];
} pdf_gen_params;

typedef struct pdf_netbuf pdf_netbuf;  /* a library-owned host netlist */

pdf_status pdf_gen_netlist(const pdf_gen_params *p, pdf_netbuf **out);
pdf_status pdf_netbuf_from(const pdf_netlist *nl, pdf_netbuf **out);  /* deep copy */
void pdf_netbuf_view(const pdf_netbuf *b, pdf_netlist *view);
void pdf_netbuf_free(pdf_netbuf *b);

/* Uniform random pairs: every code bit of every (PI, pair) independent and
 * uniform.  Writes n_pi rows of ld words into v and t (host memory); bits at
 * pair indices >= n_pairs are 0. */
pdf_status pdf_gen_pairs(uint64_t seed, uint32_t n_pi, uint64_t n_pairs, uint64_t ld,
                         uint32_t *v, uint32_t *t);

/* Reference-compatible pair formation from one vector stream
 * (simkernel.cuh:115-124): pair p = (vector p, vector p+1); the last pair wraps
 * to vector 0.  vec is n_pi rows of n_vec bytes (0/1).  Produces n_vec pairs. */
pdf_status pdf_pairs_from_vectors(const uint8_t *vec, uint32_t n_pi, uint64_t n_vec,
                                  uint64_t ld, uint32_t *v, uint32_t *t);

/* ---- netlist and vector files, debug dumps (the fcount command line) ---- */

/*
 * The reference reads circuits and vectors through its util/ submodule
 * (Circuit::read_bench, Circuit::load, get_vector_dim, read_vectors;
 * main.cu:128-156), which the reference snapshot does not contain; these
 * formats are this library's own.
 *
 * ISCAS .bench: INPUT(n), OUTPUT(n), n = TYPE(a, b, ...) with TYPE one of
 * AND NAND OR NOR XOR XNOR NOT BUF BUFF FROM DFF, '#' comments.  Flip-flops are
 * cut for full scan: the output of q = DFF(d) becomes a primary input (after
 * the declared inputs) and d a primary output.  Gates are levelized (level =
 * longest distance from an input) and numbered by level, then file order.
 * PDF_BENCH_BRANCHES inserts a FROM gate on every fan-out branch of a net
 * read more than once.  On error, msg (if given) names the file and line.
 */
#define PDF_BENCH_BRANCHES 0x1u
pdf_status pdf_read_bench(const char *path, uint32_t flags, pdf_netbuf **out, char *msg, size_t msg_len);
/* Writes gates as g<id>; reading it back gives the same netlist when its
 * levels are longest-path levels, it has no DFF gates and fan-outs are listed
 * in consumer order. */
pdf_status pdf_write_bench(const pdf_netlist *nl, const char *path);
/* Levelized text: a line "pdf-level 1", a line "n_gates n_levels", then one
 * line per gate in id order: "id level TYPE po nfi fan-ins... nfo fan-outs...".
 * Round-trips every field of a pdf_netlist. */
pdf_status pdf_read_level(const char *path, pdf_netbuf **out, char *msg, size_t msg_len);
pdf_status pdf_write_level(const pdf_netlist *nl, const char *path);
/* Vector files: one vector per line, one '0'/'1' per primary input
 * (whitespace ignored, '#' comments).  pdf_vectors_dim returns the vector
 * count and width (get_vector_dim); pdf_vectors_read fills vec[n_pi][n_vec]
 * (the layout pdf_pairs_from_vectors takes) and fails unless the file holds
 * exactly n_vec vectors of n_pi bits. */
pdf_status pdf_vectors_dim(const char *path, uint64_t *n_vec, uint32_t *width);
pdf_status pdf_vectors_read(const char *path, uint32_t n_pi, uint64_t n_vec, uint8_t *vec);
/* Text dumps of host planes in the reference's debug-log layouts: a header of
 * gate ids then one line per pair, "Vector <pair_base + p>:" and a code per
 * gate (S0/S1/T0/T1; debugSimulationOutput, simkernel.cuh:250-295) or a mark
 * (Y/N; debugMarkOutput, markkernel.cuh:357-394).  append != 0 adds lines to
 * an existing file without the header (later chunks).  pdf_dump_merge writes
 * "Gate <g>: x,y" per net with ids as signed 32-bit, -1 = none
 * (debugMergeOutput, mergekernel.cuh:269-284). */
pdf_status pdf_dump_sim(const char *path, const uint32_t *sim_v, const uint32_t *sim_t, uint32_t n_gates,
                        uint64_t n_pairs, uint64_t ld, uint64_t pair_base, int append);
pdf_status pdf_dump_mark(const char *path, const uint32_t *mark, uint32_t n_gates, uint64_t n_pairs,
                         uint64_t ld, uint64_t pair_base, int append);
pdf_status pdf_dump_merge(const char *path, const uint32_t *first_x, const uint32_t *first_y, uint32_t n_gates);
/* gpucover.log (debugCover, coverkernel.cuh:44-66): a header of the primary
 * inputs' gate ids, then per pair "Vector <pair_base + p>:" and the paths
 * each input credits to it, from pdf_cover_counts (exact decimal). */
pdf_status pdf_dump_cover(const char *path, const uint64_t *counts, uint32_t n_pi, uint64_t n_pairs,
                          uint64_t pair_base, int append);
/* Segments longer than one net: "Segment <s>(g_0,...,g_{N-1}): x,y" per
 * segment, ids signed (debugSegmentList, mergekernel.cuh:25-46). */
pdf_status pdf_dump_segments(const char *path, const uint32_t *gates, uint32_t seg_len, uint64_t n_segments,
                             const uint32_t *first_x, const uint32_t *first_y);

#ifdef __cplusplus
}
#endif
#endif /* PDF_H */
