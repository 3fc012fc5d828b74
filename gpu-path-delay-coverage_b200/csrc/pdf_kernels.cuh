// pdf_kernels.cuh -- launch interface between the host API and the kernels.
#ifndef PDF_KERNELS_CUH
#define PDF_KERNELS_CUH

#include <cuda_runtime.h>

#include <cstdint>

#include "pdf_device.cuh"

struct DevCircuit {
    const GateRec *rec;         // [n_gates]
    const uint32_t *edges;      // fan-ins then fan-outs per gate
    const uint32_t *level_off;  // [n_levels + 1]
    uint32_t n_gates, n_levels, n_pi;
};

// Kernel stage selection for the forward kernel.
enum FwdMode {
    FWD_FUSED = 0,   // sim from the PI planes, forward mark, prune, merge
    FWD_SIM = 1,     // sim only (pdf_sim)
    FWD_MARK = 2     // sim planes given; forward mark + prune (pdf_mark)
};

// Batch accumulators kept in device memory by a pdf_state.
struct DevAcc {
    unsigned long long batch_lo, batch_hi;  // this batch's count
    unsigned long long total_lo, total_hi;  // running total
    unsigned long long pairs;
    unsigned int flags;                     // PDF_FLAG_*
    unsigned int batch_flags;
    unsigned int err;                       // device-side error code (0 = none)
    unsigned int done;                      // cover CTAs finished (the last one closes the batch)
    unsigned int n_over;                    // pairs queued for the spill cover (more nets than the table)
    unsigned int done_over;                 // spill-cover CTAs finished
};

struct FwdArgs {
    DevCircuit c;
    const Piece *pieces;          // level-ordered runs of gates (the unit of staging and of sync)
    uint32_t n_pieces;
    uint32_t cap, ecap;           // gates / edge words per staging buffer
    const uint32_t *far_ids;      // per piece, the far fan-ins it reads (Piece::far_off / far_n),
                                  // each list padded to a multiple of 4 entries
    uint32_t farcap;              // slots per far buffer (>= every piece's far_n)
    const uint32_t *pi_v, *pi_t;  // [n_pi][pi_ld]
    uint64_t pi_ld;
    uint32_t *V, *T, *M;          // planes [n_gates][ld]
    uint64_t ld;
    uint32_t store_all;           // 1: write every plane row; 0: only the rows read back later
                                  // (RF_SPILL gates, gates with a forward mark)
    uint32_t no_prune;            // FWD_MARK: stop after the forward marks (no removal pass)
    uint32_t *nzb;                // [n_blocks][bm_words] gates with a nonzero mark
    uint32_t *blk_maxlvl;         // [n_blocks] highest level holding a mark (+1), 0 = none
    // lane kernel, fused: the same after the prune for each quarter (8 words)
    // of a column block, [n_blocks * 4][bm_words] and [n_blocks * 4] (the
    // cover's bitmaps; a bound for the level), or null
    uint32_t *nzb_fine, *maxlvl_fine;
    uint32_t bm_words;
    uint32_t bm_shared;           // 1: the bitmap lives in shared memory during the kernel
    uint32_t *first_x, *first_y;  // [n_gates] (FWD_FUSED only)
    DevAcc *acc;                  // FWD_FUSED: the batch count, zeroed by block 0 (may be null)
    uint32_t *active;             // FWD_FUSED: the cover's active-pair bitmap [W] + count, zeroed (may be null)
    uint32_t *err;                // device error word (PDF_ETIMEOUT on a wait that expired)
    uint32_t wait_polls;          // bound of the record waits: 0 = kSpinLimit blocking polls,
                                  // n = n non-blocking polls (tests of the timeout path)
    uint64_t n_pairs;
    uint32_t W;                   // ceil(n_pairs / 32)
    uint32_t pair_base;
    uint32_t ring_gates;          // forward ring slots R (power of two, >= cap)
    uint32_t ring2_gates;         // reverse ring slots (power of two, or 0)
    // shared-memory byte offsets
    uint32_t off_ring;            // forward: ring [3][R][BW]; reverse: ring2 [R2][BW]
    uint32_t off_rec;             // [2][cap] staged gate records
    uint32_t off_edge;            // reverse: [2][ecap] staged edges; forward: far buffers [2][3][farcap][BW]
    uint32_t off_fid;             // forward: [2][farcap] staged far ids of the piece after the staged one
    uint32_t off_bm, off_pbits, off_mbar;
};

// Device error bits (DevAcc::err and the circuit's error word).
constexpr unsigned int kErrTimeout = 0x4u;     // a bounded wait expired (PDF_ETIMEOUT)
constexpr unsigned int kErrHashFull = 0x100u;  // a pair marked more nets than the cover table holds

// Segments longer than one net (seg_len N = 2..8): directed subpaths of N
// nets, listed by first net (CSR over it).
struct SegArgs {
    const uint32_t *segs;     // [S][N] gate ids
    const uint32_t *seg_off;  // [n_gates + 1]: segments starting at net g are [seg_off[g], seg_off[g + 1])
    uint32_t N;               // 0 or 1: per-net first ids (no segment list)
    uint32_t S;
};

struct CoverArgs {
    DevCircuit c;
    const uint32_t *M;            // pruned marks [n_gates][ld]
    uint64_t ld;
    const uint32_t *nzb;          // per column block bitmaps
    const uint32_t *blk_maxlvl;
    uint32_t bm_words;
    uint32_t bw;                  // words per column block
    const uint32_t *first_x, *first_y;
    uint64_t n_pairs;
    uint32_t pair_base;
    uint32_t *active;             // [W] bitmap of first-detecting pairs
    uint32_t *active_list;        // [min(n_pairs, 2 * n_gates)] their indices, in no order
    uint32_t *active_count;       // [1]
    DevAcc *acc;
    uint32_t hash_cap;            // nets one pair may mark (the cover's shared-memory net list)
    // pairs that mark more nets than hash_cap: queued here (count in
    // acc->n_over) and counted by k_cover_spill with per-net values in global
    // memory, slot k ([2][n_gates] u128) for its CTA k; spill_slots = 0: no
    // spill scratch (such a pair reports kErrHashFull)
    uint32_t *over_list;          // [min(n_pairs, 2 * n_gates)]
    unsigned char *spill;
    uint32_t spill_slots;
    // optional: the paths each primary input credits to each pair,
    // [n_pi][n_pairs] u128 as (low, high) u64 pairs, zeroed by the caller
    unsigned long long *pi_counts;
    // segments longer than one net: first_x / first_y are per segment, and
    // the (net, pair) pairs where a pair is first are a hash set built by
    // k_seg_first (keys net << 32 | pair index, ~0 = empty)
    SegArgs seg;
    unsigned long long *seg_first;
    uint64_t seg_first_mask;
};

// Per-segment first-detect merge after the forward kernel (sparse planes).
struct SegMergeArgs {
    SegArgs seg;
    const uint32_t *V, *M;
    uint64_t ld;
    const uint32_t *nzb;          // per column block bitmaps of marked nets (after the prune)
    uint32_t bm_words, bw, W, pair_base;
    uint32_t *first_x, *first_y;  // [S]
};

// Tile widths of the lane forward kernel (k_forward_lanes): a warp per gate
// and LW consecutive words per lane (one 4 LW-byte access per lane and row),
// so a column block is 32 LW words: 32, 64 or 128 words (1,024, 2,048 or
// 4,096 pairs).  A gate's record decode, row addressing, votes and branches
// are paid once per block, so wider lanes spend fewer instructions per pair
// (9.4e9 warp instructions for a pass at 32 words, 4.1e9 at 64).  CTAs of
// 1,024 threads (32 warps) at up to 64 registers for LW = 1, 2; of 512
// threads at up to 128 for LW = 4, whose rows of four words per fan-in
// spill at 64.
constexpr uint32_t kLaneWords = 32;
constexpr uint32_t kLaneWords2 = 64;
constexpr uint32_t kLaneWords4 = 128;
constexpr uint32_t kLaneThreads1 = 1024;
constexpr uint32_t kLaneThreads2 = 1024;
constexpr uint32_t kLaneThreads4 = 512;
constexpr bool lane_tile(uint32_t bw) { return bw == kLaneWords || bw == kLaneWords2 || bw == kLaneWords4; }
constexpr uint32_t lane_threads(uint32_t bw) {
    return bw == kLaneWords4 ? kLaneThreads4 : bw == kLaneWords2 ? kLaneThreads2 : kLaneThreads1;
}
// Words per cover bitmap of a lane circuit (a quarter of a 32-word column
// block, an eighth of a 64-word one, ...).
constexpr uint32_t kLaneCoverWords = 8;
// Forward launches of a batch at most: (tile width, CTAs per SM) classes of
// the thread-per-gate kernel and the two lane tiles.
constexpr uint32_t kMaxBatchClasses = 10;

// Batched grading (k_batch_forward, k_batch_active, k_batch_cover).
struct BatchCtl {
    unsigned int n_items;  // first-detecting (circuit, pair) items of this pass
    unsigned int done;     // cover CTAs finished
    unsigned int err;      // OR of every circuit's device error word after the pass
    unsigned int n_over;   // items queued for the spill cover
    unsigned int done_over;
    unsigned int n_mid;    // items the small-table cover passed to the large-table cover
    unsigned int done_mid;
    unsigned int pad[1];
};
// One forward launch of a batch: jobs of equal tile width and CTAs per SM.
struct BatchClass {
    uint32_t bw, occ, blk0, blocks, threads;
    size_t smem;
};
struct BatchLaunch {
    FwdArgs *fargs;        // [n] per circuit, device
    CoverArgs *cargs;      // [n] per circuit, device
    const uint32_t *bpref; // [n + 1] first forward CTA of each circuit
    const uint32_t *gpref; // [n + 1] first gate of each circuit
    uint2 *items;          // [sum of min(n_pairs, 2 n_gates)]
    uint2 *mid_items;      // [same]: items whose pair marks more nets than the small table
    uint2 *over_items;     // [same]: items whose pair marks more nets than the cover's table
    uint32_t spill_grid;   // CTAs of the batch's spill cover (<= every spilling circuit's slots)
    BatchCtl *ctl;
    uint32_t n, total_blocks, total_gates;
    uint32_t sem, threads, cover_grid, hash_cap, append;  // sem: PDF_MARK_*
    // the small-table cover that runs first: nets per pair, CTAs
    uint32_t small_cap, small_grid;
    size_t fwd_smem;
    uint32_t n_class;      // forward launches: classes of jobs (tile width x CTAs per SM)
    BatchClass cls[kMaxBatchClasses];
    // classes after the first run on side streams, forked from and joined
    // back to the launching stream (parallel branches when captured)
    cudaStream_t side[kMaxBatchClasses - 1];
    cudaEvent_t fork, join[kMaxBatchClasses - 1];
    // profiling (optional): events recorded on the launching stream before
    // the forward launches, after they have all joined, and after the cover;
    // prof_external: recorded as event nodes of a captured graph
    cudaEvent_t prof[3];
    uint32_t prof_external;
};
// Registers per thread of the fused forward kernel for (tile words, mode); <= 0 on error.
int forward_kernel_regs(int bw, int sem);
cudaError_t prepare_batch(const BatchLaunch &b);  // kernel attributes; call before launching or capturing
cudaError_t launch_batch(const BatchLaunch &b, cudaStream_t st);

// Host-side launchers (pdf_kernels.cu).  All return cudaError_t of the launch.
cudaError_t launch_forward(const FwdArgs &a, int mode, int sem, uint32_t bw, uint32_t threads,
                           size_t smem, cudaStream_t st);
// Cover of one batch: k_active then k_cover, whose last CTA closes the batch
// (total += batch, pairs += n_pairs).  The active bitmap [W] and its count
// must be zero (k_forward clears them; zero_active asks for a memset).
cudaError_t launch_cover(const CoverArgs &a, uint32_t grid, uint32_t threads, bool zero_active, cudaStream_t st);
size_t cover_smem_bytes(uint32_t hash_cap);
// The batch's small-table cover: several CTAs per SM, each listing at most
// the returned number of nets per pair in shared memory (0 on error).
uint32_t cover_small_cap(int device, uint32_t *ctas_per_sm);
size_t cover_small_smem_bytes(uint32_t cap);
cudaError_t launch_merge_dense(const DevCircuit &c, const uint32_t *V, const uint32_t *M,
                               uint64_t ld, uint64_t n_pairs, uint32_t pair_base,
                               uint32_t *first_x, uint32_t *first_y, cudaStream_t st);
cudaError_t launch_seg_merge(const SegMergeArgs &a, uint32_t n_blocks, cudaStream_t st);
cudaError_t launch_seg_merge_dense(const SegArgs &seg, const uint32_t *V, const uint32_t *M, uint64_t ld,
                                   uint64_t n_pairs, uint32_t pair_base, uint32_t *first_x, uint32_t *first_y,
                                   cudaStream_t st);
cudaError_t launch_bitmap_from_marks(const DevCircuit &c, const uint32_t *M, uint64_t ld,
                                     uint64_t n_pairs, uint32_t bw, uint32_t *nzb,
                                     uint32_t *blk_maxlvl, uint32_t bm_words, cudaStream_t st);
// Fixed scratch of pdf_cover_noalloc (a file-scope __device__ array).
constexpr size_t kNoAllocScratchBytes = (size_t)8 << 20;
cudaError_t noalloc_scratch(int device, unsigned char **out);

cudaError_t launch_batch_begin(DevAcc *acc, cudaStream_t st);
// Copies n16 16-byte words from mapped pinned host memory to device memory
// with SM loads, so the copy does not queue behind other host threads'
// transfers on the copy engines.  src and dst 16-byte aligned.
cudaError_t launch_copy_from_host(void *dst, const void *src_mapped, size_t n16, cudaStream_t st);

#endif
