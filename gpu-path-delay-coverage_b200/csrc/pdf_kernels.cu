// pdf_kernels.cu -- sm_100a kernels of the grading path.
//
// Layout: every per-(net, pair) quantity is a bit-plane, gate-major, ld words
// per gate row, 32 pairs per word.  A CTA owns one column block of BW words
// (32 * BW pairs) and walks every gate of the circuit in level order for it:
// the only dependency between pairs is the first-detect minimum, so column
// blocks never wait on one another and no grid-wide barrier is needed.
//
//   k_forward   sim + forward robust mark (levels ascending, warps as
//               dataflow: each gate waits only for its own fan-ins), then,
//               in the same CTA, the prune (levels descending) and the
//               first-detect merge over the gates whose marks are nonzero.
//   k_active / k_cover
//               path counting, only for pairs that first-detect some net
//               (every other pair credits nothing), over only the nets those
//               pairs mark, in exact 128-bit integers.
#include "pdf_kernels.cuh"

#include <algorithm>
#include <map>
#include <mutex>

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ GateRec load_rec(const GateRec *p) {
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    const uint4 a = __ldg(q), b = __ldg(q + 1);
    GateRec r;
    r.w[0] = a.x;
    r.w[1] = a.y;
    r.w[2] = a.z;
    r.w[3] = a.w;
    r.w[4] = b.x;
    r.w[5] = b.y;
    r.w[6] = b.z;
    r.w[7] = b.w;
    return r;
}

// Set bit g of a bitmap with one atomic per distinct word among the calling
// lanes.
__device__ __forceinline__ void bitmap_set_aggregated(uint32_t *bm, uint32_t g) {
    const unsigned active = __activemask();
    const uint32_t word = g >> 5;
    const unsigned grp = __match_any_sync(active, word);
    const uint32_t bits = __reduce_or_sync(grp, 1u << (g & 31));
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(grp) - 1)) atomicOr(bm + word, bits);
}

__device__ __forceinline__ bool bit_test(const uint32_t *bm, uint32_t g) { return (bm[g >> 5] >> (g & 31)) & 1u; }

// ---- TMA bulk copies and mbarriers (inline PTX, sm_90+ / sm_100a) ----

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes)
                 : "memory");
}
// One untiled bulk copy global -> shared; both addresses 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *m) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(m))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(phase)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t *m, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Every wait is bounded: on expiry the caller reports PDF_ETIMEOUT.  polls =
// 0: up to kSpinLimit blocking polls (try_wait may suspend the thread until
// the phase completes); polls > 0: that many non-blocking polls, a bound
// small enough to run out (tests of the timeout path).
constexpr uint32_t kSpinLimit = 1u << 24;
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t phase, uint32_t polls = 0) {
    if (polls) {
        for (uint32_t i = 0; i < polls; i++)
            if (mbar_test_wait(m, phase)) return true;
        return false;
    }
    for (uint32_t i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(m, phase)) return true;
    return false;
}

// Asynchronous global -> shared copy of BW words (cp.async, completed by
// cp.async.wait_all in the issuing thread).
template <int BW>
__device__ __forceinline__ void cp_async_vec(uint32_t *dst, const uint32_t *src) {
    if constexpr (BW == 1) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
    } else if constexpr (BW == 2) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
    } else {
#pragma unroll
        for (int i = 0; i < BW; i += 4)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + i)), "l"(src + i)
                         : "memory");
    }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared-memory layout of k_forward (byte offsets from the host plan).
struct FwdSmem {
    uint32_t *ring;   // forward: [3][R][BW] V, T, M; reverse: [R2][BW] pruned marks
    GateRec *rec;     // [2][cap] staged gate records of a piece
    uint32_t *edge;   // reverse: [2][ecap] staged edge slices
    uint32_t *far;    // forward: [2][3][farcap][BW] far fan-in V, T, M (same memory as edge)
    uint32_t *fid;    // forward: [2][farcap] far-id lists staged with the records
    uint32_t *bm;     // nonzero-mark bitmap (shared or global)
    uint32_t *pbits;  // pieces that hold a forward mark
    uint64_t *mbar;   // [2]
};

// Stage piece `p` into buffer `buf`: its gate records and, for the reverse
// pass, its edge slice; for the forward pass, the far-id list of the piece
// after it (lists are stored in piece order, each padded to 4 entries, so it
// starts at p.far_off + 4 * ceil(p.far_n / 4)).  Called by one thread.
__device__ __forceinline__ void stage_piece(const FwdArgs &a, const FwdSmem &S, const Piece &p, int buf,
                                            bool edges) {
    const uint32_t rb = (p.b - p.a) * (uint32_t)sizeof(GateRec);
    const bool e = edges && p.ea != 0xFFFFFFFFu;
    const uint32_t eb = e ? (p.eb - p.ea) * 4u : 0u;
    const uint32_t fb = edges ? 0u : ((p.nfar_n + 3u) & ~3u) * 4u;
    fence_proxy_async();
    mbar_expect_tx(S.mbar + buf, rb + eb + fb);
    bulk_g2s(S.rec + (size_t)buf * a.cap, a.c.rec + p.a, rb, S.mbar + buf);
    if (e) bulk_g2s(S.edge + (size_t)buf * a.ecap, a.c.edges + p.ea, eb, S.mbar + buf);
    if (fb)
        bulk_g2s(S.fid + (size_t)buf * a.farcap, a.far_ids + p.far_off + ((p.far_n + 3u) & ~3u), fb, S.mbar + buf);
}

// BW consecutive words of one plane row, moved with 16-byte (or 8-byte)
// vector accesses.  Every address passed here is a multiple of BW words.
template <int BW>
struct Vec {
    uint32_t x[BW];
};
template <int BW>
__device__ __forceinline__ Vec<BW> vld(const uint32_t *p) {
    Vec<BW> v;
    if constexpr (BW == 1) {
        v.x[0] = *p;
    } else if constexpr (BW == 2) {
        const uint2 q = *reinterpret_cast<const uint2 *>(p);
        v.x[0] = q.x;
        v.x[1] = q.y;
    } else {
#pragma unroll
        for (int i = 0; i < BW; i += 4) {
            const uint4 q = *reinterpret_cast<const uint4 *>(p + i);
            v.x[i] = q.x;
            v.x[i + 1] = q.y;
            v.x[i + 2] = q.z;
            v.x[i + 3] = q.w;
        }
    }
    return v;
}
template <int BW>
__device__ __forceinline__ Vec<BW> vldg(const uint32_t *p) {  // read-only data (pairs)
    Vec<BW> v;
    if constexpr (BW == 1) {
        v.x[0] = __ldg(p);
    } else if constexpr (BW == 2) {
        const uint2 q = __ldg(reinterpret_cast<const uint2 *>(p));
        v.x[0] = q.x;
        v.x[1] = q.y;
    } else {
#pragma unroll
        for (int i = 0; i < BW; i += 4) {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p + i));
            v.x[i] = q.x;
            v.x[i + 1] = q.y;
            v.x[i + 2] = q.z;
            v.x[i + 3] = q.w;
        }
    }
    return v;
}
// BW words from shared memory at byte address sa (ld.shared, 16-byte
// vectors; sa a multiple of 4 * BW).
template <int BW>
__device__ __forceinline__ Vec<BW> vlds(uint32_t sa) {
    Vec<BW> v;
    if constexpr (BW == 1) {
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v.x[0]) : "r"(sa));
    } else if constexpr (BW == 2) {
        asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x[0]), "=r"(v.x[1]) : "r"(sa));
    } else {
#pragma unroll
        for (int i = 0; i < BW; i += 4)
            asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                         : "=r"(v.x[i]), "=r"(v.x[i + 1]), "=r"(v.x[i + 2]), "=r"(v.x[i + 3])
                         : "r"(sa + 4u * i));
    }
    return v;
}
template <int BW>
__device__ __forceinline__ void vst(uint32_t *p, const Vec<BW> &v) {
    if constexpr (BW == 1) {
        *p = v.x[0];
    } else if constexpr (BW == 2) {
        *reinterpret_cast<uint2 *>(p) = make_uint2(v.x[0], v.x[1]);
    } else {
#pragma unroll
        for (int i = 0; i < BW; i += 4)
            *reinterpret_cast<uint4 *>(p + i) = make_uint4(v.x[i], v.x[i + 1], v.x[i + 2], v.x[i + 3]);
    }
}
template <int BW>
__device__ __forceinline__ bool vany(const Vec<BW> &v) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < BW; i++) o |= v.x[i];
    return o != 0;
}

// The side-input test of a marked multi-input gate (markkernel.cuh:253-261
// with robust()/nonrobust(), :43-72) in one pass over its nfi fan-ins
// (sens_step, pdf_device.cuh).  fetch(q, V, T) reads fan-in q; fan-ins 0..3
// are unrolled.
// The two-term table (LUT_NR) keeps 8 accumulator words per pair word, so
// wide tiles take the fan-ins in passes of two words (fan-ins re-read from
// shared memory) to stay within the launch bound's registers.
template <int BW, int ROBUST, class Fetch>
__device__ __forceinline__ Vec<BW> sens_any(const GateRec &r, uint32_t nfi, Fetch fetch) {
    const bool or_like = (r.w[0] & RF_IM) != 0;
    constexpr int SUB = (ROBUST || BW <= 2) ? BW : 2;
    Vec<BW> out;
#pragma unroll
    for (int j0 = 0; j0 < BW; j0 += SUB) {
        SensAcc acc[SUB];
#pragma unroll
        for (int j = 0; j < SUB; j++) sens_init(acc[j]);
        auto step = [&](uint32_t q) {
            Vec<BW> v, t;
            fetch(q, v, t);
#pragma unroll
            for (int j = 0; j < SUB; j++) sens_step<ROBUST>(acc[j], or_like, v.x[j0 + j], t.x[j0 + j]);
        };
#pragma unroll
        for (int q = 0; q < kInlineFanins; q++)
            if ((uint32_t)q < nfi) step(q);
        for (uint32_t q = kInlineFanins; q < nfi; q++) step(q);
#pragma unroll
        for (int j = 0; j < SUB; j++) out.x[j0 + j] = sens_result<ROBUST>(acc[j]);
    }
    return out;
}

// The FIXED modes' test (sens_step_fixed): OR over fan-ins i carrying a mark
// of AND over the other fan-ins of the side table; fetch also gives marks.
template <int BW, int NONROBUST, class Fetch3>
__device__ __forceinline__ Vec<BW> sens_any_fixed(const GateRec &r, uint32_t nfi, Fetch3 fetch) {
    const uint32_t mor = flagmask(r.w[0], RF_IM), mxor = flagmask(r.w[0], RF_XOR), mand = ~(mor | mxor);
    constexpr int SUB = (NONROBUST || BW <= 2) ? BW : 2;  // passes of two words, as sens_any
    Vec<BW> out;
#pragma unroll
    for (int j0 = 0; j0 < BW; j0 += SUB) {
        SensAcc acc[SUB];
#pragma unroll
        for (int j = 0; j < SUB; j++) sens_init(acc[j]);
        auto step = [&](uint32_t q) {
            Vec<BW> v, t, m;
            fetch(q, v, t, m);
#pragma unroll
            for (int j = 0; j < SUB; j++)
                sens_step_fixed<NONROBUST>(acc[j], mand, mor, mxor, v.x[j0 + j], t.x[j0 + j], m.x[j0 + j]);
        };
#pragma unroll
        for (int q = 0; q < kInlineFanins; q++)
            if ((uint32_t)q < nfi) step(q);
        for (uint32_t q = kInlineFanins; q < nfi; q++) step(q);
#pragma unroll
        for (int j = 0; j < SUB; j++) out.x[j0 + j] = sens_result<NONROBUST>(acc[j]);
    }
    return out;
}

// A CTA that gave up on an expired wait publishes an empty column block (no
// marked net, no marked level), so the kernels that run after it (cover,
// segment merge) read nothing the CTA did not finish.
__device__ __forceinline__ void empty_block(const FwdArgs &a, uint32_t blk, uint32_t *gbm) {
    if (gbm)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) gbm[q] = 0;
    if (a.blk_maxlvl && threadIdx.x == 0) a.blk_maxlvl[blk] = 0;
}

// Reverse pass (prune, markkernel.cuh:271-293) and first-detect merge
// (mergekernel.cuh:116-198) of k_forward, after its forward pass: only
// pieces that hold a forward mark, descending, only gates whose bitmap bit is
// set.  While piece i runs, the mark (and value) rows of the next marked
// piece's marked gates are copied into a staging buffer with cp.async.  A
// gate's pruned mark is final once its fan-outs are, so it is folded into
// first_x / first_y right away.  `phase` carries the parity bits of the two
// record mbarriers.
template <int BW, int MODE>
__device__ __forceinline__ void prune_and_merge(const FwdArgs &a, const FwdSmem &S, uint32_t blk, uint32_t *gbm,
                                                uint32_t phase) {
    const uint32_t w0 = blk * BW;
    const uint32_t *edges = a.c.edges;
    const uint32_t R2 = a.ring2_gates, R2m = R2 - 1;
    uint32_t *ring2 = S.ring;
    uint32_t *mst = S.ring + (size_t)R2 * BW;  // [2][cap][2][BW]: M and V rows
    auto prev_marked = [&](int from) -> int {  // highest marked piece index < from
        for (int q = (from - 1) >> 5; q >= 0 && from > 0; q--) {
            uint32_t bits = S.pbits[q];
            if (q == (from - 1) >> 5) bits &= (from & 31) ? ((1u << (from & 31)) - 1u) : 0xFFFFFFFFu;
            if (bits) return q * 32 + 31 - __clz(bits);
        }
        return -1;
    };
    auto stage_rows = [&](const Piece &Q, int b) {
        for (uint32_t gi = threadIdx.x; gi < Q.b - Q.a; gi += blockDim.x) {
            const uint32_t g = Q.a + gi;
            if (!bit_test(S.bm, g)) continue;
            uint32_t *d = mst + ((size_t)b * a.cap + gi) * 2 * BW;
            const size_t o = (size_t)g * a.ld + w0;
            cp_async_vec<BW>(d, a.M + o);
            if (MODE == FWD_FUSED) cp_async_vec<BW>(d + BW, a.V + o);
        }
    };
    bool failed = false;
    int cur = prev_marked((int)a.n_pieces);
    uint32_t maxlvl = 0;
    int sbuf = 0;
    // descriptors of the current and the next marked piece; the one after
    // is loaded a piece ahead, so its latency hides behind a piece's work
    Piece Pc{}, Pn{};
    if (cur >= 0) {
        Pc = a.pieces[cur];
        if (threadIdx.x == 0) stage_piece(a, S, Pc, 0, true);
        stage_rows(Pc, 0);
        cp_async_wait_all();
    }
    int nxt = cur >= 0 ? prev_marked(cur) : -1;
    if (nxt >= 0) Pn = a.pieces[nxt];
    while (cur >= 0) {
        const Piece P = Pc;
        if (nxt >= 0) {
            if (threadIdx.x == 0) stage_piece(a, S, Pn, sbuf ^ 1, true);
            stage_rows(Pn, sbuf ^ 1);
        }
        const int nxt2 = nxt >= 0 ? prev_marked(nxt) : -1;
        Piece Pn2{};
        if (nxt2 >= 0) Pn2 = a.pieces[nxt2];
        const bool ok = mbar_wait(S.mbar + sbuf, (phase >> sbuf) & 1u, a.wait_polls);
        phase ^= 1u << sbuf;
        if (__syncthreads_or(!ok)) {
            // no CTA leaves with a copy in flight: wait (at the full bound)
            // for this piece's copy and the next one's, then report
            failed = true;
            (void)mbar_wait(S.mbar + sbuf, ((phase >> sbuf) & 1u) ^ 1u);
            if (nxt >= 0) (void)mbar_wait(S.mbar + (sbuf ^ 1), (phase >> (sbuf ^ 1)) & 1u);
            cp_async_wait_all();
            break;
        }
        const GateRec *recs = S.rec + (size_t)sbuf * a.cap;
        const uint32_t *es = S.edge + (size_t)sbuf * a.ecap;
        const uint32_t *rows = mst + (size_t)sbuf * a.cap * 2 * BW;
        const bool staged = P.ea != 0xFFFFFFFFu;
        const uint32_t win = P.a + R2;  // fan-outs below this are in ring2
        bool any = false;
        for (uint32_t gi = threadIdx.x; gi < P.b - P.a; gi += blockDim.x) {
            const uint32_t g = P.a + gi;
            if (!bit_test(S.bm, g)) continue;
            const GateRec &r = recs[gi];
            const Vec<BW> mk = vld<BW>(rows + (size_t)gi * 2 * BW);
            Vec<BW> keep;
#pragma unroll
            for (int j = 0; j < BW; j++) keep.x[j] = rec_po(r) ? 0xFFFFFFFFu : 0u;
            if (!rec_po(r)) {
                const uint32_t nfo = r.w[1], base = r.w[2] + rec_nfi(r);
                for (uint32_t k = 0; k < nfo; k++) {
                    const uint32_t fo = staged ? es[base + k - P.ea] : __ldg(edges + base + k);
                    if (!bit_test(S.bm, fo)) continue;
                    const Vec<BW> fm =
                        fo < win ? vld<BW>(ring2 + (fo & R2m) * BW) : vld<BW>(a.M + (size_t)fo * a.ld + w0);
#pragma unroll
                    for (int j = 0; j < BW; j++) keep.x[j] |= fm.x[j];
                }
            }
            Vec<BW> nm;
            bool changed = false;
#pragma unroll
            for (int j = 0; j < BW; j++) {
                nm.x[j] = mk.x[j] & keep.x[j];
                changed |= nm.x[j] != mk.x[j];
            }
            if (changed) vst<BW>(a.M + (size_t)g * a.ld + w0, nm);
            if (g < win) vst<BW>(ring2 + (g & R2m) * BW, nm);
            const bool nz = vany(nm);
            if (!nz) {
                atomicAnd(S.bm + (g >> 5), ~(1u << (g & 31)));
            } else if (MODE == FWD_FUSED && a.first_x) {  // merge: first falling / rising pair
                const Vec<BW> v = vld<BW>(rows + (size_t)gi * 2 * BW + BW);
                uint32_t cx = kEmpty, cy = kEmpty;
#pragma unroll
                for (int j = BW - 1; j >= 0; j--) {  // lowest word wins
                    const uint32_t x = nm.x[j] & ~v.x[j], y = nm.x[j] & v.x[j];
                    if (x) cx = (w0 + j) * 32 + (__ffs(x) - 1);
                    if (y) cy = (w0 + j) * 32 + (__ffs(y) - 1);
                }
                if (cx != kEmpty) atomicMin(a.first_x + g, a.pair_base + cx);
                if (cy != kEmpty) atomicMin(a.first_y + g, a.pair_base + cy);
            }
            any |= nz;
        }
        cp_async_wait_all();  // this thread's rows for the next piece
        if (__syncthreads_or(any) && P.level + 1 > maxlvl) maxlvl = P.level + 1;
        cur = nxt;
        nxt = nxt2;
        Pc = Pn;
        Pn = Pn2;
        sbuf ^= 1;
    }
    if (failed) {
        empty_block(a, blk, gbm);
        if (threadIdx.x == 0) atomicOr(a.err, kErrTimeout);
        return;
    }
    // publish the bitmap of surviving marks for the cover kernels
    if (a.bm_shared && gbm)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) gbm[q] = S.bm[q];
    if (threadIdx.x == 0) a.blk_maxlvl[blk] = maxlvl;
}

// ---------------------------------------------------------------------------
// Forward kernel: one CTA per column block of BW words (32 * BW pairs); one
// thread per gate, carrying all BW words of the block.
//
// Gates are walked in pieces (runs of one level, <= cap gates), one
// __syncthreads per piece; each piece's records are staged into shared
// memory by a TMA bulk copy issued one piece ahead.
//
// Forward (sim + forward mark, simkernel.cuh:96-156, markkernel.cuh:215-270):
// a ring of the last R gates' V, T, M words sits in shared memory
// (slot = gate & (R - 1)); every gate writes its slot.  During piece [a, b)
// a fan-in f >= b - R is read from the ring: no gate of [f + 1, b) shares its
// slot.  Older fan-ins are the piece's far fan-ins, listed at circuit upload
// (deduplicated, per piece) together with one source byte per fan-in in the
// gate record.  While piece i runs, threads without a gate of piece i copy
// the rows of piece i + 1's far fan-ins (gates below piece i, so complete)
// into a far buffer with cp.async; piece i + 1 reads them from there.  A
// far fan-in the list could not hold is read from its plane row.
//
// Reverse (prune, markkernel.cuh:271-293) and merge (mergekernel.cuh:116-198):
// see prune_and_merge.  Pruned marks of recent gates sit in a second ring
// (the same memory, R2 slots of BW words): during piece [a, b) a fan-out fo
// is read from it iff fo < a + R2 and only gates g < a + R2 write it.
//
// Plane rows are read and written BW words at a time: ld and pi_ld are
// multiples of BW and every row holds all n_blocks * BW words; words at or
// past ceil(n_pairs / 32) are masked to zero.
// ---------------------------------------------------------------------------
// One CTA's work: column block `blk` of the circuit in `a`.
// SEM: the circuit's PDF_MARK_* mode (0, 1: the reference's tables; 2, 3:
// true n-input gates with the FIXED tables).
template <int BW, int SEM, int MODE>
__device__ __forceinline__ void forward_cta(const FwdArgs &a, const uint32_t blk) {
    constexpr bool FIX = SEM >= 2;
    extern __shared__ __align__(128) unsigned char smraw[];
    FwdSmem S;
    S.ring = reinterpret_cast<uint32_t *>(smraw + a.off_ring);
    S.rec = reinterpret_cast<GateRec *>(smraw + a.off_rec);
    S.edge = reinterpret_cast<uint32_t *>(smraw + a.off_edge);
    S.far = reinterpret_cast<uint32_t *>(smraw + a.off_edge);
    S.fid = reinterpret_cast<uint32_t *>(smraw + a.off_fid);
    S.pbits = reinterpret_cast<uint32_t *>(smraw + a.off_pbits);
    S.mbar = reinterpret_cast<uint64_t *>(smraw + a.off_mbar);
    const uint32_t w0 = blk * BW;
    S.bm = a.bm_shared ? reinterpret_cast<uint32_t *>(smraw + a.off_bm) : a.nzb + (size_t)blk * a.bm_words;
    uint32_t *gbm = a.nzb ? a.nzb + (size_t)blk * a.bm_words : nullptr;
    const uint32_t *edges = a.c.edges;
    const uint32_t R = a.ring_gates, Rm = R - 1;
    uint32_t *rV = S.ring, *rT = S.ring + (size_t)R * BW, *rM = S.ring + 2 * (size_t)R * BW;
    const size_t fplane = (size_t)a.farcap * BW;  // words per far-buffer plane
    const uint32_t fplane_b = (uint32_t)fplane * 4u, ring_b = R * BW * 4u;
    const uint32_t ring_sa = smem_u32(S.ring);
    const bool tail = w0 + BW >= a.W;             // the block holds padding words
    Vec<BW> wm;                                   // valid bits of each word of this block
#pragma unroll
    for (int j = 0; j < BW; j++) {
        const uint32_t w = w0 + j;
        wm.x[j] = w + 1 < a.W ? 0xFFFFFFFFu
                              : (w + 1 == a.W ? ((a.n_pairs & 31) ? (1u << (a.n_pairs & 31)) - 1u : 0xFFFFFFFFu) : 0u);
    }

    if (MODE != FWD_SIM)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) S.bm[q] = 0;
    for (uint32_t q = threadIdx.x; q < (a.n_pieces + 31) / 32; q += blockDim.x) S.pbits[q] = 0;
    if (MODE == FWD_FUSED) {  // the batch's cover state (the cover kernels run after this one)
        // active words w0 .. w0 + BW - 1 of this block; word W (the count) by the last block
        if (a.active && threadIdx.x < BW && w0 + threadIdx.x <= a.W) a.active[w0 + threadIdx.x] = 0;
        if (a.active && blk == 0 && threadIdx.x == 0) a.active[a.W] = 0;
        if (a.acc && blk == 0 && threadIdx.x == 0) {
            a.acc->batch_lo = 0;
            a.acc->batch_hi = 0;
            a.acc->batch_flags = 0;
            a.acc->done = 0;
            a.acc->n_over = 0;
            a.acc->done_over = 0;
        }
    }
    __shared__ uint32_t s_fail;
    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(S.mbar, 1);
        mbar_init(S.mbar + 1, 1);
        fence_mbar_init();
    }
    __syncthreads();

    // Copy the n far fan-ins listed at ids (shared memory) into far buffer
    // fb; entry e goes to thread blockDim - 1 - e, a thread without a gate
    // when the piece running now is smaller than the CTA.
    auto prefetch = [&](uint32_t n, uint32_t fb, const uint32_t *ids) {
        for (uint32_t e = blockDim.x - 1 - threadIdx.x; e < n; e += blockDim.x) {
            const uint32_t f = ids[e];
            const size_t o = (size_t)f * a.ld + w0;
            uint32_t *d = S.far + (size_t)fb * 3 * fplane + (size_t)e * BW;
            cp_async_vec<BW>(d, a.V + o);
            cp_async_vec<BW>(d + fplane, a.T + o);
            // the reference modes read a fan-in's mark only when its bitmap
            // bit is set, and unmarked rows are not written (below)
            if (MODE != FWD_SIM && (FIX || a.store_all || bit_test(S.bm, f))) cp_async_vec<BW>(d + 2 * fplane, a.M + o);
        }
    };

    uint32_t phase = 0;  // bit b: parity of the next wait on mbar[b]
    // ------------------------------------------------------------- forward
    // Piece i's copy (buffer i & 1) brings its records and piece i + 1's
    // far-id list, so no global load stands between a piece's start and the
    // far-row copies of the next piece.  The last thread issues it: it holds
    // a gate only when the piece fills the CTA.
    const uint32_t stager = blockDim.x - 1;
    if (threadIdx.x == stager) stage_piece(a, S, a.pieces[0], 0, false);
    Piece P1 = a.n_pieces > 1 ? a.pieces[1] : a.pieces[0];
    for (uint32_t i = 0; i < a.n_pieces; i++) {
        const Piece P = i == 0 ? a.pieces[0] : P1;
        const int buf = i & 1;
        const bool has_next = i + 1 < a.n_pieces;
        if (has_next) P1 = a.pieces[i + 1];
        if (threadIdx.x == stager && has_next) stage_piece(a, S, P1, buf ^ 1, false);
        // every thread waits for the records itself; the piece's only
        // barrier is at its end
        const bool ok = mbar_wait(S.mbar + buf, (phase >> buf) & 1u, a.wait_polls);
        phase ^= 1u << buf;
        if (!ok) s_fail = 1;
        if (has_next && ok) prefetch(P.nfar_n, buf ^ 1, S.fid + (size_t)buf * a.farcap);
        const GateRec *recs = S.rec + (size_t)buf * a.cap;
        const uint32_t far_sa = smem_u32(S.far) + (uint32_t)buf * 3u * fplane_b;
        const uint32_t ring_lo = P.b - R;  // (wraps below 0: every fan-in is in the ring then)
        bool any = false;
        for (uint32_t gi = threadIdx.x; ok && gi < P.b - P.a; gi += blockDim.x) {
            const uint32_t g = P.a + gi;
            const GateRec r = recs[gi];
            const uint32_t h = r.w[0];
            // source word of fan-in q (pdf_device.cuh); q is a constant for
            // the inline fan-ins 0..3
            auto srcw = [&](uint32_t q) -> uint32_t {
                if (q < (uint32_t)kInlineFanins) return r.w[3 + q];
                const uint32_t f = __ldg(edges + r.w[2] + q);
                return (P.b <= R || f >= ring_lo) ? (f & Rm) : (SRC_PLANE | f);
            };
            // plane k (0 V, 1 T, 2 M) of the gate behind source word sw
            auto load = [&](uint32_t sw, uint32_t k) -> Vec<BW> {
                if (sw & SRC_PLANE) {
                    const uint32_t *pl = k == 0 ? a.V : (k == 1 ? a.T : a.M);
                    return vld<BW>(pl + (size_t)(sw & ~SRC_PLANE) * a.ld + w0);
                }
                const uint32_t sa = (sw & SRC_FAR) ? far_sa + k * fplane_b + (sw & SRC_IDX) * (4u * BW)
                                                   : ring_sa + k * ring_b + sw * (4u * BW);
                return vlds<BW>(sa);
            };
            Vec<BW> V, T, M;
            if (MODE == FWD_MARK) {
                V = vld<BW>(a.V + (size_t)g * a.ld + w0);
                T = vld<BW>(a.T + (size_t)g * a.ld + w0);
            } else if (h & RF_INPT) {  // simkernel.cuh:112-125, pairs already formed
                V = vldg<BW>(a.pi_v + (size_t)g * a.pi_ld + w0);
                T = vldg<BW>(a.pi_t + (size_t)g * a.pi_ld + w0);
            }
            if (tail && (MODE == FWD_MARK || (h & RF_INPT))) {
#pragma unroll
                for (int j = 0; j < BW; j++) {
                    V.x[j] &= wm.x[j];
                    T.x[j] &= wm.x[j];
                }
            }
            if (MODE != FWD_MARK && !(h & RF_INPT)) {
                Vec<BW> v1;
                {
                    const uint32_t s0 = r.w[3];
                    const Vec<BW> fv = load(s0, 0), ft = load(s0, 1);
#pragma unroll
                    for (int j = 0; j < BW; j++) eval_first(h, fv.x[j], ft.x[j], V.x[j], v1.x[j]);
                }
                const uint32_t nfold = hdr_nfold(h);
                auto fold = [&](uint32_t q) {
                    const uint32_t sq = srcw(q);
                    const Vec<BW> fv = load(sq, 0), ft = load(sq, 1);
#pragma unroll
                    for (int j = 0; j < BW; j++) eval_fold<FIX>(h, V.x[j], v1.x[j], fv.x[j], ft.x[j]);
                };
#pragma unroll
                for (int q = 1; q < kInlineFanins; q++)
                    if ((uint32_t)q <= nfold) fold(q);
                for (uint32_t q = kInlineFanins; q <= nfold; q++) fold(q);
#pragma unroll
                for (int j = 0; j < BW; j++) eval_finish<FIX>(h, V.x[j], v1.x[j], T.x[j]);
                if (tail) {
#pragma unroll
                    for (int j = 0; j < BW; j++) {
                        V.x[j] &= wm.x[j];
                        T.x[j] &= wm.x[j];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < BW; j++) M.x[j] = 0;
            if (MODE != FWD_SIM) {  // markkernel.cuh:226-267
                if (h & RF_INPT) {
                    M = T;
                } else if ((h & RF_MARKF0) && vany(T) && bit_test(S.bm, r.w[7])) {
                    // fan-in 0 (gate w[7]) holds a mark: its bitmap bit is set
                    const Vec<BW> m0 = load(r.w[3], 2);
#pragma unroll
                    for (int j = 0; j < BW; j++) M.x[j] = T.x[j] & m0.x[j];
                    if ((h & RF_SENS) && vany(M)) {
                        auto fetch = [&](uint32_t q, Vec<BW> &fv, Vec<BW> &ft) {
                            const uint32_t sq = srcw(q);
                            fv = load(sq, 0);
                            ft = load(sq, 1);
                        };
                        const Vec<BW> sv = sens_any<BW, SEM & 1>(r, rec_nfi(r), fetch);
#pragma unroll
                        for (int j = 0; j < BW; j++) M.x[j] &= sv.x[j];
                    }
                } else if (FIX && (h & RF_MANY) && vany(T)) {
                    // any fan-in may carry the path: its own mark enters the side test
                    auto fetch3 = [&](uint32_t q, Vec<BW> &fv, Vec<BW> &ft, Vec<BW> &fm) {
                        const uint32_t sq = srcw(q);
                        fv = load(sq, 0);
                        ft = load(sq, 1);
                        fm = load(sq, 2);
                    };
                    const Vec<BW> sv = sens_any_fixed<BW, SEM == PDF_MARK_FIXED_NONROBUST>(r, rec_nfi(r), fetch3);
#pragma unroll
                    for (int j = 0; j < BW; j++) M.x[j] = T.x[j] & sv.x[j];
                }
            }
            const bool marked = MODE != FWD_SIM && vany(M);
            // plane rows: every row when asked for; else the rows that are
            // read back (far fan-ins, and the marked gates the prune, merge
            // and cover visit)
            if (a.store_all || (h & RF_SPILL) || marked) {
                const size_t o = (size_t)g * a.ld + w0;
                if (MODE != FWD_MARK) {
                    vst<BW>(a.V + o, V);
                    vst<BW>(a.T + o, T);
                }
                // an unmarked row stays unwritten: its readers (fan-outs in the
                // reference modes, prune, merge, cover) test the bitmap first
                if (MODE != FWD_SIM && (FIX || a.store_all || marked)) vst<BW>(a.M + o, M);
            }
            const uint32_t slot = (g & Rm) * BW;
            vst<BW>(rV + slot, V);
            vst<BW>(rT + slot, T);
            if (MODE != FWD_SIM) vst<BW>(rM + slot, M);
            if (marked) {
                bitmap_set_aggregated(S.bm, g);
                any = true;
            }
        }
        cp_async_wait_all();  // this thread's copies for piece i + 1
        if (__syncthreads_or(any) && threadIdx.x == 0) S.pbits[i >> 5] |= 1u << (i & 31);
        if (s_fail) {
            // no CTA leaves with a copy in flight: wait (at the full bound)
            // for this piece's record copy and the next one's, then report
            (void)mbar_wait(S.mbar + buf, ((phase >> buf) & 1u) ^ 1u);
            if (has_next) (void)mbar_wait(S.mbar + (buf ^ 1), (phase >> (buf ^ 1)) & 1u);
            if (MODE != FWD_SIM) empty_block(a, blk, gbm);
            if (threadIdx.x == 0) atomicOr(a.err, kErrTimeout);
            return;
        }
    }
    if constexpr (MODE != FWD_SIM) {
        if (MODE == FWD_MARK && a.no_prune) return;
        __syncthreads();
        prune_and_merge<BW, MODE>(a, S, blk, gbm, phase);
    }
}

template <int BW, int SEM, int MODE>
__global__ void __launch_bounds__(BW >= 8 ? 512 : 1024) k_forward(const FwdArgs a) {
    forward_cta<BW, SEM, MODE>(a, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Lane forward kernel (tiles of 32 x LW words, LW = 1 or 2): the same stages
// as forward_cta (sim, forward mark, prune, merge) with the roles of threads
// turned around.  Lane j of every warp carries words w0 + LW j .. + LW - 1 of
// the column block, and a warp evaluates one gate at a time for the whole
// block, so every instruction of a gate is uniform across the warp (no
// divergence on gate type or fan-in count), a gate's record is decoded once
// per 1,024 LW pairs, and every plane-row access is one coalesced line of
// 128 LW bytes.  Warps take the gates of a level in turn; the gates of a
// level depend only on lower levels, so a CTA needs one barrier per level
// (not per piece of a level), and every fan-in is read from its plane row
// (L1/L2), which is what wide levels need: nothing of the circuit is kept on
// chip except the block's mark bitmap and the staged records.  Several gates
// per warp are in flight at a time (their fan-in rows are loaded before any
// is evaluated).
//
// Every gate with fan-outs writes its V and T rows (its readers load them);
// a gate writes its M row only when it holds a mark (every reader of a mark
// row tests the gate's bitmap bit first), or when the caller asked for the
// planes (store_all).  Words past the last pair of a row are read (rows are
// padded to whole blocks) but masked, and never written.
// ---------------------------------------------------------------------------

// A lane's view of the planes: its first word in row 0 of each plane, and
// the row pitch in bytes (below 2^32: planes_fit), so that a row address is
// one wide multiply-add.
struct LanePlanes {
    char *V, *T, *M;
    uint32_t ld4;
};
template <typename P>
__device__ __forceinline__ uint32_t *lrow(P *base, uint32_t f, uint32_t ld4) {
    return reinterpret_cast<uint32_t *>(const_cast<char *>(base) + (size_t)f * ld4);
}
template <int LW>
__device__ __forceinline__ void lload(const uint32_t *p, uint32_t (&d)[LW]) {
    if constexpr (LW == 4) {
        const uint4 v = *reinterpret_cast<const uint4 *>(p);
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
    } else if constexpr (LW == 2) {
        const uint2 v = *reinterpret_cast<const uint2 *>(p);
        d[0] = v.x;
        d[1] = v.y;
    } else {
        d[0] = *p;
    }
}
template <int LW>
__device__ __forceinline__ void lload_nc(const uint32_t *p, uint32_t (&d)[LW]) {
    if constexpr (LW == 4) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(p));
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
    } else if constexpr (LW == 2) {
        const uint2 v = __ldg(reinterpret_cast<const uint2 *>(p));
        d[0] = v.x;
        d[1] = v.y;
    } else {
        d[0] = __ldg(p);
    }
}
// nw: the lane's words that hold pairs (1..LW); the others are not written
template <int LW>
__device__ __forceinline__ void lstore(uint32_t *p, const uint32_t (&s)[LW], uint32_t nw) {
    if constexpr (LW == 4) {
        if (nw == 4) {
            *reinterpret_cast<uint4 *>(p) = make_uint4(s[0], s[1], s[2], s[3]);
        } else {
#pragma unroll
            for (int j = 0; j < 3; j++)
                if ((uint32_t)j < nw) p[j] = s[j];
        }
    } else if constexpr (LW == 2) {
        if (nw == 2) *reinterpret_cast<uint2 *>(p) = make_uint2(s[0], s[1]);
        else p[0] = s[0];
    } else {
        p[0] = s[0];
    }
}
template <int LW>
__device__ __forceinline__ void lzero(uint32_t (&d)[LW]) {
#pragma unroll
    for (int j = 0; j < LW; j++) d[j] = 0;
}
template <int LW>
__device__ __forceinline__ bool lany(const uint32_t (&d)[LW]) {
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < LW; j++) o |= d[j];
    return o != 0;
}

// Fan-in rows of one gate, loaded before it is evaluated (its record stays
// in shared memory; the header travels here).
template <int LW>
struct LaneIn {
    uint32_t h;                          // record header
    uint32_t fv[kInlineFanins][LW], ft[kInlineFanins][LW];
    uint32_t m0[LW];                     // mark row of fan-in 0 (when its bitmap bit is set)
    uint32_t fm[kInlineFanins][LW];      // FIXED modes: mark rows of fan-ins 0..3 with their bits set
    uint32_t sv[LW], st[LW];             // stage call pdf_mark: the gate's own given V and T
    bool bit0;                           // fan-in 0 holds a mark in this column block
};

template <int SEM, int MODE, int LW>
__device__ __forceinline__ void lane_load(const FwdArgs &a, const LanePlanes &P, const uint32_t *bm,
                                          const GateRec *rp, uint32_t g, uint32_t w, bool live, LaneIn<LW> &x) {
    constexpr bool FIX = SEM >= 2;
    const uint4 r0 = reinterpret_cast<const uint4 *>(rp)[0], r1 = reinterpret_cast<const uint4 *>(rp)[1];
    const uint32_t h = r0.x, nfi = (h >> 8) & 0xFFu;
    x.h = h;
    // Whether fan-in 0 holds a mark in the block: the same on every lane of
    // the warp (the branch in lane_gate that it guards holds warp votes), so
    // it is set before any lane leaves.  m0 is read only where bit0 and
    // RF_MARKF0 had it loaded.
    x.bit0 = MODE != FWD_SIM && !(h & (RF_INPT | RF_KILL)) && bit_test(bm, r1.w);
    // A lane past the last pair loads nothing: what it evaluates is masked.
    if (!live) return;
    if (h & RF_INPT) {
        if (MODE == FWD_MARK) {
            lload<LW>(lrow(P.V, g, P.ld4), x.fv[0]);
            lload<LW>(lrow(P.T, g, P.ld4), x.ft[0]);
        } else {
            const uint32_t pld4 = (uint32_t)(a.pi_ld * 4);
            lload_nc<LW>(lrow(reinterpret_cast<const char *>(a.pi_v + w), g, pld4), x.fv[0]);
            lload_nc<LW>(lrow(reinterpret_cast<const char *>(a.pi_t + w), g, pld4), x.ft[0]);
        }
        return;
    }
    if (MODE == FWD_MARK) {  // the gate's own values are given; fan-ins feed the side test only
        lload<LW>(lrow(P.V, g, P.ld4), x.sv);
        lload<LW>(lrow(P.T, g, P.ld4), x.st);
    }
    // A killed gate's value is S0 whatever its fan-ins (and it cannot mark):
    // nothing to load.  Fan-ins 0 .. nl - 1 follow warp-uniform branches on
    // the count, so absent fan-ins cost no predicated-off slots; a killed
    // fan-in is S0 (its row is not written), except in the stage call
    // pdf_mark, whose given planes are read as they are.
    if (h & RF_KILL) return;
    const uint32_t nl = min(nfi, (uint32_t)kInlineFanins);
    const auto fanin = [&](int q, uint32_t sw) {
        const uint32_t f = sw & ~SRC_ZERO;
        if (MODE == FWD_MARK || !(sw & SRC_ZERO)) {
            lload<LW>(lrow(P.V, f, P.ld4), x.fv[q]);
            lload<LW>(lrow(P.T, f, P.ld4), x.ft[q]);
        } else {
            lzero<LW>(x.fv[q]);
            lzero<LW>(x.ft[q]);
        }
        if (FIX && MODE != FWD_SIM) {
            if (bit_test(bm, f)) lload<LW>(lrow(P.M, f, P.ld4), x.fm[q]);
            else lzero<LW>(x.fm[q]);
        }
    };
    if (nl > 0) {
        fanin(0, r0.w);
        if (nl > 1) {
            fanin(1, r1.x);
            if (nl > 2) {
                fanin(2, r1.y);
                if (nl > 3) fanin(3, r1.z);
            }
        }
    }
    if (MODE != FWD_SIM && (h & RF_MARKF0) && x.bit0) lload<LW>(lrow(P.M, r1.w, P.ld4), x.m0);
}

// Evaluate, mark and store one gate; returns whether it holds a mark in the
// block (warp-uniform).  wm: the lane's word masks (pairs present).
template <int SEM, int MODE, int LW>
__device__ __forceinline__ bool lane_gate(const FwdArgs &a, const LanePlanes &P, uint32_t *bm, const GateRec *rp,
                                          uint32_t g, bool live, uint32_t nw, const uint32_t (&wm)[LW],
                                          const LaneIn<LW> &x) {
    constexpr bool FIX = SEM >= 2;
    const uint32_t h = x.h, nfi = (h >> 8) & 0xFFu;
    // fan-in q > 3 of the gate (its id from the edge array), read from its rows
    const auto far_row = [&](uint32_t q, uint32_t (&v)[LW], uint32_t (&t)[LW]) {
        const uint32_t f = __ldg(a.c.edges + rp->w[2] + q);
        lzero<LW>(v);
        lzero<LW>(t);
        if (live) {
            lload<LW>(lrow(P.V, f, P.ld4), v);
            lload<LW>(lrow(P.T, f, P.ld4), t);
        }
        return f;
    };
    uint32_t V[LW], T[LW], M[LW];
    lzero<LW>(M);
    if (h & RF_INPT) {
#pragma unroll
        for (int j = 0; j < LW; j++) {
            V[j] = x.fv[0][j] & wm[j];
            T[j] = x.ft[0][j] & wm[j];
        }
    } else if (MODE == FWD_MARK) {
#pragma unroll
        for (int j = 0; j < LW; j++) {
            V[j] = x.sv[j] & wm[j];
            T[j] = x.st[j] & wm[j];
        }
    } else if ((h & RF_KILL) || !live) {
        lzero<LW>(V);
        lzero<LW>(T);
        if (FIX && (h & RF_OINV)) {
#pragma unroll
            for (int j = 0; j < LW; j++) V[j] = wm[j];  // S0 inverted under both vectors: S1
        }
    } else {
        uint32_t v1[LW];
#pragma unroll
        for (int j = 0; j < LW; j++) eval_first(h, x.fv[0][j], x.ft[0][j], V[j], v1[j]);
        // fold steps in fan-in order, behind warp-uniform branches on the count
        const uint32_t nfold = hdr_nfold(h);
        const auto fold = [&](int q) {
#pragma unroll
            for (int j = 0; j < LW; j++) eval_fold<FIX>(h, V[j], v1[j], x.fv[q][j], x.ft[q][j]);
        };
        if (nfold >= 1) {
            fold(1);
            if (nfold >= 2) {
                fold(2);
                if (nfold >= 3) fold(3);
            }
        }
        for (uint32_t q = kInlineFanins; q <= nfold; q++) {
            uint32_t rv[LW], rt[LW];
            far_row(q, rv, rt);
#pragma unroll
            for (int j = 0; j < LW; j++) eval_fold<FIX>(h, V[j], v1[j], rv[j], rt[j]);
        }
#pragma unroll
        for (int j = 0; j < LW; j++) {
            eval_finish<FIX>(h, V[j], v1[j], T[j]);
            V[j] &= wm[j];
            T[j] &= wm[j];
        }
    }
    if (MODE != FWD_SIM) {  // markkernel.cuh:226-267
        const bool anyT = __any_sync(0xFFFFFFFFu, lany<LW>(T));
        if (h & RF_INPT) {
#pragma unroll
            for (int j = 0; j < LW; j++) M[j] = T[j];
        } else if ((h & RF_MARKF0) && x.bit0 && anyT) {
            // fan-in 0 (gate w[7]) holds a mark: its bitmap bit is set
#pragma unroll
            for (int j = 0; j < LW; j++) M[j] = T[j] & x.m0[j];
            if ((h & RF_SENS) && __any_sync(0xFFFFFFFFu, lany<LW>(M))) {
                // the side test over the fan-in rows already loaded (past the
                // fourth, read here)
                SensAcc s[LW];
                const bool or_like = (h & RF_IM) != 0;
#pragma unroll
                for (int j = 0; j < LW; j++) sens_init(s[j]);
#pragma unroll
                for (int q = 0; q < kInlineFanins; q++)
                    if ((uint32_t)q < nfi)
#pragma unroll
                        for (int j = 0; j < LW; j++) sens_step<SEM & 1>(s[j], or_like, x.fv[q][j], x.ft[q][j]);
                for (uint32_t q = kInlineFanins; q < nfi; q++) {
                    uint32_t rv[LW], rt[LW];
                    far_row(q, rv, rt);
#pragma unroll
                    for (int j = 0; j < LW; j++) sens_step<SEM & 1>(s[j], or_like, rv[j], rt[j]);
                }
#pragma unroll
                for (int j = 0; j < LW; j++) M[j] &= sens_result<SEM & 1>(s[j]);
            }
        } else if (FIX && (h & RF_MANY) && anyT) {
            // any fan-in may carry the path: its own mark enters the side test
            const uint32_t mor = flagmask(h, RF_IM), mxor = flagmask(h, RF_XOR), mand = ~(mor | mxor);
            SensAcc s[LW];
#pragma unroll
            for (int j = 0; j < LW; j++) sens_init(s[j]);
#pragma unroll
            for (int q = 0; q < kInlineFanins; q++)
                if ((uint32_t)q < nfi)
#pragma unroll
                    for (int j = 0; j < LW; j++)
                        sens_step_fixed<SEM == PDF_MARK_FIXED_NONROBUST>(s[j], mand, mor, mxor, x.fv[q][j],
                                                                         x.ft[q][j], x.fm[q][j]);
            for (uint32_t q = kInlineFanins; q < nfi; q++) {
                uint32_t rv[LW], rt[LW], rm[LW];
                const uint32_t f = far_row(q, rv, rt);
                lzero<LW>(rm);
                if (live && bit_test(bm, f)) lload<LW>(lrow(P.M, f, P.ld4), rm);
#pragma unroll
                for (int j = 0; j < LW; j++)
                    sens_step_fixed<SEM == PDF_MARK_FIXED_NONROBUST>(s[j], mand, mor, mxor, rv[j], rt[j], rm[j]);
            }
#pragma unroll
            for (int j = 0; j < LW; j++) M[j] = T[j] & sens_result<SEM == PDF_MARK_FIXED_NONROBUST>(s[j]);
        }
    }
    const bool marked = MODE != FWD_SIM && __any_sync(0xFFFFFFFFu, lany<LW>(M));
    if (live) {
        if (MODE != FWD_MARK && (a.store_all || (h & RF_SPILL) || marked)) {
            lstore<LW>(lrow(P.V, g, P.ld4), V, nw);
            lstore<LW>(lrow(P.T, g, P.ld4), T, nw);
        }
        if (MODE != FWD_SIM && (a.store_all || marked)) lstore<LW>(lrow(P.M, g, P.ld4), M, nw);
    }
    if (marked && (threadIdx.x & 31) == 0) atomicOr(bm + (g >> 5), 1u << (g & 31));
    return marked;
}

// U: gates per warp in flight (their fan-in rows are loaded before any of
// them is evaluated), as many as the registers hold.
template <int SEM, int MODE, int U, int LW>
__device__ __forceinline__ void forward_lanes_cta(const FwdArgs &a, const uint32_t blk) {
    extern __shared__ __align__(128) unsigned char smraw[];
    constexpr uint32_t BWL = 32 * LW;                    // words per column block
    constexpr uint32_t NF = BWL / kLaneCoverWords;       // cover bitmaps per block
    constexpr uint32_t SUBL = kLaneCoverWords / LW;      // lanes per cover bitmap
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
    const uint32_t w0 = blk * BWL, w = w0 + lane * LW;
    const bool live = w < a.W;
    const uint32_t nw = live ? min((uint32_t)LW, a.W - w) : 0u;  // words of the lane that hold pairs
    uint32_t wm[LW];
#pragma unroll
    for (int j = 0; j < LW; j++)
        wm[j] = w + j >= a.W ? 0u
                             : (w + j + 1 < a.W ? 0xFFFFFFFFu
                                                : ((a.n_pairs & 31) ? (1u << (a.n_pairs & 31)) - 1u : 0xFFFFFFFFu));
    LanePlanes P;
    P.ld4 = (uint32_t)(a.ld * 4);
    P.V = reinterpret_cast<char *>(a.V + w);
    P.T = reinterpret_cast<char *>(a.T + w);
    P.M = reinterpret_cast<char *>(a.M + w);
    uint32_t *bm = a.bm_shared ? reinterpret_cast<uint32_t *>(smraw + a.off_bm) : a.nzb + (size_t)blk * a.bm_words;
    uint32_t *gbm = a.nzb ? a.nzb + (size_t)blk * a.bm_words : nullptr;
    GateRec *recs = reinterpret_cast<GateRec *>(smraw + a.off_rec);  // [2][a.cap]
    const uint32_t *lo = a.c.level_off;

    if (MODE != FWD_SIM)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) bm[q] = 0;
    uint32_t *fine = MODE == FWD_FUSED && a.nzb_fine ? a.nzb_fine + (size_t)blk * NF * a.bm_words : nullptr;
    if (fine)
        for (uint32_t q = threadIdx.x; q < NF * a.bm_words; q += blockDim.x) fine[q] = 0;
    if (MODE == FWD_FUSED) {  // the batch's cover state (the cover kernels run after this one)
        if (a.active && threadIdx.x < BWL && w0 + threadIdx.x <= a.W) a.active[w0 + threadIdx.x] = 0;
        if (a.active && blk == 0 && threadIdx.x == 0) a.active[a.W] = 0;
        if (a.acc && blk == 0 && threadIdx.x == 0) {
            a.acc->batch_lo = 0;
            a.acc->batch_hi = 0;
            a.acc->batch_flags = 0;
            a.acc->done = 0;
            a.acc->n_over = 0;
            a.acc->done_over = 0;
        }
    }
    __syncthreads();

    // ------------------------------------------------------------- forward
    // Pieces (runs of one level, <= a.cap gates) in level order; each
    // piece's gate records are copied into shared memory (cp.async, 16 bytes
    // per thread and copy) while the piece before it is evaluated, and its
    // descriptor is loaded a piece earlier still.  One barrier per piece.
    const auto stage = [&](uint32_t ga, uint32_t gb, int buf) {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.c.rec + ga);
        uint4 *dst = reinterpret_cast<uint4 *>(recs + (size_t)buf * a.cap);
        for (uint32_t i = threadIdx.x; i < 2 * (gb - ga); i += blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + i)), "l"(src + i) : "memory");
    };
    // gates [pa, pb) of level pl: the next piece to evaluate; (na, nb, nlv):
    // the one after it, loaded a piece ahead
    uint32_t top = 0;  // levels below `top` may hold a forward mark
    uint32_t pa = a.pieces[0].a, pb = a.pieces[0].b, pl = a.pieces[0].level, na = 0, nb = 0, nlv = 0;
    if (a.n_pieces > 1) {
        na = a.pieces[1].a;
        nb = a.pieces[1].b;
        nlv = a.pieces[1].level;
    }
    stage(pa, pb, 0);
    bool any = false;
    uint32_t prev_level = 0;
    for (uint32_t i = 0; i < a.n_pieces; i++) {
        cp_async_wait_all();  // this thread's copies of piece i's records
        if (__syncthreads_or(any) && i) top = max(top, prev_level + 1);
        any = false;
        if (i + 1 < a.n_pieces) stage(na, nb, (i + 1) & 1);  // into the buffer of piece i - 1, which every warp has left
        const uint32_t ga = pa, gb = pb;
        prev_level = pl;
        pa = na;
        pb = nb;
        pl = nlv;
        if (i + 2 < a.n_pieces) {
            na = __ldg(&a.pieces[i + 2].a);
            nb = __ldg(&a.pieces[i + 2].b);
            nlv = __ldg(&a.pieces[i + 2].level);
        }
        const GateRec *rb = recs + (size_t)(i & 1) * a.cap;
        for (uint32_t g = ga + warp; g < gb; g += U * NW) {
            LaneIn<LW> x[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t gu = g + u * NW;
                if (gu < gb) lane_load<SEM, MODE, LW>(a, P, bm, rb + (gu - ga), gu, w, live, x[u]);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t gu = g + u * NW;
                if (gu < gb) any |= lane_gate<SEM, MODE, LW>(a, P, bm, rb + (gu - ga), gu, live, nw, wm, x[u]);
            }
        }
    }
    if (__syncthreads_or(any)) top = max(top, prev_level + 1);
    if constexpr (MODE == FWD_SIM) {
        return;
    } else {
        if (MODE == FWD_MARK && a.no_prune) return;
        // ------------------------------------------------- prune and merge
        // (markkernel.cuh:271-293, mergekernel.cuh:116-198) levels descending;
        // a warp takes 32-gate words of the bitmap and visits their marked
        // gates; a gate's pruned mark is final once its fan-outs' are.
        uint32_t maxlvl = 0;
        for (int l = (int)top - 1; l >= 0; l--) {
            const uint32_t ga = __ldg(lo + l), gb = __ldg(lo + l + 1);
            bool any = false;
            for (uint32_t q = (ga >> 5) + warp; q < (gb + 31) >> 5; q += NW) {
                uint32_t bits = bm[q];
                if (q == ga >> 5 && (ga & 31)) bits &= ~((1u << (ga & 31)) - 1u);
                if (q == (gb - 1) >> 5 && (gb & 31)) bits &= (1u << (gb & 31)) - 1u;
                while (bits) {
                    const uint32_t g = q * 32 + (__ffs(bits) - 1);
                    bits &= bits - 1;
                    const GateRec r = load_rec(a.c.rec + g);
                    uint32_t *mrow = lrow(P.M, g, P.ld4);
                    uint32_t mk[LW], keep[LW], nm[LW];
                    lzero<LW>(mk);
                    if (live) lload<LW>(mrow, mk);
#pragma unroll
                    for (int j = 0; j < LW; j++) {
                        mk[j] &= wm[j];  // words past the last pair hold no mark
                        keep[j] = rec_po(r) ? 0xFFFFFFFFu : 0u;
                    }
                    if (!rec_po(r)) {
                        const uint32_t nfo = r.w[1], base = r.w[2] + rec_nfi(r);
                        for (uint32_t k = 0; k < nfo; k += 4) {  // four fan-out rows in flight
                            uint32_t fo[4], m[4][LW];
#pragma unroll
                            for (int u = 0; u < 4; u++) fo[u] = k + u < nfo ? __ldg(a.c.edges + base + k + u) : kEmpty;
#pragma unroll
                            for (int u = 0; u < 4; u++) {
                                lzero<LW>(m[u]);
                                if (fo[u] != kEmpty && live && bit_test(bm, fo[u])) lload<LW>(lrow(P.M, fo[u], P.ld4), m[u]);
                            }
#pragma unroll
                            for (int j = 0; j < LW; j++) keep[j] |= m[0][j] | m[1][j] | m[2][j] | m[3][j];
                        }
                    }
                    bool changed = false;
#pragma unroll
                    for (int j = 0; j < LW; j++) {
                        nm[j] = mk[j] & keep[j];
                        changed |= nm[j] != mk[j];
                    }
                    if (live && changed) lstore<LW>(mrow, nm, nw);
                    const uint32_t nzl = __ballot_sync(0xFFFFFFFFu, lany<LW>(nm));  // lanes still marked
                    const bool nz = nzl != 0;
                    if (!nz) {
                        if (lane == 0) atomicAnd(bm + (g >> 5), ~(1u << (g & 31)));
                    } else if (fine && lane < NF && ((nzl >> (SUBL * lane)) & ((1u << SUBL) - 1u))) {
                        atomicOr(fine + (size_t)lane * a.bm_words + (g >> 5), 1u << (g & 31));  // bitmap `lane`
                    }
                    if (nz && MODE == FWD_FUSED && a.first_x) {  // merge: first falling / rising pair
                        uint32_t v[LW];
                        lzero<LW>(v);
                        if (live) lload<LW>(lrow(P.V, g, P.ld4), v);
                        uint32_t cx = kEmpty, cy = kEmpty;
#pragma unroll
                        for (int j = LW - 1; j >= 0; j--) {  // the lowest word last
                            const uint32_t x = nm[j] & ~v[j], y = nm[j] & v[j];
                            if (x) cx = (w + j) * 32 + (__ffs(x) - 1);
                            if (y) cy = (w + j) * 32 + (__ffs(y) - 1);
                        }
                        cx = __reduce_min_sync(0xFFFFFFFFu, cx);
                        cy = __reduce_min_sync(0xFFFFFFFFu, cy);
                        if (lane == 0) {
                            if (cx != kEmpty) atomicMin(a.first_x + g, a.pair_base + cx);
                            if (cy != kEmpty) atomicMin(a.first_y + g, a.pair_base + cy);
                        }
                    }
                    any |= nz;
                }
            }
            if (__syncthreads_or(any) && !maxlvl) maxlvl = (uint32_t)l + 1;
        }
        // publish the bitmap of surviving marks for the cover kernels
        if (a.bm_shared && gbm)
            for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) gbm[q] = bm[q];
        if (threadIdx.x == 0) a.blk_maxlvl[blk] = maxlvl;
        if (fine && threadIdx.x < NF) a.maxlvl_fine[blk * NF + threadIdx.x] = maxlvl;
    }
}

// Gates per warp in flight, by tile and semantics (the FIXED modes and the
// stage call pdf_mark carry more rows per gate).  More warps beat more gates
// per warp: on a 1M-gate circuit at 64 words, 1,024 threads with one gate
// each took 36 ms against 46 ms for 512 threads with three or four.
template <int SEM, int MODE, int LW>
struct LaneU {
    static constexpr bool heavy = SEM >= 2 || MODE == FWD_MARK;
    static constexpr int value = LW == 1 ? (heavy ? 2 : 2) : LW == 2 ? (heavy ? 1 : 1) : (heavy ? 1 : 1);
};

template <int SEM, int MODE, int LW>
__global__ void __launch_bounds__(lane_threads(32 * LW), 1) k_forward_lanes(const FwdArgs a) {
    forward_lanes_cta<SEM, MODE, LaneU<SEM, MODE, LW>::value, LW>(a, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Cover.
// ---------------------------------------------------------------------------

// Pairs that first-detect some net in this batch: bitmap, and a list (in no
// order) of each such pair once.
// Gate g: its first-detecting pairs into the bitmap; emit(d) for each pair
// whose bit it set.
template <class Emit>
__device__ __forceinline__ void active_gate(const CoverArgs &a, uint32_t g, Emit emit) {
    const uint32_t f[2] = {a.first_x[g], a.first_y[g]};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const uint32_t d = f[k] - a.pair_base;
        if (f[k] == kEmpty || d >= a.n_pairs) continue;
        const uint32_t bit = 1u << (d & 31);
        if (!(atomicOr(a.active + (d >> 5), bit) & bit)) emit(d);
    }
}
__global__ void k_active(const CoverArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.c.n_gates) return;
    active_gate(a, g, [&](uint32_t d) { a.active_list[atomicAdd(a.active_count, 1u)] = d; });
}

// ---- segments longer than one net ----------------------------------------

constexpr unsigned long long kEmpty64 = ~0ull;
__device__ __forceinline__ uint64_t key_slot(unsigned long long k, uint64_t mask) {
    k ^= k >> 33;  // 64-bit finaliser (murmur3 fmix64)
    k *= 0xFF51AFD7ED558CCDull;
    k ^= k >> 33;
    k *= 0xC4CEB9FE1A85EC53ull;
    k ^= k >> 33;
    return k & mask;
}
// Open addressing, linear probing, at most one pass over the table.
__device__ __forceinline__ bool first_set_insert(unsigned long long *t, uint64_t mask, unsigned long long key) {
    uint64_t h = key_slot(key, mask);
    for (uint64_t i = 0; i <= mask; i++) {
        const unsigned long long old = atomicCAS(t + h, kEmpty64, key);
        if (old == kEmpty64 || old == key) return true;
        h = (h + 1) & mask;
    }
    return false;
}
__device__ __forceinline__ bool first_set_find(const unsigned long long *t, uint64_t mask, unsigned long long key) {
    uint64_t h = key_slot(key, mask);
    for (uint64_t i = 0; i <= mask; i++) {
        const unsigned long long v = t[h];
        if (v == key) return true;
        if (v == kEmpty64) return false;
        h = (h + 1) & mask;
    }
    return false;
}

// Per segment: its first pairs that fall in this batch mark every net of the
// segment as first for that pair (findActiveThreads, coverkernel.cuh:130-154),
// and list the pair as active.
__global__ void k_seg_first(const CoverArgs a) {
    const uint32_t N = a.seg.N;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < a.seg.S;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f[2] = {a.first_x[s], a.first_y[s]};
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const uint32_t d = f[k] - a.pair_base;
            if (f[k] == kEmpty || d >= a.n_pairs) continue;
            const uint32_t *sg = a.seg.segs + s * N;
            for (uint32_t i = 0; i < N; i++)
                if (!first_set_insert(a.seg_first, a.seg_first_mask, ((unsigned long long)sg[i] << 32) | d))
                    atomicOr(&a.acc->err, kErrHashFull);
            const uint32_t bit = 1u << (d & 31);
            if (!(atomicOr(a.active + (d >> 5), bit) & bit)) a.active_list[atomicAdd(a.active_count, 1u)] = d;
        }
    }
}

// After the forward kernel: for each column block, each marked net g0 and
// each segment starting at g0 whose nets are all marked in the block, the
// first falling / rising pair marking all of them (kernSegmentReduce2<N>,
// mergekernel.cuh:116-198; direction by the first net's value, :140-143).
// One CTA per column block; a warp per bitmap word, lanes over segments.
__global__ void k_seg_merge(const SegMergeArgs a) {
    const uint32_t blk = blockIdx.x, w0 = blk * a.bw, wend = min(a.W, w0 + a.bw), N = a.seg.N;
    const uint32_t *bm = a.nzb + (size_t)blk * a.bm_words;
    const uint32_t lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (uint32_t q = threadIdx.x >> 5; q < a.bm_words; q += nw) {
        uint32_t bits = bm[q];
        while (bits) {
            const uint32_t g0 = q * 32 + (__ffs(bits) - 1);
            bits &= bits - 1;
            const uint32_t s1 = a.seg.seg_off[g0 + 1];
            for (uint32_t s = a.seg.seg_off[g0] + lane; s < s1; s += 32) {
                const uint32_t *sg = a.seg.segs + (size_t)s * N;
                bool ok = true;
                for (uint32_t i = 1; i < N && ok; i++) ok = bit_test(bm, sg[i]);
                if (!ok) continue;
                uint32_t cx = kEmpty, cy = kEmpty;
                for (uint32_t w = w0; w < wend && (cx == kEmpty || cy == kEmpty); w++) {
                    uint32_t m = a.M[(size_t)g0 * a.ld + w];
                    for (uint32_t i = 1; i < N && m; i++) m &= a.M[(size_t)sg[i] * a.ld + w];
                    if (!m) continue;
                    const uint32_t v = a.V[(size_t)g0 * a.ld + w];
                    const uint32_t x = m & ~v, y = m & v;
                    if (x && cx == kEmpty) cx = w * 32 + (__ffs(x) - 1);
                    if (y && cy == kEmpty) cy = w * 32 + (__ffs(y) - 1);
                }
                if (cx != kEmpty) atomicMin(a.first_x + s, a.pair_base + cx);
                if (cy != kEmpty) atomicMin(a.first_y + s, a.pair_base + cy);
            }
        }
    }
}

// Dense variant over given planes (stage call pdf_merge): a warp per
// (segment, 32-word chunk), warp minimum, one atomicMin per warp.
__global__ void k_seg_merge_dense(const SegArgs seg, const uint32_t *V, const uint32_t *M, uint64_t ld,
                                  uint64_t n_pairs, uint32_t W, uint32_t pair_base, uint32_t *first_x,
                                  uint32_t *first_y) {
    const uint32_t chunks = (W + 31) / 32;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= (uint64_t)seg.S * chunks) return;
    const uint32_t s = (uint32_t)(warp / chunks), w = (uint32_t)(warp % chunks) * 32 + lane;
    const uint32_t *sg = seg.segs + (size_t)s * seg.N;
    uint32_t cx = kEmpty, cy = kEmpty;
    if (w < W) {
        uint32_t m = M[(size_t)sg[0] * ld + w];
        for (uint32_t i = 1; i < seg.N && m; i++) m &= M[(size_t)sg[i] * ld + w];
        if (w == W - 1 && (n_pairs & 31)) m &= (1u << (n_pairs & 31)) - 1u;
        if (m) {
            const uint32_t v = V[(size_t)sg[0] * ld + w];
            const uint32_t x = m & ~v, y = m & v;
            if (x) cx = w * 32 + (__ffs(x) - 1);
            if (y) cy = w * 32 + (__ffs(y) - 1);
        }
    }
    cx = __reduce_min_sync(0xFFFFFFFFu, cx);
    cy = __reduce_min_sync(0xFFFFFFFFu, cy);
    if (lane == 0) {
        if (cx != kEmpty) atomicMin(first_x + s, pair_base + cx);
        if (cy != kEmpty) atomicMin(first_y + s, pair_base + cy);
    }
}

// Close a batch: total = min(2^128 - 1, total + batch); flags are sticky.
__device__ void batch_close(DevAcc *acc, uint64_t n_pairs) {
    pdf_u128 b = ((pdf_u128)acc->batch_hi << 64) | acc->batch_lo;
    if (acc->batch_flags & PDF_FLAG_OVERFLOW) {
        b = ~(pdf_u128)0;
        acc->batch_lo = ~0ull;
        acc->batch_hi = ~0ull;
    }
    pdf_u128 t = ((pdf_u128)acc->total_hi << 64) | acc->total_lo;
    bool ovf = false;
    t = add_sat(t, b, ovf);
    acc->total_lo = (unsigned long long)t;
    acc->total_hi = (unsigned long long)(t >> 64);
    acc->flags |= acc->batch_flags | (ovf ? PDF_FLAG_OVERFLOW : 0u);
    acc->pairs += n_pairs;
}

__device__ __forceinline__ pdf_u128 shfl_down_u128(pdf_u128 v, int d) {
    const unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
    const unsigned long long l2 = __shfl_down_sync(0xFFFFFFFFu, lo, d);
    const unsigned long long h2 = __shfl_down_sync(0xFFFFFFFFu, hi, d);
    return ((pdf_u128)h2 << 64) | l2;
}

// Add a 128-bit count into (lo, hi) with 64-bit atomics; flags an overflow.
__device__ void atomic_add_u128(unsigned long long *lo, unsigned long long *hi, unsigned int *flags,
                                pdf_u128 v) {
    const unsigned long long vl = (unsigned long long)v, vh = (unsigned long long)(v >> 64);
    const unsigned long long old = atomicAdd(lo, vl);
    const unsigned long long carry = (old + vl < old) ? 1ull : 0ull;
    if (vh == ~0ull && carry) {
        atomicOr(flags, PDF_FLAG_OVERFLOW);
        return;
    }
    const unsigned long long add = vh + carry;
    if (add) {
        const unsigned long long oh = atomicAdd(hi, add);
        if (oh + add < oh) atomicOr(flags, PDF_FLAG_OVERFLOW);
    }
}

// Exclusive prefix sum of one value per thread over the CTA (blockDim a
// multiple of 32, <= 1024); *total gets the sum.  Uses s_warp[32].
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t v, uint32_t *s_warp, uint32_t *total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? s_warp[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        if (lane < nw) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp ? s_warp[warp - 1] : 0u) + x - v;
    *total = s_warp[nw - 1];
    __syncthreads();
    return before;
}

// Index of gate g in the ascending list lid[0, n), or kEmpty.
__device__ __forceinline__ uint32_t find_net(const uint32_t *lid, uint32_t n, uint32_t g) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (lid[mid] < g) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && lid[lo] == g ? lo : kEmpty;
}

// Level of gate g: the last l with level_off[l] <= g.
__device__ __forceinline__ uint32_t level_of(const uint32_t *lo_tab, uint32_t n_levels, uint32_t g) {
    uint32_t lo = 0, hi = n_levels;  // answer in [lo, hi)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (lo_tab[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Path counting (kernCover, coverkernel.cuh:193-229, and kernSumSingle,
// :77-105) for the pairs that first-detect some net.  One CTA per such pair
// (persistent over the list).  All global reads are gathered first, each
// phase in parallel across the CTA:
//   A  the nets with a surviving mark in the pair's column block (bitmap
//      words, in gate order, CAND at a time),
//   B  of those, the nets the pair itself marks (one mark word each): the
//      pair's net list, ascending (hence level order),
//   C  per listed net its record, first-detect ids, level, and its fan-outs
//      that are listed (as list indices);
// then the recurrence runs in shared memory, levels descending:
//   H = [po] + sum h(fo);  C = sum c(fo);  first = pid is first_x or first_y
//   c = C + (first ? H : 0);  h = first ? 0 : H;  h = 0 on INPT
// (a net the pair does not mark has h = c = 0).  Level-0 INPT c values are
// the pair's count.  A pair marking more than net_cap nets is counted by
// nothing here: cover_pair returns true and the caller queues the pair for
// the spill cover (spill_pair); fan-out lists past the adjacency buffer are
// read in place.
constexpr uint32_t kCoverCand = 4096;   // candidates per window (k_cover and the large-table batch cover)
constexpr uint32_t kCoverCandSmall = 2048;  // candidates per window of the small-table batch cover
constexpr uint32_t kCoverLevels = 2048; // level table entries kept in shared memory
constexpr uint32_t kNetPo = 1u << 31, kNetInpt = 1u << 30, kNetFirst = 1u << 29, kNetLevel = (1u << 29) - 1;
// Shared memory of cover_pair's tables for `cap` nets and a window of
// `cand` candidates: h, c (u128), the net list, flags, adjacency offsets and
// lengths, 4 cap adjacency entries and the candidates.
__host__ __device__ constexpr size_t cover_smem_tables(uint32_t cap, uint32_t cand) {
    return (size_t)cap * (2 * sizeof(pdf_u128) + 4 * 4 + 4 * 4) + (size_t)cand * 4;
}
// Byte offset of the level table in k_cover's shared memory (after the tables).
__host__ __device__ constexpr size_t cover_smem_lvt(uint32_t cap) { return cover_smem_tables(cap, kCoverCand); }

// Each thread of the candidate test below takes up to CAND / blockDim
// candidates in registers: the cover kernels run 256 threads.
constexpr uint32_t kCoverThreads = 256;
static_assert(kCoverCand / kCoverThreads <= 16, "cover_pair keeps 16 candidate mark words per thread");
static_assert(kCoverCandSmall % kCoverThreads == 0 && kCoverCandSmall <= kCoverCand, "small window");

// Paths primary input g credits to pair p (the values the reference dumps to
// gpucover.log, coverkernel.cuh:44-66).
__device__ __forceinline__ void put_pi_count(const CoverArgs &a, uint32_t g, uint32_t p, pdf_u128 c) {
    unsigned long long *d = a.pi_counts + ((size_t)g * a.n_pairs + p) * 2;
    d[0] = (unsigned long long)c;
    d[1] = (unsigned long long)(c >> 64);
}

// The cover of pair p (index within the batch) of the circuit in `a`;
// lo_tab is its level table (shared or global memory); cap: nets the table
// holds; CAND: candidates per window.  Returns true (the same in every
// thread) when the pair marks more nets than the table holds: then nothing
// is counted.
template <uint32_t CAND>
__device__ __forceinline__ bool cover_pair(const CoverArgs &a, const uint32_t p, const uint32_t *lo_tab,
                                           const uint32_t cap) {
    extern __shared__ __align__(128) unsigned char smraw[];
    constexpr uint32_t kPer = CAND / kCoverThreads;  // candidates per thread and window
    const uint32_t acap = 4 * cap;
    pdf_u128 *hv = reinterpret_cast<pdf_u128 *>(smraw);
    pdf_u128 *cv = hv + cap;
    uint32_t *lid = reinterpret_cast<uint32_t *>(cv + cap);  // [cap] listed nets, ascending
    uint32_t *info = lid + cap;                               // [cap] kNet* flags | level
    uint32_t *aoff = info + cap;                              // [cap] adjacency offset, kEmpty: read in place
    uint32_t *acnt = aoff + cap;                              // [cap] adjacency length
    uint32_t *adj = acnt + cap;                               // [4 cap] listed fan-outs (list indices)
    uint32_t *cand = adj + acap;                              // [CAND]
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_n, s_adj, s_over;
    __shared__ pdf_u128 s_red[8];
    __shared__ unsigned int s_flags;

    const uint32_t L = a.c.n_levels;
    const uint32_t pid = a.pair_base + p;
    const uint32_t wp = p >> 5, bit = p & 31, blk = wp / a.bw;
    const uint32_t *nzb = a.nzb + (size_t)blk * a.bm_words;
    const uint32_t top = a.blk_maxlvl[blk];
    const uint32_t gend = lo_tab[top];
    const uint32_t nwords = (gend + 31) / 32;
    if (threadIdx.x == 0) {
        s_n = 0;
        s_adj = 0;
        s_over = 0;
        s_flags = 0;
    }
    __syncthreads();
    // ---- A: every thread counts the candidates (nets with a surviving mark in
    // the block: bitmap bits) of its own run of bitmap words; one scan orders
    // them
    const uint32_t per_w = (nwords + blockDim.x - 1) / blockDim.x;
    const uint32_t q_lo = min(nwords, threadIdx.x * per_w), q_hi = min(nwords, q_lo + per_w);
    auto word = [&](uint32_t q) {
        uint32_t b = nzb[q];
        if (q == nwords - 1 && (gend & 31)) b &= (1u << (gend & 31)) - 1u;
        return b;
    };
    uint32_t mine = 0;
    for (uint32_t q = q_lo; q < q_hi; q++) mine += __popc(word(q));
    uint32_t total_c;
    const uint32_t first_c = block_scan_excl(mine, s_warp, &total_c);
    // ---- B: in windows of CAND candidates, those the pair marks (one
    // mark word each) join the pair's list, in gate order
    for (uint32_t c_lo = 0; c_lo < total_c; c_lo += CAND) {
        const uint32_t c_hi = min(total_c, c_lo + CAND);
        if (first_c < c_hi && first_c + mine > c_lo) {  // this thread's candidates in the window
            uint32_t idx = first_c;
            for (uint32_t q = q_lo; q < q_hi && idx < c_hi; q++) {
                uint32_t b = word(q);
                for (; b && idx < c_hi; idx++, b &= b - 1)
                    if (idx >= c_lo) cand[idx - c_lo] = q * 32 + (__ffs(b) - 1);
            }
        }
        __syncthreads();
        const uint32_t nc = c_hi - c_lo;
        // each thread tests a contiguous run of candidates (order kept)
        const uint32_t per = (nc + blockDim.x - 1) / blockDim.x;
        const uint32_t c0 = min(nc, threadIdx.x * per), c1 = min(nc, c0 + per);
        uint32_t keep = 0, nk = 0;  // per <= kPer <= 16: one bit each
        uint32_t mw[kPer];
#pragma unroll
        for (int k = 0; k < (int)kPer; k++) mw[k] = c0 + k < c1 ? a.M[(size_t)cand[c0 + k] * a.ld + wp] : 0u;
#pragma unroll
        for (int k = 0; k < (int)kPer; k++) {
            const uint32_t m = (mw[k] >> bit) & 1u;
            keep |= m << k;
            nk += m;
        }
        uint32_t nl;
        const uint32_t at = block_scan_excl(nk, s_warp, &nl);
        const uint32_t base = s_n;
        if (base + nl > cap) {
            if (threadIdx.x == 0) s_over = 1;
        } else {
            uint32_t o = base + at;
            for (uint32_t i = c0; i < c1; i++)
                if ((keep >> (i - c0)) & 1u) lid[o++] = cand[i];
        }
        __syncthreads();
        if (threadIdx.x == 0 && !s_over) s_n = base + nl;
        __syncthreads();
        if (s_over) break;
    }
    if (s_over) {  // more nets than the list holds
        __syncthreads();
        return true;
    }
    const uint32_t n = s_n;
    // ---- C: records, first ids, levels, listed fan-outs
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t g = lid[i];
        const GateRec r = load_rec(a.c.rec + g);
        bool first;
        if (a.seg.N > 1) {
            first = first_set_find(a.seg_first, a.seg_first_mask, ((unsigned long long)g << 32) | p);
        } else {
            const uint32_t fx = a.first_x[g], fy = a.first_y[g];
            first = fx == pid || fy == pid;
        }
        const uint32_t nfo = r.w[1], eb = r.w[2] + rec_nfi(r);
        uint32_t k = 0;
        for (uint32_t j = 0; j < nfo; j += 4) {  // four fan-out loads in flight
            uint32_t fo[4];
#pragma unroll
            for (int u = 0; u < 4; u++) fo[u] = j + u < nfo ? __ldg(a.c.edges + eb + j + u) : kEmpty;
#pragma unroll
            for (int u = 0; u < 4; u++) k += fo[u] != kEmpty && find_net(lid, n, fo[u]) != kEmpty ? 1u : 0u;
        }
        info[i] = (rec_po(r) ? kNetPo : 0u) | (rec_type(r) == PDF_INPT ? kNetInpt : 0u) |
                  (first ? kNetFirst : 0u) | level_of(lo_tab, L, g);
        const uint32_t o = k ? atomicAdd(&s_adj, k) : 0u;
        if (o + k > acap) {
            aoff[i] = kEmpty;  // fan-outs read in place during the recurrence
            acnt[i] = nfo;
        } else {
            aoff[i] = o;
            acnt[i] = k;
            uint32_t w = o;
            for (uint32_t j = 0; j < nfo && k; j++) {
                const uint32_t x = find_net(lid, n, __ldg(a.c.edges + eb + j));
                if (x != kEmpty) adj[w++] = x;
            }
        }
    }
    __syncthreads();
    // ---- the recurrence, levels descending.  The list is in gate order, so
    // each level's nets are one run of it: bnd[l] = the first listed net of
    // level >= l (binary searches, in parallel), and a level without nets
    // costs neither a pass over the list nor a barrier.
    pdf_u128 total = 0;
    bool ovf = false;
    const uint32_t lv_hi = n ? (info[n - 1] & kNetLevel) : 0;
    uint32_t *bnd = cand;  // [lv_hi + 2] (the candidates are no longer needed)
    const bool runs = lv_hi + 2 <= CAND;
    if (runs) {
        for (uint32_t l = threadIdx.x; l <= lv_hi + 1; l += blockDim.x) {
            const uint32_t g0 = lo_tab[l];
            uint32_t lo = 0, hi = n;  // first index with lid >= g0
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (lid[mid] < g0) lo = mid + 1;
                else hi = mid;
            }
            bnd[l] = lo;
        }
        __syncthreads();
    }
    for (int lv = (int)lv_hi; lv >= 0 && n; lv--) {
        const uint32_t i0 = runs ? bnd[lv] : 0, i1 = runs ? bnd[lv + 1] : n;
        if (i0 == i1) continue;  // the same in every thread
        for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const uint32_t inf = info[i];
            if ((inf & kNetLevel) != (uint32_t)lv) continue;
            pdf_u128 H = (inf & kNetPo) ? 1 : 0, C = 0;
            bool dummy = false;
            auto add = [&](uint32_t x) {
                C = add_sat(C, cv[x], ovf);
                H = add_sat(H, hv[x], dummy);
            };
            if (aoff[i] != kEmpty) {
                for (uint32_t j = 0; j < acnt[i]; j++) add(adj[aoff[i] + j]);
            } else {
                const GateRec r = load_rec(a.c.rec + lid[i]);
                const uint32_t eb = r.w[2] + rec_nfi(r);
                for (uint32_t j = 0; j < acnt[i]; j++) {
                    const uint32_t x = find_net(lid, n, __ldg(a.c.edges + eb + j));
                    if (x != kEmpty) add(x);
                }
            }
            pdf_u128 c = C, h = H;
            if (inf & kNetFirst) {
                c = add_sat(C, H, ovf);
                h = 0;
            }
            if (c == ~(pdf_u128)0) ovf = true;
            if (inf & kNetInpt) {
                h = 0;
                if (lv == 0) {
                    total = add_sat(total, c, ovf);
                    if (a.pi_counts) put_pi_count(a, lid[i], p, c);
                }
            }
            hv[i] = h;
            cv[i] = c;
        }
        __syncthreads();
    }
    // ---- the pair's count into the batch count
    for (int d = 16; d > 0; d >>= 1) total = add_sat(total, shfl_down_u128(total, d), ovf);
    if (ovf) atomicOr(&s_flags, PDF_FLAG_OVERFLOW);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = total;
    __syncthreads();
    if (threadIdx.x < 32) {
        pdf_u128 t = threadIdx.x < (blockDim.x + 31) / 32 ? s_red[threadIdx.x] : 0;
        bool o2 = false;
        for (int d = 16; d > 0; d >>= 1) t = add_sat(t, shfl_down_u128(t, d), o2);
        if (threadIdx.x == 0) {
            if (o2 || s_flags) atomicOr(&a.acc->batch_flags, PDF_FLAG_OVERFLOW);
            if (t) atomic_add_u128(&a.acc->batch_lo, &a.acc->batch_hi, &a.acc->batch_flags, t);
        }
    }
    __syncthreads();
    return false;
}

// The same recurrence for a pair that marks more nets than cover_pair's
// table holds, with every net's (h, c) in global memory: slot = [2][n_gates]
// u128, indexed by gate.  Levels descending from the column block's highest
// marked level; a net takes part when its bitmap bit is set and the pair
// marks it (the mark bit read from the plane).
__device__ void spill_pair(const CoverArgs &a, const uint32_t p, pdf_u128 *Hs) {
    __shared__ pdf_u128 s_red[8];
    __shared__ unsigned int s_flags;
    pdf_u128 *Cs = Hs + a.c.n_gates;
    const uint32_t pid = a.pair_base + p;
    const uint32_t wp = p >> 5, bit = p & 31, blk = wp / a.bw;
    const uint32_t *nzb = a.nzb + (size_t)blk * a.bm_words;
    const uint32_t top = a.blk_maxlvl[blk];
    if (threadIdx.x == 0) s_flags = 0;
    __syncthreads();
    auto marks = [&](uint32_t g) { return bit_test(nzb, g) && ((a.M[(size_t)g * a.ld + wp] >> bit) & 1u); };
    pdf_u128 total = 0;
    bool ovf = false;
    for (int lv = (int)top - 1; lv >= 0; lv--) {
        const uint32_t g1 = __ldg(a.c.level_off + lv + 1);
        for (uint32_t g = __ldg(a.c.level_off + lv) + threadIdx.x; g < g1; g += blockDim.x) {
            if (!marks(g)) continue;
            const GateRec r = load_rec(a.c.rec + g);
            pdf_u128 H = rec_po(r) ? 1 : 0, C = 0;
            bool dummy = false;
            const uint32_t nfo = r.w[1], eb = r.w[2] + rec_nfi(r);
            for (uint32_t k = 0; k < nfo; k++) {
                const uint32_t fo = __ldg(a.c.edges + eb + k);
                if (!marks(fo)) continue;
                C = add_sat(C, Cs[fo], ovf);
                H = add_sat(H, Hs[fo], dummy);
            }
            const bool first = a.seg.N > 1
                                   ? first_set_find(a.seg_first, a.seg_first_mask, ((unsigned long long)g << 32) | p)
                                   : (a.first_x[g] == pid || a.first_y[g] == pid);
            pdf_u128 c = C, h = H;
            if (first) {
                c = add_sat(C, H, ovf);
                h = 0;
            }
            if (c == ~(pdf_u128)0) ovf = true;
            if (rec_type(r) == PDF_INPT) {
                h = 0;
                if (lv == 0) {
                    total = add_sat(total, c, ovf);
                    if (a.pi_counts) put_pi_count(a, g, p, c);
                }
            }
            Hs[g] = h;
            Cs[g] = c;
        }
        __syncthreads();
    }
    for (int d = 16; d > 0; d >>= 1) total = add_sat(total, shfl_down_u128(total, d), ovf);
    if (ovf) atomicOr(&s_flags, PDF_FLAG_OVERFLOW);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = total;
    __syncthreads();
    if (threadIdx.x < 32) {
        pdf_u128 t = threadIdx.x < (blockDim.x + 31) / 32 ? s_red[threadIdx.x] : 0;
        bool o2 = false;
        for (int d = 16; d > 0; d >>= 1) t = add_sat(t, shfl_down_u128(t, d), o2);
        if (threadIdx.x == 0) {
            if (o2 || s_flags) atomicOr(&a.acc->batch_flags, PDF_FLAG_OVERFLOW);
            if (t) atomic_add_u128(&a.acc->batch_lo, &a.acc->batch_hi, &a.acc->batch_flags, t);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ pdf_u128 *spill_slot(const CoverArgs &a, uint32_t k) {
    return reinterpret_cast<pdf_u128 *>(a.spill) + (size_t)k * 2 * a.c.n_gates;
}

__global__ void __launch_bounds__(kCoverThreads) k_cover(const CoverArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    uint32_t *lvt = reinterpret_cast<uint32_t *>(smraw + cover_smem_lvt(a.hash_cap));  // [kCoverLevels] level_off
    const uint32_t L = a.c.n_levels;
    const bool lv_shared = L + 1 <= kCoverLevels;
    if (lv_shared)
        for (uint32_t i = threadIdx.x; i <= L; i += blockDim.x) lvt[i] = a.c.level_off[i];
    const uint32_t *lo_tab = lv_shared ? lvt : a.c.level_off;
    __syncthreads();
    const uint32_t n_active = *a.active_count;
    for (uint32_t ai = blockIdx.x; ai < n_active; ai += gridDim.x) {
        const uint32_t p = a.active_list[ai];
        if (cover_pair<kCoverCand>(a, p, lo_tab, a.hash_cap) && threadIdx.x == 0) {
            if (a.spill_slots) a.over_list[atomicAdd(&a.acc->n_over, 1u)] = p;  // for k_cover_spill
            else atomicOr(&a.acc->err, kErrHashFull);
        }
    }
    // the last CTA to finish closes the batch, unless pairs wait for the spill cover
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&a.acc->done, 1u) == gridDim.x - 1) {
            __threadfence();
            if (!a.acc->n_over) batch_close(a.acc, a.n_pairs);
            a.acc->done = 0;
        }
    }
}

// After k_cover: the pairs it queued, one per CTA at a time (CTA k uses
// spill slot k); the last CTA closes the batch.
__global__ void __launch_bounds__(kCoverThreads) k_cover_spill(const CoverArgs a) {
    const uint32_t n_over = a.acc->n_over;
    if (!n_over) return;  // k_cover closed the batch
    for (uint32_t j = blockIdx.x; j < n_over; j += gridDim.x) spill_pair(a, a.over_list[j], spill_slot(a, blockIdx.x));
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&a.acc->done_over, 1u) == gridDim.x - 1) {
            __threadfence();
            batch_close(a.acc, a.n_pairs);
            a.acc->n_over = 0;
            a.acc->done_over = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Batched grading: many circuits in one pass of three launches.  Circuit i
// owns CTAs [bpref[i], bpref[i+1]) of k_batch_forward and gates
// [gpref[i], gpref[i+1]) of k_batch_active; the first-detecting pairs of all
// circuits form one item list that k_batch_cover works through.  Each
// circuit's arguments live in device arrays, so the launches can be captured
// once in a CUDA graph and replayed; with `append` the last cover CTA also
// advances every circuit's pair_base by its pair count, so the next replay
// grades the next vector pairs of each circuit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t prefix_find(const uint32_t *pref, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;  // last i with pref[i] <= x
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(pref + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One launch per class of circuits (equal CTAs per SM): this launch's CTAs
// are the batch's CTAs blk0 .. blk0 + gridDim.x - 1.
template <int BW, int SEM>
__global__ void __launch_bounds__(BW >= 8 ? 512 : 1024)
    k_batch_forward(const FwdArgs *args, const uint32_t *bpref, uint32_t n, BatchCtl *ctl, uint32_t blk0) {
    __shared__ FwdArgs s_a;
    __shared__ uint32_t s_blk;
    if (threadIdx.x == 0) {
        const uint32_t gb = blk0 + blockIdx.x;
        const uint32_t ci = prefix_find(bpref, n, gb);
        s_a = args[ci];
        s_blk = gb - __ldg(bpref + ci);
        if (gb == 0) {
            ctl->n_items = 0;
            ctl->done = 0;
            ctl->err = 0;
            ctl->n_over = 0;
            ctl->done_over = 0;
            ctl->n_mid = 0;
            ctl->done_mid = 0;
        }
    }
    __syncthreads();
    forward_cta<BW, SEM, FWD_FUSED>(s_a, s_blk);
}

// The same for the circuits of a batch that take a lane tile.
template <int SEM, int LW>
__global__ void __launch_bounds__(lane_threads(32 * LW), 1)
    k_batch_forward_lanes(const FwdArgs *args, const uint32_t *bpref, uint32_t n, BatchCtl *ctl, uint32_t blk0) {
    __shared__ FwdArgs s_a;
    __shared__ uint32_t s_blk;
    if (threadIdx.x == 0) {
        const uint32_t gb = blk0 + blockIdx.x;
        const uint32_t ci = prefix_find(bpref, n, gb);
        s_a = args[ci];
        s_blk = gb - __ldg(bpref + ci);
        if (gb == 0) {
            ctl->n_items = 0;
            ctl->done = 0;
            ctl->err = 0;
            ctl->n_over = 0;
            ctl->done_over = 0;
            ctl->n_mid = 0;
            ctl->done_mid = 0;
        }
    }
    __syncthreads();
    forward_lanes_cta<SEM, FWD_FUSED, LaneU<SEM, FWD_FUSED, LW>::value, LW>(s_a, s_blk);
}

__global__ void k_batch_active(const CoverArgs *args, const uint32_t *gpref, uint32_t n, uint2 *items,
                               BatchCtl *ctl) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= __ldg(gpref + n)) return;
    const uint32_t ci = prefix_find(gpref, n, t);
    const CoverArgs &a = args[ci];
    active_gate(a, t - __ldg(gpref + ci),
                [&](uint32_t d) { items[atomicAdd(&ctl->n_items, 1u)] = make_uint2(ci, d); });
}

// Close every circuit's batch (by the last CTA of a batch's cover).
__device__ void batch_close_all(CoverArgs *args, FwdArgs *fargs, uint32_t n, BatchCtl *ctl, uint32_t append) {
    unsigned int err = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t np = args[i].n_pairs;
        err |= args[i].acc->err;
        batch_close(args[i].acc, np);
        if (append) {
            args[i].pair_base += (uint32_t)np;
            fargs[i].pair_base += (uint32_t)np;
        }
    }
    err = __reduce_or_sync(0xFFFFFFFFu, err);
    if ((threadIdx.x & 31) == 0 && err) atomicOr(&ctl->err, err);
}

// The batch's cover in two passes of the same code.  TIER 0 lists at most
// `cap` nets per pair in a small table, so several CTAs share an SM (the
// per-pair phases are chains of dependent loads and barriers, which one CTA
// per SM leaves mostly idle); a pair that marks more nets is passed on
// (out_items, ctl->n_mid).  TIER 1 counts those with the large table (one
// CTA per SM) and queues what still does not fit for the spill cover
// (ctl->n_over).  The last CTA of the last pass that has work closes every
// circuit's batch.
template <int TIER>
__global__ void __launch_bounds__(kCoverThreads) k_batch_cover(CoverArgs *args, FwdArgs *fargs, uint32_t n,
                                                               const uint2 *in_items, uint2 *out_items, BatchCtl *ctl,
                                                               uint32_t append, uint32_t cap) {
    __shared__ CoverArgs s_a;
    __shared__ uint32_t s_last;
    const uint32_t n_items = TIER == 0 ? ctl->n_items : ctl->n_mid;
    if (TIER == 1 && !n_items) return;  // the small-table pass closed the batch
    for (uint32_t ai = blockIdx.x; ai < n_items; ai += gridDim.x) {
        const uint2 it = in_items[ai];
        if (threadIdx.x == 0) s_a = args[it.x];
        __syncthreads();
        const bool over = TIER == 0 ? cover_pair<kCoverCandSmall>(s_a, it.y, s_a.c.level_off, cap)
                                    : cover_pair<kCoverCand>(s_a, it.y, s_a.c.level_off, cap);  // end with a barrier
        if (over && threadIdx.x == 0) {
            if (TIER == 0) out_items[atomicAdd(&ctl->n_mid, 1u)] = it;             // for the large table
            else if (s_a.spill_slots) out_items[atomicAdd(&ctl->n_over, 1u)] = it;  // for k_batch_cover_spill
            else atomicOr(&s_a.acc->err, kErrHashFull);
        }
        __syncthreads();
    }
    // the last CTA to finish closes every circuit's batch, unless items wait
    // for the next pass
    unsigned int *done = TIER == 0 ? &ctl->done : &ctl->done_mid;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (!(TIER == 0 ? ctl->n_mid : ctl->n_over)) batch_close_all(args, fargs, n, ctl, append);
    if (threadIdx.x == 0) *done = 0;
}

// After k_batch_cover: the items it queued (CTA k uses spill slot k of the
// item's circuit; every spilling circuit has at least gridDim slots).
__global__ void __launch_bounds__(kCoverThreads) k_batch_cover_spill(CoverArgs *args, FwdArgs *fargs, uint32_t n,
                                                                     const uint2 *over_items, BatchCtl *ctl,
                                                                     uint32_t append) {
    __shared__ CoverArgs s_a;
    __shared__ uint32_t s_last;
    const uint32_t n_over = ctl->n_over;
    if (!n_over) return;  // k_batch_cover closed the batch
    for (uint32_t j = blockIdx.x; j < n_over; j += gridDim.x) {
        const uint2 it = over_items[j];
        if (threadIdx.x == 0) s_a = args[it.x];
        __syncthreads();
        spill_pair(s_a, it.y, spill_slot(s_a, blockIdx.x));  // ends with a barrier
    }
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&ctl->done_over, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    batch_close_all(args, fargs, n, ctl, append);
    if (threadIdx.x == 0) {
        ctl->n_over = 0;
        ctl->done_over = 0;
    }
}

// Dense first-detect merge over given planes (stage call pdf_merge): one warp
// per (gate, 32-word chunk), warp minimum, one atomicMin per warp.
__global__ void k_merge_dense(const DevCircuit c, const uint32_t *V, const uint32_t *M, uint64_t ld,
                              uint64_t n_pairs, uint32_t W, uint32_t pair_base, uint32_t *first_x,
                              uint32_t *first_y) {
    const uint32_t chunks = (W + 31) / 32;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= (uint64_t)c.n_gates * chunks) return;
    const uint32_t g = (uint32_t)(warp / chunks), w = (uint32_t)(warp % chunks) * 32 + lane;
    uint32_t cx = kEmpty, cy = kEmpty;
    if (w < W) {
        uint32_t m = M[(size_t)g * ld + w];
        if (w == W - 1 && (n_pairs & 31)) m &= (1u << (n_pairs & 31)) - 1u;
        if (m) {
            const uint32_t v = V[(size_t)g * ld + w];
            const uint32_t x = m & ~v, y = m & v;
            if (x) cx = w * 32 + (__ffs(x) - 1);
            if (y) cy = w * 32 + (__ffs(y) - 1);
        }
    }
    cx = __reduce_min_sync(0xFFFFFFFFu, cx);
    cy = __reduce_min_sync(0xFFFFFFFFu, cy);
    if (lane == 0) {
        if (cx != kEmpty) atomicMin(first_x + g, pair_base + cx);
        if (cy != kEmpty) atomicMin(first_y + g, pair_base + cy);
    }
}

// Column-block bitmaps of nets with a nonzero mark, from a mark plane (stage
// call pdf_cover).
__global__ void k_bitmap_from_marks(const DevCircuit c, const uint32_t *M, uint64_t ld,
                                    uint64_t n_pairs, uint32_t W, uint32_t bw, uint32_t n_blocks,
                                    uint32_t *nzb, uint32_t *blk_maxlvl, uint32_t bm_words) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_blocks) blk_maxlvl[t] = c.n_levels;
    if (t >= (uint64_t)c.n_gates * n_blocks) return;
    const uint32_t g = (uint32_t)(t % c.n_gates), blk = (uint32_t)(t / c.n_gates);
    uint32_t any = 0;
    for (uint32_t j = 0; j < bw; j++) {
        const uint32_t w = blk * bw + j;
        if (w >= W) break;
        uint32_t m = M[(size_t)g * ld + w];
        if (w == W - 1 && (n_pairs & 31)) m &= (1u << (n_pairs & 31)) - 1u;
        any |= m;
    }
    if (any) atomicOr(nzb + (size_t)blk * bm_words + (g >> 5), 1u << (g & 31));
}

__global__ void k_batch_begin(DevAcc *acc) {
    acc->batch_lo = 0;
    acc->batch_hi = 0;
    acc->batch_flags = 0;
    acc->done = 0;
    acc->n_over = 0;
    acc->done_over = 0;
}

template <int BW, int SEM, int MODE>
cudaError_t launch_fwd_t(const FwdArgs &a, uint32_t threads, size_t smem, cudaStream_t st) {
    auto kern = k_forward<BW, SEM, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = (a.W + BW - 1) / BW;
    if (blocks == 0 || a.n_pieces == 0) return cudaErrorInvalidValue;
    kern<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int SEM, int MODE, int LW>
cudaError_t launch_lanes_t(const FwdArgs &a, uint32_t threads, size_t smem, cudaStream_t st) {
    auto kern = k_forward_lanes<SEM, MODE, LW>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = (a.W + 32 * LW - 1) / (32 * LW);
    if (blocks == 0 || threads % 32 || threads > lane_threads(32 * LW)) return cudaErrorInvalidValue;
    kern<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int SEM, int LW>
cudaError_t launch_lanes_sem(const FwdArgs &a, int mode, uint32_t threads, size_t smem, cudaStream_t st) {
    switch (mode) {
        case FWD_FUSED: return launch_lanes_t<SEM, FWD_FUSED, LW>(a, threads, smem, st);
        case FWD_SIM: return launch_lanes_t<SEM, FWD_SIM, LW>(a, threads, smem, st);
        default: return launch_lanes_t<SEM, FWD_MARK, LW>(a, threads, smem, st);
    }
}

template <int LW>
cudaError_t launch_lanes(const FwdArgs &a, int mode, int sem, uint32_t threads, size_t smem, cudaStream_t st) {
    switch (sem) {
        case 0: return launch_lanes_sem<0, LW>(a, mode, threads, smem, st);
        case 1: return launch_lanes_sem<1, LW>(a, mode, threads, smem, st);
        case 2: return launch_lanes_sem<2, LW>(a, mode, threads, smem, st);
        case 3: return launch_lanes_sem<3, LW>(a, mode, threads, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int BW, int SEM>
cudaError_t launch_fwd_sem(const FwdArgs &a, int mode, uint32_t threads, size_t smem, cudaStream_t st) {
    switch (mode) {
        case FWD_FUSED: return launch_fwd_t<BW, SEM, FWD_FUSED>(a, threads, smem, st);
        case FWD_SIM: return launch_fwd_t<BW, SEM, FWD_SIM>(a, threads, smem, st);
        default: return launch_fwd_t<BW, SEM, FWD_MARK>(a, threads, smem, st);
    }
}

template <int BW>
cudaError_t launch_fwd_bw(const FwdArgs &a, int mode, int sem, uint32_t threads, size_t smem, cudaStream_t st) {
    switch (sem) {
        case 0: return launch_fwd_sem<BW, 0>(a, mode, threads, smem, st);
        case 1: return launch_fwd_sem<BW, 1>(a, mode, threads, smem, st);
        case 2: return launch_fwd_sem<BW, 2>(a, mode, threads, smem, st);
        case 3: return launch_fwd_sem<BW, 3>(a, mode, threads, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace


namespace {
template <int BW, int SEM>
int regs_t() {
    cudaFuncAttributes fa{}, fb{};
    if (cudaFuncGetAttributes(&fa, k_forward<BW, SEM, FWD_FUSED>) != cudaSuccess ||
        cudaFuncGetAttributes(&fb, k_batch_forward<BW, SEM>) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1;
    }
    return std::max(fa.numRegs, fb.numRegs);
}
template <int BW>
int regs_bw(int sem) {
    switch (sem) {
        case 0: return regs_t<BW, 0>();
        case 1: return regs_t<BW, 1>();
        case 2: return regs_t<BW, 2>();
        case 3: return regs_t<BW, 3>();
        default: return -1;
    }
}
template <int SEM, int LW>
int regs_lanes_t() {
    cudaFuncAttributes fa{}, fb{};
    if (cudaFuncGetAttributes(&fa, k_forward_lanes<SEM, FWD_FUSED, LW>) != cudaSuccess ||
        cudaFuncGetAttributes(&fb, k_batch_forward_lanes<SEM, LW>) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1;
    }
    return std::max(fa.numRegs, fb.numRegs);
}
template <int LW>
int regs_lanes(int sem) {
    switch (sem) {
        case 0: return regs_lanes_t<0, LW>();
        case 1: return regs_lanes_t<1, LW>();
        case 2: return regs_lanes_t<2, LW>();
        case 3: return regs_lanes_t<3, LW>();
        default: return -1;
    }
}
}  // namespace

int forward_kernel_regs(int bw, int sem) {
    switch (bw) {
        case 1: return regs_bw<1>(sem);
        case 2: return regs_bw<2>(sem);
        case 4: return regs_bw<4>(sem);
        case 8: return regs_bw<8>(sem);
        case kLaneWords: return regs_lanes<1>(sem);
        case kLaneWords2: return regs_lanes<2>(sem);
        case kLaneWords4: return regs_lanes<4>(sem);
        default: return -1;
    }
}

cudaError_t launch_forward(const FwdArgs &a, int mode, int sem, uint32_t bw, uint32_t threads,
                           size_t smem, cudaStream_t st) {
    switch (bw) {
        case kLaneWords: return launch_lanes<1>(a, mode, sem, threads, smem, st);
        case kLaneWords2: return launch_lanes<2>(a, mode, sem, threads, smem, st);
        case kLaneWords4: return launch_lanes<4>(a, mode, sem, threads, smem, st);
        case 1: return launch_fwd_bw<1>(a, mode, sem, threads, smem, st);
        case 2: return launch_fwd_bw<2>(a, mode, sem, threads, smem, st);
        case 4: return launch_fwd_bw<4>(a, mode, sem, threads, smem, st);
        case 8: return launch_fwd_bw<8>(a, mode, sem, threads, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

size_t cover_smem_bytes(uint32_t net_cap) { return cover_smem_lvt(net_cap) + (size_t)kCoverLevels * 4; }
size_t cover_small_smem_bytes(uint32_t cap) { return cover_smem_tables(cap, kCoverCandSmall); }

// CTAs per SM of the batch's small-table cover, and the nets per pair its
// table then holds: an equal share of the SM's shared memory less what the
// system keeps per CTA and the kernel's static variables.  Four CTAs of 256
// threads: the kernel's registers allow five.
uint32_t cover_small_cap(int device, uint32_t *ctas_per_sm) {
    constexpr uint32_t kCtas = 4;
    int per_sm = 0, reserved = 0, optin = 0;
    cudaFuncAttributes fa{};
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, k_batch_cover<0>) != cudaSuccess)
        return 0;
    const int64_t share = std::min<int64_t>(optin, per_sm / kCtas - reserved - (int64_t)fa.sharedSizeBytes);
    const int64_t room = share - (int64_t)kCoverCandSmall * 4;
    const uint32_t per_net = (uint32_t)cover_smem_tables(1, 0);
    if (room < (int64_t)per_net * 32) return 0;
    if (ctas_per_sm) *ctas_per_sm = kCtas;
    return (uint32_t)(room / per_net) & ~31u;
}

cudaError_t launch_cover(const CoverArgs &a, uint32_t grid, uint32_t threads, bool zero_active, cudaStream_t st) {
    const uint32_t W = (uint32_t)((a.n_pairs + 31) / 32);
    if (zero_active) {
        cudaError_t e = cudaMemsetAsync(a.active, 0, (size_t)(W + 1) * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
    }
    if (a.seg.N > 1) {
        cudaError_t e = cudaMemsetAsync(a.seg_first, 0xFF, (a.seg_first_mask + 1) * sizeof(unsigned long long), st);
        if (e != cudaSuccess) return e;
        const uint32_t blocks = (uint32_t)std::min<uint64_t>(((uint64_t)a.seg.S + 255) / 256, 148u * 16u);
        k_seg_first<<<std::max(1u, blocks), 256, 0, st>>>(a);
    } else {
        k_active<<<(a.c.n_gates + 255) / 256, 256, 0, st>>>(a);
    }
    if (threads != kCoverThreads) return cudaErrorInvalidValue;
    const size_t smem = cover_smem_bytes(a.hash_cap);
    cudaError_t e = cudaFuncSetAttribute(k_cover, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_cover<<<grid, threads, smem, st>>>(a);
    if (a.spill_slots) {
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_cover_spill<<<a.spill_slots, kCoverThreads, 0, st>>>(a);
    }
    return cudaGetLastError();
}

namespace {
// The dynamic shared-memory limit of a batch kernel on the current device,
// raised only when a batch asks for more than any earlier one did: a
// serving loop rebinds its batch every step, and only these calls set the
// batch kernels' limits, so the limit never falls below a request.
cudaError_t raise_smem_limit(const void *fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> have;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t &h = have[{dev, fn}];
    if (smem <= h) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) h = smem;
    return e;
}
template <typename F>
cudaError_t raise_smem(F *fn, size_t smem) {
    return raise_smem_limit(reinterpret_cast<const void *>(fn), smem);
}

// Kernel attributes and launch of one forward class (tile width, semantics).
template <int SEM>
cudaError_t prepare_class_sem(uint32_t bw, size_t smem) {
    switch (bw) {
        case 1: return raise_smem(k_batch_forward<1, SEM>, smem);
        case 2: return raise_smem(k_batch_forward<2, SEM>, smem);
        case 4: return raise_smem(k_batch_forward<4, SEM>, smem);
        case 8: return raise_smem(k_batch_forward<8, SEM>, smem);
        case kLaneWords: return raise_smem(k_batch_forward_lanes<SEM, 1>, smem);
        case kLaneWords2: return raise_smem(k_batch_forward_lanes<SEM, 2>, smem);
        case kLaneWords4: return raise_smem(k_batch_forward_lanes<SEM, 4>, smem);
        default: return cudaErrorInvalidValue;
    }
}
template <int SEM>
cudaError_t launch_class_sem(const BatchLaunch &b, const BatchClass &c, cudaStream_t s) {
    switch (c.bw) {
        case 1: k_batch_forward<1, SEM><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0); break;
        case 2: k_batch_forward<2, SEM><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0); break;
        case 4: k_batch_forward<4, SEM><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0); break;
        case 8: k_batch_forward<8, SEM><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0); break;
        case kLaneWords:
            k_batch_forward_lanes<SEM, 1><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0);
            break;
        case kLaneWords2:
            k_batch_forward_lanes<SEM, 2><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0);
            break;
        case kLaneWords4:
            k_batch_forward_lanes<SEM, 4><<<c.blocks, c.threads, c.smem, s>>>(b.fargs, b.bpref, b.n, b.ctl, c.blk0);
            break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
cudaError_t prepare_class(uint32_t sem, uint32_t bw, size_t smem) {
    switch (sem) {
        case 0: return prepare_class_sem<0>(bw, smem);
        case 1: return prepare_class_sem<1>(bw, smem);
        case 2: return prepare_class_sem<2>(bw, smem);
        case 3: return prepare_class_sem<3>(bw, smem);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t launch_class(const BatchLaunch &b, const BatchClass &c, cudaStream_t s) {
    switch (b.sem) {
        case 0: return launch_class_sem<0>(b, c, s);
        case 1: return launch_class_sem<1>(b, c, s);
        case 2: return launch_class_sem<2>(b, c, s);
        case 3: return launch_class_sem<3>(b, c, s);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace

cudaError_t prepare_batch(const BatchLaunch &b) {
    for (uint32_t k = 0; k < b.n_class; k++) {
        // every class of one tile width shares its kernel: the largest request wins
        size_t smem = 0;
        for (uint32_t j = 0; j < b.n_class; j++)
            if (b.cls[j].bw == b.cls[k].bw) smem = std::max(smem, b.cls[j].smem);
        const cudaError_t e = prepare_class(b.sem, b.cls[k].bw, smem);
        if (e != cudaSuccess) return e;
    }
    const cudaError_t e = raise_smem(k_batch_cover<0>, cover_small_smem_bytes(b.small_cap));
    if (e != cudaSuccess) return e;
    return raise_smem(k_batch_cover<1>, cover_smem_tables(b.hash_cap, kCoverCand));
}

// The classes' forward launches are independent (different circuits), so
// they run side by side: the first on `st`, the others on side streams that
// wait for `st` and that `st` waits for before the cover.  Run one after
// another, a class's last CTAs held the GPU alone (its longest level chain)
// before the next class could start.
cudaError_t launch_batch(const BatchLaunch &b, cudaStream_t st) {
    if (!b.n || !b.total_blocks) return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    const unsigned pflag = b.prof_external ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (b.prof[0] && (e = cudaEventRecordWithFlags(b.prof[0], st, pflag)) != cudaSuccess) return e;
    bool fork = false;  // recorded before the first class's launch, which it must not wait for
    for (uint32_t k = 1; k < b.n_class; k++) fork |= b.cls[k].blocks && b.side[k - 1];
    if (fork && (e = cudaEventRecord(b.fork, st)) != cudaSuccess) return e;
    for (uint32_t k = 0; k < b.n_class; k++) {
        const BatchClass &c = b.cls[k];
        if (!c.blocks) continue;
        cudaStream_t s = st;
        if (k > 0 && b.side[k - 1]) {
            s = b.side[k - 1];
            if ((e = cudaStreamWaitEvent(s, b.fork, 0)) != cudaSuccess) return e;
        }
        if ((e = launch_class(b, c, s)) != cudaSuccess) return e;
        if (s != st) {
            if ((e = cudaEventRecord(b.join[k - 1], s)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(st, b.join[k - 1], 0)) != cudaSuccess) return e;
        }
    }
    if (b.prof[1] && (e = cudaEventRecordWithFlags(b.prof[1], st, pflag)) != cudaSuccess) return e;
    k_batch_active<<<(b.total_gates + 255) / 256, 256, 0, st>>>(b.cargs, b.gpref, b.n, b.items, b.ctl);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_batch_cover<0><<<b.small_grid, kCoverThreads, cover_small_smem_bytes(b.small_cap), st>>>(
        b.cargs, b.fargs, b.n, b.items, b.mid_items, b.ctl, b.append, b.small_cap);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_batch_cover<1><<<b.cover_grid, kCoverThreads, cover_smem_tables(b.hash_cap, kCoverCand), st>>>(
        b.cargs, b.fargs, b.n, b.mid_items, b.over_items, b.ctl, b.append, b.hash_cap);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (b.spill_grid) {
        k_batch_cover_spill<<<b.spill_grid, kCoverThreads, 0, st>>>(b.cargs, b.fargs, b.n, b.over_items, b.ctl,
                                                                    b.append);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (b.prof[2] && (e = cudaEventRecordWithFlags(b.prof[2], st, pflag)) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t launch_seg_merge(const SegMergeArgs &a, uint32_t n_blocks, cudaStream_t st) {
    if (n_blocks == 0) return cudaSuccess;
    k_seg_merge<<<n_blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_seg_merge_dense(const SegArgs &seg, const uint32_t *V, const uint32_t *M, uint64_t ld,
                                   uint64_t n_pairs, uint32_t pair_base, uint32_t *first_x, uint32_t *first_y,
                                   cudaStream_t st) {
    const uint32_t W = (uint32_t)((n_pairs + 31) / 32);
    const uint64_t warps = (uint64_t)seg.S * ((W + 31) / 32);
    const uint64_t blocks = (warps * 32 + 255) / 256;
    if (blocks == 0) return cudaSuccess;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    k_seg_merge_dense<<<(unsigned)blocks, 256, 0, st>>>(seg, V, M, ld, n_pairs, W, pair_base, first_x, first_y);
    return cudaGetLastError();
}

cudaError_t launch_merge_dense(const DevCircuit &c, const uint32_t *V, const uint32_t *M, uint64_t ld,
                               uint64_t n_pairs, uint32_t pair_base, uint32_t *first_x,
                               uint32_t *first_y, cudaStream_t st) {
    const uint32_t W = (uint32_t)((n_pairs + 31) / 32);
    const uint64_t warps = (uint64_t)c.n_gates * ((W + 31) / 32);
    const uint64_t blocks = (warps * 32 + 255) / 256;
    if (blocks == 0) return cudaSuccess;
    k_merge_dense<<<(unsigned)blocks, 256, 0, st>>>(c, V, M, ld, n_pairs, W, pair_base, first_x, first_y);
    return cudaGetLastError();
}

cudaError_t launch_bitmap_from_marks(const DevCircuit &c, const uint32_t *M, uint64_t ld,
                                     uint64_t n_pairs, uint32_t bw, uint32_t *nzb,
                                     uint32_t *blk_maxlvl, uint32_t bm_words, cudaStream_t st) {
    const uint32_t W = (uint32_t)((n_pairs + 31) / 32);
    const uint32_t n_blocks = (W + bw - 1) / bw;
    cudaError_t e = cudaMemsetAsync(nzb, 0, (size_t)n_blocks * bm_words * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const uint64_t n = std::max<uint64_t>((uint64_t)c.n_gates * n_blocks, n_blocks);
    k_bitmap_from_marks<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c, M, ld, n_pairs, W, bw, n_blocks,
                                                                     nzb, blk_maxlvl, bm_words);
    return cudaGetLastError();
}

__global__ void k_copy_from_host(uint4 *dst, const uint4 *src, size_t n16) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

cudaError_t launch_copy_from_host(void *dst, const void *src_mapped, size_t n16, cudaStream_t st) {
    if (n16 == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<size_t>((n16 + 255) / 256, 64);
    k_copy_from_host<<<blocks, 256, 0, st>>>(static_cast<uint4 *>(dst), static_cast<const uint4 *>(src_mapped),
                                             n16);
    return cudaGetLastError();
}

cudaError_t launch_batch_begin(DevAcc *acc, cudaStream_t st) {
    k_batch_begin<<<1, 1, 0, st>>>(acc);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fixed scratch of pdf_cover_noalloc.
//
// Callers that may not enter the CUDA allocator (a host framework that owns
// every device byte through its own pool, or a latency-bound loop where a
// cudaMalloc could synchronise the device or fail under memory pressure) get
// a cover call whose scratch is this file-scope array instead of memory
// allocated per call.  Every GPU that loads the library holds it until the
// process exits.  All calls on a device share it, so calls that overlap on
// the GPU race.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_cover_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};
}  // namespace

// Device address of g_cover_scratch on `device`, which the caller has made
// current.  In host code the array's name is only a host-side stand-in, so
// its device address is looked up once per device and cached.
cudaError_t noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        unsigned char *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_cover_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}
