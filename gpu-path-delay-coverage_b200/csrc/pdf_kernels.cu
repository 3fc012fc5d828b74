// pdf_kernels.cu -- sm_100a kernels of the grading path.
//
// Layout: every per-(net, pair) quantity is a bit-plane, gate-major, ld words
// per gate row, 32 pairs per word.  A CTA owns one column block of BW words
// (32 * BW pairs) and walks every gate of the circuit in level order for it:
// the only dependency between pairs is the first-detect minimum, so column
// blocks never wait on one another and no grid-wide barrier is needed.
//
//   k_forward   sim + forward robust mark (levels ascending, one
//               __syncthreads per level), then, in the same CTA, the
//               prune + first-detect merge over the gates whose marks are
//               nonzero (levels descending).
//   k_active / k_active_compact / k_cover
//               path counting, only for pairs that first-detect some net
//               (every other pair credits nothing), over only the nets those
//               pairs mark, in exact 128-bit integers.
#include "pdf_kernels.cuh"

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

__device__ __forceinline__ uint32_t fanin_id(const GateRec &r, const uint32_t *edges, uint32_t j) {
    switch (j) {
        case 0: return r.w[3];
        case 1: return r.w[4];
        case 2: return r.w[5];
        case 3: return r.w[6];
        case 4: return r.w[7];
        default: return __ldg(edges + r.w[2] + j);
    }
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
// Every wait is bounded: on expiry the caller reports PDF_ETIMEOUT.
constexpr uint32_t kSpinLimit = 1u << 24;
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t phase) {
    for (uint32_t i = 0; i < kSpinLimit; i++)
        if (mbar_try_wait(m, phase)) return true;
    return false;
}

// Asynchronous global -> shared copies of BW words (cp.async, completed by
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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared-memory layout of k_forward (byte offsets from the host plan).
struct FwdSmem {
    uint32_t *ring;      // forward: [R][3][BW] (V, T, M); reverse: [R2][BW] pruned marks
    GateRec *rec;        // [3][cap] staged gate records of a piece
    uint32_t *edge;      // [2][ecap] staged edge slices (reverse pass; shares memory with far)
    uint32_t *far;       // [2][3][farcap][BW] prefetched far fan-in V, T, M (forward pass)
    uint16_t *slot;      // [2][cap][kPrefetchFanins] far-buffer slot of each fan-in (0xFFFF: none)
    uint32_t *bm;        // nonzero-mark bitmap (shared or global)
    uint32_t *pbits;     // pieces that hold a forward mark
    uint32_t *farcnt;    // [2] far slots handed out
    uint64_t *mbar;      // [3]
};

// Stage piece `p` into buffer `buf`: its gate records and, for the reverse
// pass, its edge slice.  Called by one thread.
__device__ __forceinline__ void stage_piece(const FwdArgs &a, const FwdSmem &S, const Piece &p, int buf,
                                            bool edges) {
    const uint32_t rb = (p.b - p.a) * (uint32_t)sizeof(GateRec);
    const bool e = edges && p.ea != 0xFFFFFFFFu;
    const uint32_t eb = e ? (p.eb - p.ea) * 4u : 0u;
    fence_proxy_async();
    mbar_expect_tx(S.mbar + buf, rb + eb);
    bulk_g2s(S.rec + (size_t)buf * a.cap, a.c.rec + p.a, rb, S.mbar + buf);
    if (e) bulk_g2s(S.edge + (size_t)buf * a.ecap, a.c.edges + p.ea, eb, S.mbar + buf);
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

// Rarely needed: OR over on-path candidates i of AND over side inputs x != i
// of the sensitisation test (markkernel.cuh:253-261 with robust()/
// nonrobust(), :43-72), restricted to the pairs in `need`.
template <int BW, int ROBUST, class Fetch>
__device__ __forceinline__ Vec<BW> sens_any(const GateRec &r, const uint32_t *edges, uint32_t nfi,
                                            const Vec<BW> &need, Fetch fetch) {
    const bool or_like = (r.w[0] & RF_IM) != 0;
    Vec<BW> acc;
#pragma unroll
    for (int j = 0; j < BW; j++) acc.x[j] = 0;
    for (uint32_t i = 0; i < nfi; i++) {
        uint32_t left = 0;
#pragma unroll
        for (int j = 0; j < BW; j++) left |= need.x[j] & ~acc.x[j];
        if (!left) break;
        Vec<BW> iv, it;
        fetch(fanin_id(r, edges, i), iv, it);
        Vec<BW> term;
#pragma unroll
        for (int j = 0; j < BW; j++) term.x[j] = 0xFFFFFFFFu;
        for (uint32_t x = 0; x < nfi; x++) {
            if (x == i) continue;
            Vec<BW> xv, xt;
            fetch(fanin_id(r, edges, x), xv, xt);
#pragma unroll
            for (int j = 0; j < BW; j++) term.x[j] &= sens_class<ROBUST>(or_like, iv.x[j], it.x[j], xv.x[j], xt.x[j]);
        }
#pragma unroll
        for (int j = 0; j < BW; j++) acc.x[j] |= term.x[j];
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Forward kernel: one CTA per column block of BW words (32 * BW pairs); one
// thread per gate, carrying all BW words of the block.
//
// Gates are walked in pieces (runs of one level, <= cap gates) whose records
// are staged into shared memory by a TMA bulk copy issued one piece ahead.
//
// Forward (sim + forward mark, simkernel.cuh:96-156, markkernel.cuh:215-270):
// a ring of the last R gates' V, T, M words sits in shared memory
// (slot = gate & (R - 1)).  During piece [a, b) a fan-in f is read from the
// ring iff f >= b - R and only gates g >= b - R write it; within that window
// no two gates share a slot, so a ring read always sees its own gate.  Older
// fan-ins come from the global planes (written by this CTA and ordered by
// __syncthreads).
//
// Reverse (prune, markkernel.cuh:271-293): only pieces that hold a forward
// mark, descending, only gates whose bitmap bit is set.  Pruned marks of
// recent gates sit in a second ring (the same memory, R2 slots of BW words):
// during piece [a, b) a fan-out fo is read from it iff fo < a + R2 and only
// gates g < a + R2 write it.
//
// Merge (mergekernel.cuh:116-198) needs no level order: one sweep over the
// surviving marks folds the first falling / rising pair of every net into
// first_x / first_y with atomicMin.
//
// Plane rows are read and written BW words at a time: ld and pi_ld are
// multiples of BW and every row holds all n_blocks * BW words; words at or
// past ceil(n_pairs / 32) are masked to zero.
// ---------------------------------------------------------------------------
constexpr int kPrefetchFanins = 4;  // fan-ins per gate eligible for the far-buffer prefetch

template <int BW, int ROBUST, int MODE>
__global__ void __launch_bounds__(BW >= 8 ? 512 : 1024) k_forward(const FwdArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    FwdSmem S;
    S.ring = reinterpret_cast<uint32_t *>(smraw + a.off_ring);
    S.rec = reinterpret_cast<GateRec *>(smraw + a.off_rec);
    S.edge = reinterpret_cast<uint32_t *>(smraw + a.off_edge);
    S.far = reinterpret_cast<uint32_t *>(smraw + a.off_edge);
    S.slot = reinterpret_cast<uint16_t *>(smraw + a.off_slot);
    S.pbits = reinterpret_cast<uint32_t *>(smraw + a.off_pbits);
    S.farcnt = reinterpret_cast<uint32_t *>(smraw + a.off_mbar + 64);
    S.mbar = reinterpret_cast<uint64_t *>(smraw + a.off_mbar);
    const uint32_t blk = blockIdx.x;
    const uint32_t w0 = blk * BW;
    S.bm = a.bm_shared ? reinterpret_cast<uint32_t *>(smraw + a.off_bm) : a.nzb + (size_t)blk * a.bm_words;
    uint32_t *gbm = a.nzb ? a.nzb + (size_t)blk * a.bm_words : nullptr;
    const uint32_t *edges = a.c.edges;
    const uint32_t R = a.ring_gates, Rm = R - 1;
    uint32_t *rV = S.ring, *rT = S.ring + (size_t)R * BW, *rM = S.ring + 2 * (size_t)R * BW;
    const uint32_t farcap = a.farcap;
    Vec<BW> wm;  // valid bits of each word of this block
#pragma unroll
    for (int j = 0; j < BW; j++) {
        const uint32_t w = w0 + j;
        wm.x[j] = w + 1 < a.W ? 0xFFFFFFFFu
                              : (w + 1 == a.W ? ((a.n_pairs & 31) ? (1u << (a.n_pairs & 31)) - 1u : 0xFFFFFFFFu) : 0u);
    }
    // far buffer of parity p, plane k (0 V, 1 T, 2 M), slot s
    auto farp = [&](uint32_t p, uint32_t k, uint32_t sl) -> uint32_t * {
        return S.far + (((size_t)p * 3 + k) * farcap + sl) * BW;
    };

    if (MODE != FWD_SIM)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) S.bm[q] = 0;
    for (uint32_t q = threadIdx.x; q < (a.n_pieces + 31) / 32; q += blockDim.x) S.pbits[q] = 0;
    if (threadIdx.x == 0) {
        mbar_init(S.mbar, 1);
        mbar_init(S.mbar + 1, 1);
        mbar_init(S.mbar + 2, 1);
        fence_mbar_init();
        S.farcnt[0] = S.farcnt[1] = 0;
    }
    __syncthreads();

    uint32_t phase = 0;     // bit b: parity of the next wait on mbar[b]
    uint32_t inflight = 0;  // bit b: a copy on mbar[b] not yet waited for (uniform)
    bool failed = false;

    // Prefetch the fan-ins of piece P (records in `recs`) that lie outside
    // its ring window into far buffer `fb`: issued one piece ahead, so the
    // piece then reads them from shared memory.  Only gates below
    // `final_below` (the start of the piece now running) are copied: they
    // are already written.
    auto prefetch = [&](const Piece &P, const GateRec *recs, uint32_t fb, uint32_t final_below) {
        if (!farcap) return;
        const uint32_t lo = R ? (P.b > R ? P.b - R : 0) : P.b;
        for (uint32_t gi = threadIdx.x; gi < P.b - P.a; gi += blockDim.x) {
            const GateRec &r = recs[gi];
            const uint32_t h = r.w[0];
            if (h & RF_INPT) continue;
            const uint32_t nfold = hdr_nfold(h);
#pragma unroll
            for (int q = 0; q < kPrefetchFanins; q++) {
                if ((uint32_t)q > nfold) break;
                const uint32_t f = r.w[3 + q];
                if (f >= lo) continue;
                // only gates already written are copied; the rest are read
                // from the planes when the piece runs
                uint32_t sl = f < final_below ? atomicAdd(S.farcnt + fb, 1u) : 0xFFFFu;
                if (sl < farcap) {
                    cp_async_vec<BW>(farp(fb, 0, sl), a.V + (size_t)f * a.ld + w0);
                    cp_async_vec<BW>(farp(fb, 1, sl), a.T + (size_t)f * a.ld + w0);
                    if (MODE != FWD_SIM && q == 0 && (h & RF_MARKF0))
                        cp_async_vec<BW>(farp(fb, 2, sl), a.M + (size_t)f * a.ld + w0);
                } else {
                    sl = 0xFFFFu;
                }
                S.slot[((size_t)fb * a.cap + gi) * kPrefetchFanins + q] = (uint16_t)sl;
            }
        }
        cp_async_commit();
    };

    // ------------------------------------------------------------- forward
    // Records are staged two pieces ahead (three buffers, mbar[i % 3]); far
    // fan-ins one piece ahead (two buffers).
    Piece P0 = a.pieces[0], P1 = a.n_pieces > 1 ? a.pieces[1] : P0, P2 = P1;
    if (threadIdx.x == 0) {
        stage_piece(a, S, P0, 0, false);
        if (a.n_pieces > 1) stage_piece(a, S, P1, 1, false);
    }
    inflight = a.n_pieces > 1 ? 3u : 1u;
    {
        const bool ok = mbar_wait(S.mbar, 0);
        phase ^= 1u;
        inflight &= ~1u;
        if (__syncthreads_or(!ok)) failed = true;
    }
    if (!failed) prefetch(P0, S.rec, 0, P0.a);
    for (uint32_t i = 0; i < a.n_pieces && !failed; i++) {
        const Piece P = P0;
        const uint32_t rb = i % 3, fb = i & 1;
        const bool has_next = i + 1 < a.n_pieces;
        if (i + 2 < a.n_pieces) P2 = a.pieces[i + 2];
        if (threadIdx.x == 0) S.farcnt[fb ^ 1] = 0;
        bool ok = true;
        if (has_next) {
            const uint32_t nb = (i + 1) % 3;
            ok = mbar_wait(S.mbar + nb, (phase >> nb) & 1u);
            phase ^= 1u << nb;
            inflight &= ~(1u << nb);
        }
        cp_async_wait_all();  // this thread's prefetch for piece i
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (i + 2 < a.n_pieces) {
            if (threadIdx.x == 0) stage_piece(a, S, P2, (i + 2) % 3, false);
            inflight |= 1u << ((i + 2) % 3);
        }
        if (has_next) prefetch(P1, S.rec + (size_t)((i + 1) % 3) * a.cap, fb ^ 1, P.a);

        const GateRec *recs = S.rec + (size_t)rb * a.cap;
        const uint16_t *slots = S.slot + (size_t)fb * a.cap * kPrefetchFanins;
        const uint32_t ring_lo = R ? (P.b > R ? P.b - R : 0) : P.b;
        bool any = false;
        for (uint32_t gi = threadIdx.x; gi < P.b - P.a; gi += blockDim.x) {
            const uint32_t g = P.a + gi;
            auto fetch = [&](uint32_t f, Vec<BW> &fv, Vec<BW> &ft) {
                if (f >= ring_lo) {
                    fv = vld<BW>(rV + (f & Rm) * BW);
                    ft = vld<BW>(rT + (f & Rm) * BW);
                } else {
                    fv = vld<BW>(a.V + (size_t)f * a.ld + w0);
                    ft = vld<BW>(a.T + (size_t)f * a.ld + w0);
                }
            };
            const GateRec r = recs[gi];
            const uint32_t h = r.w[0];
            Vec<BW> V, T, M;
            if (MODE == FWD_MARK) {
                V = vld<BW>(a.V + (size_t)g * a.ld + w0);
                T = vld<BW>(a.T + (size_t)g * a.ld + w0);
#pragma unroll
                for (int j = 0; j < BW; j++) {
                    V.x[j] &= wm.x[j];
                    T.x[j] &= wm.x[j];
                }
            } else if (h & RF_INPT) {  // simkernel.cuh:112-125, pairs already formed
                V = vldg<BW>(a.pi_v + (size_t)g * a.pi_ld + w0);
                T = vldg<BW>(a.pi_t + (size_t)g * a.pi_ld + w0);
#pragma unroll
                for (int j = 0; j < BW; j++) {
                    V.x[j] &= wm.x[j];
                    T.x[j] &= wm.x[j];
                }
            }
            Vec<BW> m0;
#pragma unroll
            for (int j = 0; j < BW; j++) m0.x[j] = 0;
            if (!(h & RF_INPT)) {
                // Fan-in q < kPrefetchFanins comes from the ring, the far
                // buffer prefetched one piece ahead, or (far-buffer overflow)
                // the planes; later fan-ins from the ring or the planes.
                auto src = [&](uint32_t q, uint32_t f, uint32_t k) -> const uint32_t * {
                    const uint32_t *ring_k = k == 0 ? rV : (k == 1 ? rT : rM);
                    if (f >= ring_lo) return ring_k + (f & Rm) * BW;
                    // the slot table is written only while the prefetch is on
                    const uint32_t sl =
                        (farcap && q < (uint32_t)kPrefetchFanins) ? slots[gi * kPrefetchFanins + q] : 0xFFFFu;
                    if (sl != 0xFFFFu) return farp(fb, k, sl);
                    const uint32_t *plane = k == 0 ? a.V : (k == 1 ? a.T : a.M);
                    return plane + (size_t)f * a.ld + w0;
                };
                const uint32_t nfold = hdr_nfold(h);
                const uint32_t f0 = r.w[3];
                if (MODE != FWD_SIM && (h & RF_MARKF0)) m0 = vld<BW>(src(0, f0, 2));
                if (MODE != FWD_MARK) {
                    Vec<BW> v1;
                    {
                        const Vec<BW> fv = vld<BW>(src(0, f0, 0)), ft = vld<BW>(src(0, f0, 1));
#pragma unroll
                        for (int j = 0; j < BW; j++) eval_first(h, fv.x[j], ft.x[j], V.x[j], v1.x[j]);
                    }
                    for (uint32_t q = 1; q <= nfold; q++) {
                        const uint32_t f = fanin_id(r, edges, q);
                        const Vec<BW> fv = vld<BW>(src(q, f, 0)), ft = vld<BW>(src(q, f, 1));
#pragma unroll
                        for (int j = 0; j < BW; j++) eval_fold(h, V.x[j], v1.x[j], fv.x[j], ft.x[j]);
                    }
#pragma unroll
                    for (int j = 0; j < BW; j++) {
                        eval_finish(h, V.x[j], v1.x[j], T.x[j]);
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
                } else if (h & RF_MARKF0) {
#pragma unroll
                    for (int j = 0; j < BW; j++) M.x[j] = T.x[j] & m0.x[j];
                    if ((h & RF_SENS) && vany(M)) {
                        const Vec<BW> sv = sens_any<BW, ROBUST>(r, edges, rec_nfi(r), M, fetch);
#pragma unroll
                        for (int j = 0; j < BW; j++) M.x[j] &= sv.x[j];
                    }
                }
            }
            const size_t o = (size_t)g * a.ld + w0;
            if (MODE != FWD_MARK) {
                vst<BW>(a.V + o, V);
                vst<BW>(a.T + o, T);
            }
            if (MODE != FWD_SIM) vst<BW>(a.M + o, M);
            if (g >= ring_lo) {
                const uint32_t slot = (g & Rm) * BW;
                vst<BW>(rV + slot, V);
                vst<BW>(rT + slot, T);
                vst<BW>(rM + slot, M);
            }
            if (MODE != FWD_SIM && vany(M)) {
                bitmap_set_aggregated(S.bm, g);
                any = true;
            }
        }
        if (__syncthreads_or(any) && threadIdx.x == 0) S.pbits[i >> 5] |= 1u << (i & 31);
        P0 = P1;
        P1 = P2;
    }
    if (failed) {
        // wait (bounded) for the record copies still in flight, then report
        for (uint32_t b = 0; b < 3; b++)
            if ((inflight >> b) & 1u) (void)mbar_wait(S.mbar + b, (phase >> b) & 1u);
        cp_async_wait_all();
    }
    if (failed) {
        if (threadIdx.x == 0) atomicOr(a.err, kErrTimeout);
        return;
    }
    if (MODE == FWD_SIM) return;
    __syncthreads();

    // ------------------------------------------------------------- reverse
    const uint32_t R2 = a.ring2_gates, R2m = R2 - 1;
    uint32_t *ring2 = S.ring;
    auto prev_marked = [&](int from) -> int {  // highest marked piece index < from
        for (int q = (from - 1) >> 5; q >= 0 && from > 0; q--) {
            uint32_t bits = S.pbits[q];
            if (q == (from - 1) >> 5) bits &= (from & 31) ? ((1u << (from & 31)) - 1u) : 0xFFFFFFFFu;
            if (bits) return q * 32 + 31 - __clz(bits);
        }
        return -1;
    };
    int cur = prev_marked((int)a.n_pieces);
    uint32_t maxlvl = 0;
    int sbuf = 0;
    if (cur >= 0 && threadIdx.x == 0) stage_piece(a, S, a.pieces[cur], 0, true);
    while (cur >= 0) {
        const int nxt = prev_marked(cur);
        const Piece P = a.pieces[cur];
        if (threadIdx.x == 0 && nxt >= 0) stage_piece(a, S, a.pieces[nxt], sbuf ^ 1, true);
        const bool ok = mbar_wait(S.mbar + sbuf, (phase >> sbuf) & 1u);
        phase ^= 1u << sbuf;
        if (__syncthreads_or(!ok)) {
            failed = true;
            if (nxt >= 0) (void)mbar_wait(S.mbar + (sbuf ^ 1), (phase >> (sbuf ^ 1)) & 1u);
            break;
        }
        const GateRec *recs = S.rec + (size_t)sbuf * a.cap;
        const uint32_t *es = S.edge + (size_t)sbuf * a.ecap;
        const bool staged = P.ea != 0xFFFFFFFFu;
        const uint32_t win = P.a + R2;  // fan-outs below this are in ring2
        bool any = false;
        for (uint32_t gi = threadIdx.x; gi < P.b - P.a; gi += blockDim.x) {
            const uint32_t g = P.a + gi;
            if (!bit_test(S.bm, g)) continue;
            const GateRec &r = recs[gi];
            const Vec<BW> mk = vld<BW>(a.M + (size_t)g * a.ld + w0);
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
            if (!nz) atomicAnd(S.bm + (g >> 5), ~(1u << (g & 31)));
            any |= nz;
        }
        if (__syncthreads_or(any) && P.level + 1 > maxlvl) maxlvl = P.level + 1;
        cur = nxt;
        sbuf ^= 1;
    }
    if (failed) {
        if (threadIdx.x == 0) atomicOr(a.err, kErrTimeout);
        return;
    }

    // ------------------------------------------------------------- merge
    const uint32_t gend = a.c.level_off[maxlvl];
    if (MODE == FWD_FUSED) {
        for (uint32_t g = threadIdx.x; g < gend; g += blockDim.x) {
            if (!bit_test(S.bm, g)) continue;
            const Vec<BW> m = vld<BW>(a.M + (size_t)g * a.ld + w0);
            const Vec<BW> v = vld<BW>(a.V + (size_t)g * a.ld + w0);
            uint32_t cx = kEmpty, cy = kEmpty;
#pragma unroll
            for (int j = BW - 1; j >= 0; j--) {  // lowest word wins
                const uint32_t x = m.x[j] & ~v.x[j], y = m.x[j] & v.x[j];
                if (x) cx = (w0 + j) * 32 + (__ffs(x) - 1);
                if (y) cy = (w0 + j) * 32 + (__ffs(y) - 1);
            }
            if (cx != kEmpty) atomicMin(a.first_x + g, a.pair_base + cx);
            if (cy != kEmpty) atomicMin(a.first_y + g, a.pair_base + cy);
        }
    }
    // publish the bitmap of surviving marks for the cover kernels
    if (a.bm_shared && gbm)
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) gbm[q] = S.bm[q];
    if (threadIdx.x == 0) a.blk_maxlvl[blk] = maxlvl;
}

// ---------------------------------------------------------------------------
// Cover.
// ---------------------------------------------------------------------------

// Pairs that first-detect some net in this batch.
__global__ void k_active(const CoverArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.c.n_gates) return;
    const uint32_t fx = a.first_x[g], fy = a.first_y[g];
    const uint32_t dx = fx - a.pair_base, dy = fy - a.pair_base;
    if (fx != kEmpty && dx < a.n_pairs) atomicOr(a.active + (dx >> 5), 1u << (dx & 31));
    if (fy != kEmpty && dy < a.n_pairs) atomicOr(a.active + (dy >> 5), 1u << (dy & 31));
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t g, uint32_t mask) {
    return (g * 2654435761u) & mask;
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

// Path counting (kernCover, coverkernel.cuh:171-230, and kernSumSingle,
// :77-105) for the pairs of one column block that first-detect some net.
// One CTA per column block; up to kCoverSlots such pairs per pass.  Levels
// descending from the block's highest marked level, over the nets with a
// surviving mark in the block that one of the pass's pairs marks:
//   H = [po] + sum h(fo);  C = sum c(fo);  first = pid is first_x or first_y
//   c = C + (first ? H : 0);  h = first ? 0 : H;  h = 0 on INPT
// (a net a pair does not mark has h = c = 0).  (h, c) of each net, one per
// slot, sit in a shared-memory open-addressing table keyed by net id.  The
// level-0 INPT c values are the pairs' counts, summed into the batch count.
constexpr int kCoverSlots = 4;
__global__ void __launch_bounds__(256) k_cover(const CoverArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const uint32_t cap = a.hash_cap, cmask = cap - 1;
    uint32_t *keys = reinterpret_cast<uint32_t *>(smraw);
    pdf_u128 *hv = reinterpret_cast<pdf_u128 *>(smraw + (((size_t)cap * 4 + 127) & ~(size_t)127));
    pdf_u128 *cv = hv + (size_t)cap * kCoverSlots;
    __shared__ uint32_t s_pairs[256];
    __shared__ uint32_t s_na;
    __shared__ pdf_u128 s_red[8];
    __shared__ unsigned int s_flags;

    const uint32_t blk = blockIdx.x, w0 = blk * a.bw;
    const uint32_t W = (uint32_t)((a.n_pairs + 31) / 32);
    if (threadIdx.x == 0) {
        uint32_t n = 0;
        for (uint32_t j = 0; j < a.bw && w0 + j < W; j++) {
            uint32_t bits = a.active[w0 + j];
            while (bits) {
                s_pairs[n++] = (w0 + j) * 32 + (__ffs(bits) - 1);
                bits &= bits - 1;
            }
        }
        s_na = n;
        s_flags = 0;
    }
    __syncthreads();
    const uint32_t na = s_na;
    if (na == 0) return;
    const uint32_t top = a.blk_maxlvl[blk];
    const uint32_t *nzb = a.nzb + (size_t)blk * a.bm_words;
    pdf_u128 total = 0;
    bool ovf = false;
    for (uint32_t g0 = 0; g0 < na; g0 += kCoverSlots) {
        const uint32_t ns = min((uint32_t)kCoverSlots, na - g0);
        uint32_t pw[kCoverSlots], pb[kCoverSlots], pid[kCoverSlots];
#pragma unroll
        for (int k = 0; k < kCoverSlots; k++) {
            const uint32_t p = s_pairs[g0 + min((uint32_t)k, ns - 1)];
            pw[k] = p >> 5;
            pb[k] = p & 31;
            pid[k] = a.pair_base + p;
        }
        for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) keys[i] = kEmpty;
        __syncthreads();
        for (int l = (int)top - 1; l >= 0; l--) {
            const uint32_t s = a.c.level_off[l], e = a.c.level_off[l + 1];
            for (uint32_t g = s + threadIdx.x; g < e; g += blockDim.x) {
                if (!((nzb[g >> 5] >> (g & 31)) & 1u)) continue;
                uint32_t smask = 0;
#pragma unroll
                for (int k = 0; k < kCoverSlots; k++)
                    if ((uint32_t)k < ns && ((a.M[(size_t)g * a.ld + pw[k]] >> pb[k]) & 1u)) smask |= 1u << k;
                if (!smask) continue;
                const GateRec r = load_rec(a.c.rec + g);
                const uint32_t fx = a.first_x[g], fy = a.first_y[g];
                pdf_u128 H[kCoverSlots], Cc[kCoverSlots];
#pragma unroll
                for (int k = 0; k < kCoverSlots; k++) {
                    H[k] = rec_po(r) ? 1 : 0;
                    Cc[k] = 0;
                }
                const uint32_t nfo = r.w[1], eb = r.w[2] + rec_nfi(r);
                for (uint32_t q = 0; q < nfo; q++) {
                    const uint32_t fo = __ldg(a.c.edges + eb + q);
                    uint32_t sl = hash_slot(fo, cmask);
                    for (uint32_t probe = 0; probe < cap; probe++) {
                        const uint32_t key = keys[sl];
                        if (key == fo) {
                            bool hovf = false;
#pragma unroll
                            for (int k = 0; k < kCoverSlots; k++) {
                                Cc[k] = add_sat(Cc[k], cv[(size_t)sl * kCoverSlots + k], ovf);
                                H[k] = add_sat(H[k], hv[(size_t)sl * kCoverSlots + k], hovf);
                            }
                            break;
                        }
                        if (key == kEmpty) break;
                        sl = (sl + 1) & cmask;
                    }
                }
                pdf_u128 hs[kCoverSlots], cs[kCoverSlots];
#pragma unroll
                for (int k = 0; k < kCoverSlots; k++) {
                    hs[k] = 0;
                    cs[k] = 0;
                    if (!((smask >> k) & 1u)) continue;
                    const bool first = fx == pid[k] || fy == pid[k];
                    cs[k] = first ? add_sat(Cc[k], H[k], ovf) : Cc[k];
                    hs[k] = first ? 0 : H[k];
                    if (cs[k] == ~(pdf_u128)0) ovf = true;
                    if (rec_type(r) == PDF_INPT) {
                        hs[k] = 0;
                        if (l == 0) total = add_sat(total, cs[k], ovf);
                    }
                }
                if (l > 0) {  // level-0 values are never read
                    uint32_t sl = hash_slot(g, cmask);
                    uint32_t probe = 0;
                    for (; probe < cap; probe++) {
                        if (atomicCAS(keys + sl, kEmpty, g) == kEmpty) break;
                        sl = (sl + 1) & cmask;
                    }
                    if (probe == cap) {
                        atomicOr(&a.acc->err, kErrHashFull);
                    } else {
#pragma unroll
                        for (int k = 0; k < kCoverSlots; k++) {
                            hv[(size_t)sl * kCoverSlots + k] = hs[k];
                            cv[(size_t)sl * kCoverSlots + k] = cs[k];
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    // Block sum of the counts.
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
}

// total = min(2^128 - 1, total + batch); flags are sticky.
__global__ void k_batch_end(DevAcc *acc, uint64_t n_pairs) {
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

template <int BW, int ROBUST, int MODE>
cudaError_t launch_fwd_t(const FwdArgs &a, uint32_t threads, size_t smem, cudaStream_t st) {
    auto kern = k_forward<BW, ROBUST, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = (a.W + BW - 1) / BW;
    if (blocks == 0 || a.n_pieces == 0) return cudaErrorInvalidValue;
    kern<<<blocks, threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int BW>
cudaError_t launch_fwd_bw(const FwdArgs &a, int mode, int robust, uint32_t threads, size_t smem,
                          cudaStream_t st) {
    if (robust) {
        switch (mode) {
            case FWD_FUSED: return launch_fwd_t<BW, 1, FWD_FUSED>(a, threads, smem, st);
            case FWD_SIM: return launch_fwd_t<BW, 1, FWD_SIM>(a, threads, smem, st);
            default: return launch_fwd_t<BW, 1, FWD_MARK>(a, threads, smem, st);
        }
    }
    switch (mode) {
        case FWD_FUSED: return launch_fwd_t<BW, 0, FWD_FUSED>(a, threads, smem, st);
        case FWD_SIM: return launch_fwd_t<BW, 0, FWD_SIM>(a, threads, smem, st);
        default: return launch_fwd_t<BW, 0, FWD_MARK>(a, threads, smem, st);
    }
}

}  // namespace


cudaError_t launch_forward(const FwdArgs &a, int mode, int robust, uint32_t bw, uint32_t threads,
                           size_t smem, cudaStream_t st) {
    switch (bw) {
        case 1: return launch_fwd_bw<1>(a, mode, robust, threads, smem, st);
        case 2: return launch_fwd_bw<2>(a, mode, robust, threads, smem, st);
        case 4: return launch_fwd_bw<4>(a, mode, robust, threads, smem, st);
        case 8: return launch_fwd_bw<8>(a, mode, robust, threads, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

size_t cover_smem_bytes(uint32_t hash_cap) {
    return (((size_t)hash_cap * 4 + 127) & ~(size_t)127) + (size_t)hash_cap * kCoverSlots * 2 * sizeof(pdf_u128);
}

cudaError_t launch_cover(const CoverArgs &a, uint32_t threads, cudaStream_t st) {
    const uint32_t W = (uint32_t)((a.n_pairs + 31) / 32);
    cudaError_t e = cudaMemsetAsync(a.active, 0, (size_t)W * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_active<<<(a.c.n_gates + 255) / 256, 256, 0, st>>>(a);
    const size_t smem = cover_smem_bytes(a.hash_cap);
    e = cudaFuncSetAttribute(k_cover, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_cover<<<(W + a.bw - 1) / a.bw, threads, smem, st>>>(a);
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

cudaError_t launch_batch_begin(DevAcc *acc, cudaStream_t st) {
    k_batch_begin<<<1, 1, 0, st>>>(acc);
    return cudaGetLastError();
}

cudaError_t launch_batch_end(DevAcc *acc, uint64_t n_pairs, cudaStream_t st) {
    k_batch_end<<<1, 1, 0, st>>>(acc, n_pairs);
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
