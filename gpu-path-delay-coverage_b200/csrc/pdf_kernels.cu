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

// Prune (markkernel.cuh:271-293) and, when fused, merge
// (mergekernel.cuh:116-198), levels descending, only over gates whose mark in
// this column block is nonzero.
// Returns the highest level holding a surviving mark, plus one (0 = none).
template <int BW, int MODE>
__device__ __forceinline__ uint32_t prune_merge(const FwdArgs &a, uint32_t *nzb, uint32_t w0, uint32_t top) {
    const uint32_t *edges = a.c.edges;
    uint32_t maxlvl = 0;
    for (int l = (int)top - 1; l >= 0; l--) {
        const uint32_t s = a.c.level_off[l], e = a.c.level_off[l + 1];
        bool lvl_any = false;
        for (uint32_t g = s + threadIdx.x; g < e; g += blockDim.x) {
            {
                if (!((nzb[g >> 5] >> (g & 31)) & 1u)) continue;
                const GateRec r = load_rec(a.c.rec + g);
                uint32_t mk[BW], keep[BW];
#pragma unroll
                for (int j = 0; j < BW; j++) {
                    mk[j] = (w0 + j < a.W) ? a.M[(size_t)g * a.ld + w0 + j] : 0u;
                    keep[j] = rec_po(r) ? 0xFFFFFFFFu : 0u;
                }
                if (!rec_po(r)) {
                    const uint32_t nfo = r.w[1], base = r.w[2] + rec_nfi(r);
                    for (uint32_t k = 0; k < nfo; k++) {
                        const uint32_t fo = __ldg(edges + base + k);
                        if (!((nzb[fo >> 5] >> (fo & 31)) & 1u)) continue;
#pragma unroll
                        for (int j = 0; j < BW; j++)
                            if (w0 + j < a.W) keep[j] |= a.M[(size_t)fo * a.ld + w0 + j];
                    }
                }
                bool any = false;
#pragma unroll
                for (int j = 0; j < BW; j++) {
                    const uint32_t nm = mk[j] & keep[j];
                    if (nm != mk[j]) a.M[(size_t)g * a.ld + w0 + j] = nm;
                    mk[j] = nm;
                    any |= nm != 0;
                }
                if (!any) {
                    atomicAnd(nzb + (g >> 5), ~(1u << (g & 31)));
                    continue;
                }
                lvl_any = true;
                if (MODE == FWD_FUSED) {
                    uint32_t cx = kEmpty, cy = kEmpty;
#pragma unroll
                    for (int j = 0; j < BW; j++) {
                        if (!mk[j] || (cx != kEmpty && cy != kEmpty)) continue;
                        const uint32_t v = a.V[(size_t)g * a.ld + w0 + j];
                        const uint32_t x = mk[j] & ~v, y = mk[j] & v;
                        if (cx == kEmpty && x) cx = (w0 + j) * 32 + (__ffs(x) - 1);
                        if (cy == kEmpty && y) cy = (w0 + j) * 32 + (__ffs(y) - 1);
                    }
                    if (cx != kEmpty) {
                        const uint32_t id = a.pair_base + cx;
                        if (id < *(volatile uint32_t *)(a.first_x + g)) atomicMin(a.first_x + g, id);
                    }
                    if (cy != kEmpty) {
                        const uint32_t id = a.pair_base + cy;
                        if (id < *(volatile uint32_t *)(a.first_y + g)) atomicMin(a.first_y + g, id);
                    }
                }
            }
        }
        if (__syncthreads_or(lvl_any) && maxlvl == 0) maxlvl = (uint32_t)l + 1;
    }
    return maxlvl;
}

// ---------------------------------------------------------------------------
// Forward kernel.
//
// Shared memory: a ring of the last R gates' V, T, M words for this CTA's
// column block (slot = gate & (R - 1)).  While level [s, e) is computed, a
// fan-in f is read from the ring iff f >= e - R, and only gates g >= e - R
// write the ring; within that window no two gates share a slot, so every ring
// read sees its own gate.  Older fan-ins come from the global planes (written
// by this CTA, ordered by __syncthreads).
// ---------------------------------------------------------------------------
template <int BW, int ROBUST, int MODE>
__global__ void __launch_bounds__(1024) k_forward(const FwdArgs a) {
    extern __shared__ uint32_t sm[];
    const uint32_t R = a.ring_gates, Rm = R - 1;
    uint32_t *rV = sm, *rT = sm + (size_t)R * BW, *rM = sm + 2 * (size_t)R * BW;
    const uint32_t blk = blockIdx.x;
    const uint32_t w0 = blk * BW;
    const uint32_t *edges = a.c.edges;
    uint32_t *nzb = a.nzb + (size_t)blk * a.bm_words;
    const uint32_t tailmask = (a.n_pairs & 31) ? ((1u << (a.n_pairs & 31)) - 1u) : 0xFFFFFFFFu;

    if (MODE != FWD_SIM) {
        for (uint32_t q = threadIdx.x; q < a.bm_words; q += blockDim.x) nzb[q] = 0;
        __syncthreads();
    }

    uint32_t fwd_top = 0;  // highest level holding a forward mark, plus one
    for (uint32_t l = 0; l < a.c.n_levels; l++) {
        const uint32_t s = a.c.level_off[l], e = a.c.level_off[l + 1];
        const uint32_t ring_lo = R ? (e > R ? e - R : 0) : e;
        bool lvl_any = false;
        const uint32_t ntask = (e - s) * BW;
        for (uint32_t k = threadIdx.x; k < ntask; k += blockDim.x) {
            const uint32_t g = s + k / BW, j = k % BW, w = w0 + j;
            if (w >= a.W) continue;
            const uint32_t wmask = (w == a.W - 1) ? tailmask : 0xFFFFFFFFu;
            const GateRec r = load_rec(a.c.rec + g);
            const uint32_t type = rec_type(r), nfi = rec_nfi(r);
            auto fetchVT = [&](uint32_t f, uint32_t &fv, uint32_t &ft) {
                if (f >= ring_lo) {
                    fv = rV[(f & Rm) * BW + j];
                    ft = rT[(f & Rm) * BW + j];
                } else {
                    fv = a.V[(size_t)f * a.ld + w];
                    ft = a.T[(size_t)f * a.ld + w];
                }
            };
            auto fetchM = [&](uint32_t f) -> uint32_t {
                return f >= ring_lo ? rM[(f & Rm) * BW + j] : a.M[(size_t)f * a.ld + w];
            };
            uint32_t V, T;
            if (MODE == FWD_MARK) {
                V = a.V[(size_t)g * a.ld + w] & wmask;
                T = a.T[(size_t)g * a.ld + w] & wmask;
            } else if (type == PDF_INPT) {  // simkernel.cuh:112-125 (pairs already formed)
                V = __ldg(a.pi_v + (size_t)g * a.pi_ld + w) & wmask;
                T = __ldg(a.pi_t + (size_t)g * a.pi_ld + w) & wmask;
            } else {
                fetchVT(fanin_id(r, edges, 0), V, T);  // :129, :135
                if (type != PDF_BUFF && type != PDF_FROM && type != PDF_DFF) {
                    if (type == PDF_NOT) not1(V, T);  // :136-141
                    for (uint32_t jj = 1; jj < nfi; jj++) {  // :142-148
                        uint32_t fv, ft;
                        fetchVT(fanin_id(r, edges, jj), fv, ft);
                        fold2(type, V, T, fv, ft);
                    }
                }
                V &= wmask;
                T &= wmask;
            }
            uint32_t M = 0;
            if (MODE != FWD_SIM) {  // markkernel.cuh:226-267
                switch (type) {
                    case PDF_INPT: M = T; break;
                    case PDF_FROM:
                    case PDF_BUFF:
                    case PDF_DFF:
                    case PDF_NOT: M = T ? (T & fetchM(fanin_id(r, edges, 0))) : 0u; break;
                    case PDF_AND:
                    case PDF_NAND:
                    case PDF_OR:
                    case PDF_NOR:
                    case PDF_XOR:
                    case PDF_XNOR: {
                        uint32_t base = T ? (T & fetchM(fanin_id(r, edges, 0))) : 0u;
                        if (base && nfi > 1) {
                            uint32_t acc = 0;
                            for (uint32_t i = 0; i < nfi && (base & ~acc); i++) {
                                uint32_t iv, it;
                                fetchVT(fanin_id(r, edges, i), iv, it);
                                uint32_t term = 0xFFFFFFFFu;
                                for (uint32_t x = 0; x < nfi && term; x++) {
                                    if (x == i) continue;
                                    uint32_t xv, xt;
                                    fetchVT(fanin_id(r, edges, x), xv, xt);
                                    term &= sens<ROBUST>(type, iv, it, xv, xt);
                                }
                                acc |= term;
                            }
                            base &= acc;
                        }
                        M = base;
                        break;
                    }
                    default: break;
                }
            }
            const size_t o = (size_t)g * a.ld + w;
            if (MODE != FWD_MARK) {
                a.V[o] = V;
                a.T[o] = T;
            }
            if (MODE != FWD_SIM) a.M[o] = M;
            if (g >= ring_lo) {
                const uint32_t slot = (g & Rm) * BW + j;
                rV[slot] = V;
                rT[slot] = T;
                rM[slot] = M;
            }
            if (MODE != FWD_SIM && M) {
                bitmap_set_aggregated(nzb, g);
                lvl_any = true;
            }
        }
        if (__syncthreads_or(lvl_any)) fwd_top = l + 1;
    }
    if (MODE == FWD_SIM) return;
    const uint32_t maxlvl = prune_merge<BW, MODE>(a, nzb, w0, fwd_top);
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

// Ordered list of the active pairs (one CTA).
__global__ void __launch_bounds__(1024) k_active_compact(const CoverArgs a, uint32_t W) {
    __shared__ uint32_t s_cnt[1024];
    const uint32_t per = (W + blockDim.x - 1) / blockDim.x;
    const uint32_t q0 = threadIdx.x * per, q1 = min(W, q0 + per);
    uint32_t cnt = 0;
    for (uint32_t q = q0; q < q1; q++) cnt += __popc(a.active[q]);
    s_cnt[threadIdx.x] = cnt;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {  // inclusive scan
        const uint32_t v = threadIdx.x >= off ? s_cnt[threadIdx.x - off] : 0u;
        __syncthreads();
        s_cnt[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t pos = s_cnt[threadIdx.x] - cnt;
    for (uint32_t q = q0; q < q1; q++) {
        uint32_t bits = a.active[q];
        while (bits) {
            a.active_list[pos++] = q * 32 + (__ffs(bits) - 1);
            bits &= bits - 1;
        }
    }
    if (threadIdx.x == blockDim.x - 1) *a.active_count = s_cnt[threadIdx.x];
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

// One CTA per active pair (persistent over the list).  Walks the levels that
// hold marks in the pair's column block, from the top down, over the nets
// the pair marks (kernCover, coverkernel.cuh:193-229):
//   H = [po] + sum h(fo);  C = sum c(fo);  first = pid is first_x or first_y
//   c = C + (first ? H : 0);  h = first ? 0 : H;  h = 0 on INPT
// (unmarked nets hold h = c = 0 and are never stored).  (h, c) live in a
// shared-memory open-addressing table keyed by net id.  Level-0 INPT c values
// are summed into the batch count (kernSumSingle, coverkernel.cuh:77-105).
__global__ void __launch_bounds__(512) k_cover(const CoverArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const uint32_t cap = a.hash_cap, cmask = cap - 1;
    pdf_u128 *hv = reinterpret_cast<pdf_u128 *>(smraw);
    pdf_u128 *cv = hv + cap;
    uint32_t *keys = reinterpret_cast<uint32_t *>(cv + cap);
    __shared__ pdf_u128 s_red[32];
    __shared__ unsigned int s_flags;

    const uint32_t n_active = *a.active_count;
    for (uint32_t ai = blockIdx.x; ai < n_active; ai += gridDim.x) {
        const uint32_t p = a.active_list[ai];
        const uint32_t pid = a.pair_base + p;
        const uint32_t wp = p >> 5, bit = p & 31, blk = wp / a.bw;
        const uint32_t *nzb = a.nzb + (size_t)blk * a.bm_words;
        const uint32_t top = a.blk_maxlvl[blk];
        for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) keys[i] = kEmpty;
        if (threadIdx.x == 0) s_flags = 0;
        __syncthreads();
        pdf_u128 total = 0;
        bool ovf = false;
        for (int l = (int)top - 1; l >= 0; l--) {
            const uint32_t s = a.c.level_off[l], e = a.c.level_off[l + 1];
            if (e > s) {
                const uint32_t q0 = s >> 5, q1 = (e - 1) >> 5;
                for (uint32_t q = q0 + threadIdx.x; q <= q1; q += blockDim.x) {
                    uint32_t bits = nzb[q];
                    if (q == q0) bits &= 0xFFFFFFFFu << (s & 31);
                    if (q == q1) bits &= 0xFFFFFFFFu >> (31 - ((e - 1) & 31));
                    while (bits) {
                        const uint32_t g = q * 32 + (__ffs(bits) - 1);
                        bits &= bits - 1;
                        if (!((a.M[(size_t)g * a.ld + wp] >> bit) & 1u)) continue;
                        const GateRec r = load_rec(a.c.rec + g);
                        pdf_u128 H = rec_po(r) ? 1 : 0, C = 0;
                        const uint32_t nfo = r.w[1], eb = r.w[2] + rec_nfi(r);
                        for (uint32_t k = 0; k < nfo; k++) {
                            const uint32_t fo = __ldg(a.c.edges + eb + k);
                            uint32_t sl = hash_slot(fo, cmask);
                            for (uint32_t probe = 0; probe < cap; probe++) {
                                const uint32_t key = keys[sl];
                                if (key == fo) {
                                    bool dummy = false;
                                    C = add_sat(C, cv[sl], ovf);
                                    H = add_sat(H, hv[sl], dummy);
                                    break;
                                }
                                if (key == kEmpty) break;
                                sl = (sl + 1) & cmask;
                            }
                        }
                        const bool first = a.first_x[g] == pid || a.first_y[g] == pid;
                        pdf_u128 c = C, h = H;
                        if (first) {
                            c = add_sat(C, H, ovf);
                            h = 0;
                        }
                        if (c == ~(pdf_u128)0) ovf = true;
                        if (rec_type(r) == PDF_INPT) {
                            h = 0;
                            if (l == 0) total = add_sat(total, c, ovf);
                        }
                        if (l > 0) {  // level-0 values are never read
                            uint32_t sl = hash_slot(g, cmask);
                            uint32_t probe = 0;
                            for (; probe < cap; probe++) {
                                if (atomicCAS(keys + sl, kEmpty, g) == kEmpty) break;
                                sl = (sl + 1) & cmask;
                            }
                            if (probe == cap) {
                                atomicOr(&a.acc->err, 1u);  // table full
                            } else {
                                hv[sl] = h;
                                cv[sl] = c;
                            }
                        }
                    }
                }
            }
            __syncthreads();
        }
        // Block sum of the pair's count.
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

size_t forward_smem_bytes(uint32_t bw, uint32_t ring_gates) {
    return (size_t)ring_gates * bw * 3 * sizeof(uint32_t);
}

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
    return (size_t)hash_cap * (2 * sizeof(pdf_u128) + sizeof(uint32_t));
}

cudaError_t launch_cover(const CoverArgs &a, uint32_t grid, uint32_t threads, cudaStream_t st) {
    const uint32_t W = (uint32_t)((a.n_pairs + 31) / 32);
    cudaError_t e = cudaMemsetAsync(a.active, 0, (size_t)W * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_active<<<(a.c.n_gates + 255) / 256, 256, 0, st>>>(a);
    k_active_compact<<<1, 1024, 0, st>>>(a, W);
    const size_t smem = cover_smem_bytes(a.hash_cap);
    e = cudaFuncSetAttribute(k_cover, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_cover<<<grid, threads, smem, st>>>(a);
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
