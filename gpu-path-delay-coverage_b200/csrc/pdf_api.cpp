// pdf_api.cpp -- the C ABI (include/pdf.h) over the sm_100a kernels.
//
// Every call returns a status and never exits: the reference's HANDLE_ERROR
// exit(EXIT_FAILURE) (simkernel.cuh:32-39, markkernel.cuh:13-20,
// mergekernel.cuh:17-24, coverkernel.cuh:15-25) becomes PDF_ECUDA / PDF_EINVAL.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <new>
#include <vector>

#include "pdf.h"
#include "pdf_inject.h"
#include "pdf_internal.h"
#include "pdf_kernels.cuh"

#include <atomic>

namespace {
std::atomic<uint32_t> g_inject[3];
}  // namespace

bool inject_fail(int site) {
    if (site < 1 || site > 2) return false;
    uint32_t n = g_inject[site].load();
    while (n > 0)
        if (g_inject[site].compare_exchange_weak(n, n - 1)) return true;
    return false;
}
cudaError_t dev_alloc(void **p, size_t bytes) {
    if (inject_fail(PDF_INJECT_DEVICE_ALLOC)) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}
cudaError_t host_alloc(void **p, size_t bytes) {
    if (inject_fail(PDF_INJECT_HOST_ALLOC)) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaHostAlloc(p, bytes, cudaHostAllocDefault);
}

extern "C" pdf_status pdf_test_inject(int site, uint32_t count) {
    if (site < 1 || site > 2) return PDF_EINVAL;
    g_inject[site].store(count);
    return PDF_OK;
}

namespace {


// The last failing CUDA call of this thread, for pdf_last_error().
thread_local char g_last_error[256];
static void note_cuda_error(cudaError_t e, const char *call, int line) {
    std::snprintf(g_last_error, sizeof g_last_error, "%s (%d) at pdf_api.cpp:%d: %.160s", cudaGetErrorName(e),
                  (int)e, line, call);
}

#define PDF_CUDA(call)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) {                        \
            note_cuda_error(e_, #call, __LINE__);       \
            (void)cudaGetLastError();                   \
            return e_ == cudaErrorMemoryAllocation ? PDF_ENOMEM : PDF_ECUDA; \
        }                                               \
    } while (0)

pdf_status err_status(unsigned int err) {
    if (err & kErrHashFull) return PDF_ENOMEM;
    if (err & kErrTimeout) return PDF_ETIMEOUT;
    return PDF_OK;
}

void set_msg(char *msg, size_t len, const char *fmt, unsigned long long a = 0,
             unsigned long long b = 0) {
    if (msg && len) std::snprintf(msg, len, fmt, a, b);
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    void release() {
        if (p && cudaFree(p) != cudaSuccess) (void)cudaGetLastError();
        p = nullptr;
        bytes = 0;
    }
    // Grow to at least `need` bytes (contents are not kept).
    cudaError_t ensure(size_t need) {
        if (bytes >= need) return cudaSuccess;
        release();
        cudaError_t e = dev_alloc(&p, need ? need : 16);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

// Scoped device selection.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    // Every entry point that touches the device starts here.  Its launches
    // are checked with cudaGetLastError, which would also report a failure
    // that an earlier call on this thread left unchecked (the caller's own,
    // say), so that slot is cleared first; errors that poison the context
    // come back from every later call anyway.  A failure here is reported
    // through `ok` and not left pending for the caller's next check.
    explicit DeviceGuard(int dev) {
        (void)cudaGetLastError();
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
            (void)cudaGetLastError();
        }
        ok = cudaSetDevice(dev) == cudaSuccess;
        if (!ok) (void)cudaGetLastError();
    }
    ~DeviceGuard() {
        if (prev >= 0 && cudaSetDevice(prev) != cudaSuccess) (void)cudaGetLastError();
    }
};

}  // namespace

// Per-batch device workspace (owned by a state, or by a circuit for the
// stage calls).
struct Workspace {
    DevBuf nzb, maxlvl, active, active_list;
    DevBuf over_list, spill;  // pairs for the spill cover and its per-net (h, c) slots
    DevBuf nzb_fine, maxlvl_fine;  // lane circuits: the cover's bitmaps per quarter column block
    DevBuf pi_counts;         // pdf_cover_counts: paths per (primary input, pair)
    uint32_t spill_slots = 0;
    DevBuf seg_first;  // (net, pair) hash set of the cover with segments
    uint64_t seg_first_mask = 0;
    DevBuf planes;   // internal V, T, M planes when the caller gives none
    DevBuf pi;       // staged host pairs
    uint64_t plane_ld = 0, plane_words = 0;
    void release() {
        nzb.release();
        maxlvl.release();
        active.release();
        active_list.release();
        over_list.release();
        spill.release();
        nzb_fine.release();
        maxlvl_fine.release();
        pi_counts.release();
        spill_slots = 0;
        seg_first.release();
        seg_first_mask = 0;
        planes.release();
        pi.release();
    }
};

struct pdf_circuit {
    int device = 0;
    int mark_mode = PDF_MARK_DEFAULT;
    pdf_circuit_info info{};
    DevBuf rec, edges, level_off, pieces, far, err;
    DevCircuit dc{};
    uint32_t bw = 4, threads = 512, ring = 0, ring2 = 0, farcap = 0;
    uint32_t cap = 512, ecap = 2048, n_pieces = 0, bm_shared = 0;
    uint32_t off_ring = 0, off_rec = 0, off_edge = 0, off_fid = 0, off_bm = 0, off_pbits = 0, off_mbar = 0;
    size_t fwd_smem = 0;
    uint32_t hash_cap = 4096, cover_threads = 256, cover_grid = 0;
    uint32_t wait_polls = 0;  // bound of the forward kernels' waits (0 = the default)
    uint32_t occ = 1;  // forward CTAs per SM its registers and shared memory are sized for
    uint64_t chain = 0;  // length of one CTA's walk (pieces, or gates for the lane kernel)
    Workspace stage;  // scratch of the stage calls
    std::mutex mu;    // serialises the stage scratch
    // segments longer than one net
    uint32_t seg_len = 1;
    uint64_t n_segs = 0;
    DevBuf segs, seg_off;
    // entries of a state's first-detect arrays: one per segment
    uint64_t n_first() const { return seg_len > 1 ? n_segs : info.n_gates; }
    SegArgs seg_args() const {
        SegArgs a{};
        if (seg_len > 1) {
            a.segs = segs.as<uint32_t>();
            a.seg_off = seg_off.as<uint32_t>();
            a.N = seg_len;
            a.S = (uint32_t)n_segs;
        }
        return a;
    }
};

struct ProfEvents {
    cudaEvent_t ev[4];  // call start, forward end, cover end, call end
};

struct pdf_state {
    pdf_circuit *c = nullptr;
    int device = 0;  // the circuit's device (destroy does not need the circuit)
    DevBuf first_x, first_y, acc;
    DevAcc *host_acc = nullptr;  // host copy of the accumulators (pinned: read back by DMA, after a
                                 // stream sync, without the driver's staging of pageable copies)
    Workspace ws;
    std::mutex mu;
    bool profiling = false;
    std::vector<ProfEvents> prof;   // one entry per profiled call
    std::vector<ProfEvents> pool;   // recycled events
    ProfEvents *pe = nullptr;       // events of the call in progress
    // the batch marked by pdf_grade_mark_async and not yet counted
    bool pending = false;
    const uint32_t *pend_M = nullptr;
    uint64_t pend_ld = 0, pend_n = 0, pend_base = 0;
};

namespace {
void prof_release(std::vector<ProfEvents> &v) {
    for (auto &p : v)
        for (auto &e : p.ev) cudaEventDestroy(e);
    v.clear();
}
}  // namespace

// ---------------------------------------------------------------------------

extern "C" const char *pdf_last_error(void) { return g_last_error; }

extern "C" const char *pdf_status_string(int s) {
    switch (s) {
        case PDF_OK: return "ok";
        case PDF_EINVAL: return "invalid argument";
        case PDF_ENOMEM: return "out of memory";
        case PDF_EOVERFLOW: return "path count overflow";
        case PDF_ETIMEOUT: return "device wait timed out";
        case PDF_ECUDA: return "CUDA error";
        case PDF_ENOTSUP: return "not supported";
        case PDF_EBUSY: return "busy";
        case PDF_ENODEV: return "no CUDA device";
        case PDF_ELIMIT: return "request exceeds the fixed scratch of an allocation-free call";
        default: return "unknown status";
    }
}

extern "C" int pdf_abi_version(void) { return PDF_ABI_VERSION; }

extern "C" pdf_status pdf_netlist_check(const pdf_netlist *nl, char *msg, size_t len) {
    if (!nl) {
        set_msg(msg, len, "null netlist");
        return PDF_EINVAL;
    }
    const uint32_t G = nl->n_gates, L = nl->n_levels;
    if (G == 0 || G == 0xFFFFFFFFu || L == 0 || !nl->level_offsets || !nl->type || !nl->po ||
        !nl->nfi || !nl->nfo || !nl->edge_offset || (!nl->edges && nl->n_edges)) {
        set_msg(msg, len, "empty netlist or missing array");
        return PDF_EINVAL;
    }
    if (nl->n_edges >= 0xFFFFFFFFull) {
        set_msg(msg, len, "too many edges (%llu)", nl->n_edges);
        return PDF_EINVAL;
    }
    if (nl->level_offsets[0] != 0 || nl->level_offsets[L] != G) {
        set_msg(msg, len, "level_offsets must start at 0 and end at n_gates");
        return PDF_EINVAL;
    }
    for (uint32_t l = 0; l < L; l++)
        if (nl->level_offsets[l + 1] < nl->level_offsets[l]) {
            set_msg(msg, len, "level_offsets decrease at level %llu", l);
            return PDF_EINVAL;
        }
    const uint32_t npi = nl->level_offsets[1];
    if (npi == 0) {
        set_msg(msg, len, "level 0 (primary inputs) is empty");
        return PDF_EINVAL;
    }
    std::vector<uint32_t> level(G);
    for (uint32_t l = 0; l < L; l++)
        for (uint32_t g = nl->level_offsets[l]; g < nl->level_offsets[l + 1]; g++) level[g] = l;
    for (uint32_t g = 0; g < G; g++) {
        const uint32_t t = nl->type[g];
        if (t >= PDF_NTYPES) {
            set_msg(msg, len, "gate %llu: unknown type code %llu", g, t);
            return PDF_EINVAL;
        }
        if (nl->po[g] > 1) {
            set_msg(msg, len, "gate %llu: po must be 0 or 1", g);
            return PDF_EINVAL;
        }
        if ((t == PDF_INPT) != (g < npi)) {
            set_msg(msg, len, "gate %llu: INPT gates must be exactly level 0", g);
            return PDF_EINVAL;
        }
        if (t == PDF_INPT ? nl->nfi[g] != 0 : (nl->nfi[g] == 0 || nl->nfi[g] > 255)) {
            set_msg(msg, len, "gate %llu: bad fan-in count %llu", g, nl->nfi[g]);
            return PDF_EINVAL;
        }
        const uint64_t end = nl->edge_offset[g] + (uint64_t)nl->nfi[g] + nl->nfo[g];
        if (end > nl->n_edges || end < nl->edge_offset[g]) {
            set_msg(msg, len, "gate %llu: edge range out of bounds", g);
            return PDF_EINVAL;
        }
        for (uint32_t j = 0; j < nl->nfi[g]; j++) {
            const uint32_t f = nl->edges[nl->edge_offset[g] + j];
            if (f >= G || level[f] >= level[g]) {
                set_msg(msg, len, "gate %llu: fan-in %llu not on a lower level", g, f);
                return PDF_EINVAL;
            }
        }
        for (uint32_t k = 0; k < nl->nfo[g]; k++) {
            const uint32_t f = nl->edges[nl->edge_offset[g] + nl->nfi[g] + k];
            if (f >= G || level[f] <= level[g]) {
                set_msg(msg, len, "gate %llu: fan-out %llu not on a higher level", g, f);
                return PDF_EINVAL;
            }
        }
    }
    // Fan-out lists must be the transpose of the fan-in lists (as multisets).
    std::vector<uint64_t> cnt(G, 0);
    for (uint32_t g = 0; g < G; g++)
        for (uint32_t j = 0; j < nl->nfi[g]; j++) cnt[nl->edges[nl->edge_offset[g] + j]]++;
    for (uint32_t g = 0; g < G; g++)
        if (cnt[g] != nl->nfo[g]) {
            set_msg(msg, len, "gate %llu: fan-out count %llu differs from its fan-in uses", g,
                    nl->nfo[g]);
            return PDF_EINVAL;
        }
    // Multiset comparison: the consumers of each gate (transposed from the
    // fan-in lists by a counting sort, hence ascending) against its fan-out
    // list, sorted.  Linear in the edges apart from sorting each list.
    {
        std::vector<uint64_t> start(G + 1, 0);
        for (uint32_t g = 0; g < G; g++) start[g + 1] = start[g] + cnt[g];
        std::vector<uint32_t> cons(start[G]);
        std::vector<uint64_t> fill(start.begin(), start.end() - 1);
        for (uint32_t g = 0; g < G; g++)
            for (uint32_t j = 0; j < nl->nfi[g]; j++) cons[fill[nl->edges[nl->edge_offset[g] + j]]++] = g;
        std::vector<uint32_t> fo;
        for (uint32_t g = 0; g < G; g++) {
            const uint32_t *e = nl->edges + nl->edge_offset[g] + nl->nfi[g];
            fo.assign(e, e + nl->nfo[g]);
            std::sort(fo.begin(), fo.end());
            if (!std::equal(fo.begin(), fo.end(), cons.begin() + start[g])) {
                set_msg(msg, len, "fan-out lists are not the transpose of the fan-in lists (gate %llu)", g);
                return PDF_EINVAL;
            }
        }
    }
    set_msg(msg, len, "ok");
    return PDF_OK;
}

// ---------------------------------------------------------------------------

namespace {

// Segments of N nets (2..8): every directed subpath of N nets, listed by
// first net ascending, then depth first along fan-outs in edge order (the
// reference's generateSegmentList lives in its missing util/segment.cuh).
// Counted first (paths of k nets from g = sum over fan-outs of paths of k - 1
// nets), then written as [S][N] with a CSR offset per first net.
constexpr uint64_t kMaxSegWords = 1ull << 28;  // S * N gate ids at most (1 GiB)

pdf_status build_segments(pdf_circuit *c, const pdf_netlist *nl, uint32_t N) {
    const uint32_t G = nl->n_gates;
    auto fo = [&](uint32_t g, uint32_t k) { return nl->edges[nl->edge_offset[g] + nl->nfi[g] + k]; };
    std::vector<uint64_t> cnt(G, 1), nxt(G);
    for (uint32_t k = 1; k < N; k++) {
        for (uint32_t g = 0; g < G; g++) {
            uint64_t t = 0;
            for (uint32_t j = 0; j < nl->nfo[g]; j++) t = std::min(t + cnt[fo(g, j)], kMaxSegWords + 1);
            nxt[g] = t;
        }
        cnt.swap(nxt);
    }
    std::vector<uint32_t> off(G + 1, 0);
    uint64_t S = 0;
    for (uint32_t g = 0; g < G; g++) {
        S += cnt[g];
        if (S * N > kMaxSegWords) return PDF_ENOTSUP;
        off[g + 1] = (uint32_t)S;
    }
    std::vector<uint32_t> segs;
    try {
        segs.resize(S * N);
    } catch (const std::bad_alloc &) {
        return PDF_ENOMEM;
    }
    uint32_t path[8], idx[8];
    uint64_t w = 0;
    for (uint32_t g0 = 0; g0 < G; g0++) {
        int d = 0;
        path[0] = g0;
        idx[0] = 0;
        while (d >= 0) {
            if ((uint32_t)d == N - 1) {
                std::memcpy(segs.data() + w, path, N * 4);
                w += N;
                d--;
            } else if (idx[d] < nl->nfo[path[d]]) {
                path[d + 1] = fo(path[d], idx[d]++);
                idx[d + 1] = 0;
                d++;
            } else {
                d--;
            }
        }
    }
    if (w != S * N) return PDF_EINVAL;
    if (c->segs.ensure(std::max<uint64_t>(S * N * 4, 16)) != cudaSuccess ||
        c->seg_off.ensure((uint64_t)(G + 1) * 4) != cudaSuccess)
        return PDF_ENOMEM;
    if ((S && cudaMemcpy(c->segs.p, segs.data(), S * N * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(c->seg_off.p, off.data(), (uint64_t)(G + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return PDF_ECUDA;
    c->seg_len = N;
    c->n_segs = S;
    return PDF_OK;
}

}  // namespace

extern "C" pdf_status pdf_circuit_create(const pdf_netlist *nl, const pdf_circuit_opts *opts,
                                         pdf_circuit **out) {
    if (!out) return PDF_EINVAL;
    *out = nullptr;
    pdf_status st = pdf_netlist_check(nl, nullptr, 0);
    if (st != PDF_OK) return st;
    pdf_circuit_opts o{};
    if (opts) o = *opts;
    if (o.mark_mode < PDF_MARK_DEFAULT || o.mark_mode > PDF_MARK_FIXED_NONROBUST) return PDF_EINVAL;
    if (o.seg_len > 8) return PDF_EINVAL;
    if (o.tile_words && o.tile_words != 1 && o.tile_words != 2 && o.tile_words != 4 && o.tile_words != 8 &&
        !lane_tile(o.tile_words))
        return PDF_EINVAL;
    if (o.threads && (o.threads < 64 || o.threads > 1024 || o.threads % 32)) return PDF_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return PDF_ENODEV;
    }
    if (o.device < 0 || o.device >= ndev) return PDF_EINVAL;
    DeviceGuard dg(o.device);
    if (!dg.ok) return PDF_ECUDA;

    // source words address gates with 31 bits and slots with 30 (pdf_device.cuh)
    if (nl->n_gates >= SRC_FAR) return PDF_ENOTSUP;
    pdf_circuit *c = new (std::nothrow) pdf_circuit();
    if (!c) return PDF_ENOMEM;
    c->device = o.device;
    c->mark_mode = o.mark_mode;
    c->wait_polls = o.wait_polls;
    const uint32_t G = nl->n_gates, L = nl->n_levels;
    pdf_circuit_info &inf = c->info;
    inf.n_gates = G;
    inf.n_levels = L;
    inf.n_pi = nl->level_offsets[1];
    inf.n_edges = nl->n_edges;
    for (uint32_t g = 0; g < G; g++) {
        inf.n_po += nl->po[g] ? 1 : 0;
        inf.max_nfi = std::max(inf.max_nfi, nl->nfi[g]);
        inf.max_nfo = std::max(inf.max_nfo, nl->nfo[g]);
    }
    for (uint32_t l = 0; l < L; l++)
        inf.max_level_width = std::max(inf.max_level_width, nl->level_offsets[l + 1] - nl->level_offsets[l]);

    // Canonical edge array: each gate's fan-ins then fan-outs, gates in id
    // order, so that a run of gates owns one contiguous slice (staged into
    // shared memory by a bulk copy).  Padded so 16-byte rounding stays inside.
    std::vector<uint32_t> edges;
    std::vector<uint64_t> eoff(G + 1);
    edges.reserve(nl->n_edges + 8);
    for (uint32_t g = 0; g < G; g++) {
        eoff[g] = edges.size();
        const uint32_t *e = nl->edges + nl->edge_offset[g];
        edges.insert(edges.end(), e, e + nl->nfi[g] + nl->nfo[g]);
    }
    eoff[G] = edges.size();
    while (edges.size() % 4) edges.push_back(0);
    for (int i = 0; i < 4; i++) edges.push_back(0);

    std::vector<GateRec> recs(G);
    for (uint32_t g = 0; g < G; g++) {
        GateRec &r = recs[g];
        std::memset(&r, 0, sizeof r);
        r.w[0] = make_rec_header(nl->type[g], nl->po[g], nl->nfi[g], o.mark_mode >= PDF_MARK_FIXED_ROBUST);
        r.w[1] = nl->nfo[g];
        r.w[2] = (uint32_t)eoff[g];  // w[3..6]: source words, set with the launch plan below
        r.w[7] = nl->nfi[g] ? edges[eoff[g]] : 0;
    }

    // Launch plan: CTAs of `threads` threads own `bw` words of pairs; two
    // CTAs per SM share its shared memory.
    struct {
        int sharedMemPerBlockOptin = 0, sharedMemPerMultiprocessor = 0, multiProcessorCount = 0;
    } prop;
    if (cudaDeviceGetAttribute(&prop.sharedMemPerBlockOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, o.device) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&prop.sharedMemPerMultiprocessor, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                               o.device) != cudaSuccess ||
        cudaDeviceGetAttribute(&prop.multiProcessorCount, cudaDevAttrMultiProcessorCount, o.device) != cudaSuccess) {
        delete c;
        return PDF_ECUDA;
    }
    // Default tile.  The lane kernel (a warp per gate) when the circuit's
    // largest batch gives it at least one 1,024-pair column block per SM and
    // its levels average 1,024 gates or more; of its tiles the one with the
    // least modelled time, waves of CTAs (one per SM) x words per CTA x the
    // tile's time per word relative to 32 words, measured on a batch that
    // fills the GPU: 1.0, 0.67, 0.52 at 32, 64, 128 words.  (1M gates, 5,000-
    // gate levels, 262,144 pairs: 61, 36 and 58 ms at 32, 64, 128 words, 128
    // CTAs being one wave at 64 words and 64 CTAs leaving half the SMs idle
    // at 128.)  On narrower or smaller jobs the lane kernel's few CTAs leave
    // SMs idle (20,000 gates, 32,768 pairs: 0.92 against 0.25 ms): 4 words
    // (128 pairs) per CTA, or 8 when the largest batch still gives at least
    // two 8-word CTAs per SM, which halves the per-gate work of record decode
    // and staging per pair (1M gates: 137 ms at 8 words against 165 ms at 4).
    const uint64_t max_words = ((o.max_pairs ? o.max_pairs : 65536ull) + 31) / 32;
    const uint64_t mean_width = L > 1 ? (G - inf.n_pi) / (L - 1) : G;
    const uint64_t sms = (uint64_t)prop.multiProcessorCount;
    if (o.tile_words) {
        c->bw = o.tile_words;
    } else if (max_words / kLaneWords >= sms && mean_width >= 1024) {
        double best = 0;
        for (const auto &t : {std::make_pair(kLaneWords, 1.0), std::make_pair(kLaneWords2, 0.67),
                              std::make_pair(kLaneWords4, 0.52)}) {
            const uint64_t ctas = (max_words + t.first - 1) / t.first;
            const double cost = (double)((ctas + sms - 1) / sms) * t.first * t.second;
            if (!best || cost < best) {
                best = cost;
                c->bw = t.first;
            }
        }
    } else {
        c->bw = max_words / 8 >= 2ull * sms ? 8u : 4u;
    }
    const bool lanes = lane_tile(c->bw);
    if (lanes) {
        // The lane kernel reads every fan-in from its plane row: source words
        // are the fan-in ids themselves, flagged SRC_ZERO when the fan-in is
        // a killed gate (S0 whatever its inputs); a gate writes its rows
        // (RF_SPILL) only when some gate reads them.
        std::vector<uint8_t> read(G, 0);
        for (uint32_t g = 0; g < G; g++)
            for (uint32_t q = 0; q < nl->nfi[g]; q++) {
                const uint32_t f = edges[eoff[g] + q];
                const bool zero = q < kInlineFanins && (recs[f].w[0] & RF_KILL);
                if (q < kInlineFanins) recs[g].w[3 + q] = f | (zero ? SRC_ZERO : 0u);
                if (!zero) read[f] = 1;
            }
        for (uint32_t g = 0; g < G; g++)
            if (read[g]) recs[g].w[0] |= RF_SPILL;
    }
    const uint32_t max_threads = lanes ? lane_threads(c->bw) : (c->bw >= 8 ? 512 : 1024);
    uint32_t threads_default = 512;  // set from the piece size below
    auto al = [](size_t x) { return (x + 127) & ~(size_t)127; };
    const uint32_t bm_words = (G + 31) / 32;
    // Pieces (the kernels' unit of staging and of synchronisation), sized
    // from the widest level above the inputs (the inputs' level, often the
    // widest, just splits into more pieces): runs of one level, <= cap gates,
    // edge slice <= ecap words.
    uint32_t widest = 1;
    for (uint32_t l = 1; l < L; l++) widest = std::max(widest, nl->level_offsets[l + 1] - nl->level_offsets[l]);
    if (L == 1) widest = inf.max_level_width;
    c->cap = lanes ? 0u : std::min<uint32_t>(512, (widest + 31) & ~31u);
    // one thread per gate of a piece plus two warps that have none: they
    // issue the next piece's far-row copies
    threads_default = lanes ? lane_threads(c->bw) : std::min<uint32_t>(max_threads, c->cap + 64);
    c->threads = o.threads ? std::min(o.threads, max_threads) : threads_default;
    // a block size given by the caller also bounds the pieces: threads - 64
    // gates, so two warps stay free for the far-row copies
    if (!lanes && o.threads && c->threads >= 128) c->cap = std::min(c->cap, (c->threads - 64) & ~31u);
    // CTAs per SM that the registers allow for this block size (at most 4);
    // the dynamic shared memory of the forward kernels is then an equal share
    // of the SM, less 1 KiB per CTA the system keeps and 1 KiB for the
    // kernels' static variables (the batched kernel keeps its arguments there).
    {
        const int regs = forward_kernel_regs(c->bw, c->mark_mode);
        if (regs <= 0) {
            delete c;
            return PDF_ECUDA;
        }
        const uint32_t warps = (c->threads + 31) / 32;
        const uint32_t warp_regs = ((uint32_t)regs * 32 + 255) & ~255u;
        uint32_t occ = std::min<uint32_t>(65536 / (warps * warp_regs), 2048 / (warps * 32));
        c->occ = std::max<uint32_t>(1, std::min<uint32_t>(occ, 4));
    }
    const size_t budget = std::min<size_t>((size_t)prop.sharedMemPerBlockOptin,
                                           (size_t)prop.sharedMemPerMultiprocessor / c->occ - 1024) -
                          1024;
    c->ecap = 2048;
    std::vector<Piece> pieces;
    std::vector<uint32_t> far_ids;
    if (lanes) {
        // The lane kernel keeps on chip two buffers of staged gate records
        // and the column block's mark bitmap (in global memory when it does
        // not fit); its pieces are runs of one level of <= cap gates: 2 x
        // kLaneRecs when those buffers fit beside a shared-memory bitmap (a
        // barrier per piece, so wide levels take half as many), else
        // kLaneRecs.
        const size_t bm_bytes = (size_t)bm_words * 4;
        c->cap = kLaneRecs;
        if (widest > kLaneRecs &&
            2 * 2 * (size_t)kLaneRecs * sizeof(GateRec) + al(bm_bytes) + 2048 <= budget)
            c->cap = 2 * kLaneRecs;
        for (uint32_t l = 0; l < L; l++)
            for (uint32_t a = nl->level_offsets[l]; a < nl->level_offsets[l + 1]; a += c->cap) {
                Piece p{};
                p.a = a;
                p.b = std::min(a + c->cap, nl->level_offsets[l + 1]);
                p.level = l;
                pieces.push_back(p);
            }
        c->n_pieces = (uint32_t)pieces.size();
        const size_t rec_bytes = 2 * (size_t)c->cap * sizeof(GateRec);
        c->off_rec = 0;
        c->off_bm = (uint32_t)rec_bytes;
        c->bm_shared = rec_bytes + bm_bytes + 2048 <= budget ? 1u : 0u;
        c->fwd_smem = rec_bytes + (c->bm_shared ? al(bm_bytes) : 0);
        c->chain = G;
        while (far_ids.size() < 4) far_ids.push_back(0);
    } else {
        auto f4 = [](uint64_t x) { return x & ~(uint64_t)3; };
        auto c4 = [](uint64_t x) { return (x + 3) & ~(uint64_t)3; };
        for (uint32_t l = 0; l < L; l++) {
            const uint32_t s0 = nl->level_offsets[l], e0 = nl->level_offsets[l + 1];
            for (uint32_t a = s0; a < e0;) {
                uint32_t b = a + 1;
                while (b < e0 && b - a < c->cap && c4(eoff[b + 1]) - f4(eoff[a]) <= c->ecap) b++;
                Piece p{};
                p.a = a;
                p.b = b;
                p.level = l;
                if (c4(eoff[b]) - f4(eoff[a]) <= c->ecap) {
                    p.ea = (uint32_t)f4(eoff[a]);
                    p.eb = (uint32_t)c4(eoff[b]);
                } else {
                    p.ea = p.eb = 0xFFFFFFFFu;  // one gate with a huge edge list: read in place
                }
                pieces.push_back(p);
                a = b;
            }
        }
        c->n_pieces = (uint32_t)pieces.size();
        if (c->n_pieces > 65536) {
            delete c;
            return PDF_ENOTSUP;
        }
        // Far fan-ins of piece i (ring of R slots): fan-ins 0..3 of its gates
        // below b_i - R.  Those below a_{i-1} (complete when piece i - 1 starts)
        // go to the piece's deduplicated far list, up to `limit` entries; the rest
        // are read from their plane rows.  Fills the source words w[3..6].
        auto far_lists = [&](uint32_t R, uint32_t limit) -> uint32_t {
            uint32_t worst = 0;
            far_ids.clear();
            std::vector<uint32_t> seen(G, 0xFFFFFFFFu);  // gate -> slot in the current piece's list
            std::vector<uint32_t> list;
            for (size_t i = 0; i < pieces.size(); i++) {
                Piece &p = pieces[i];
                const uint32_t lo = p.b > R ? p.b - R : 0;
                const uint32_t done = i ? pieces[i - 1].a : 0;
                list.clear();
                for (uint32_t g = p.a; g < p.b; g++) {
                    const uint32_t nq = std::min<uint32_t>(nl->nfi[g], kInlineFanins);
                    for (uint32_t q = 0; q < nq; q++) {
                        const uint32_t f = edges[eoff[g] + q];
                        uint32_t sw = f & (R - 1);
                        if (f < lo) {
                            sw = SRC_PLANE | f;
                            if (f < done) {
                                if (seen[f] == 0xFFFFFFFFu && list.size() < limit) {
                                    seen[f] = (uint32_t)list.size();
                                    list.push_back(f);
                                }
                                if (seen[f] != 0xFFFFFFFFu) sw = SRC_FAR | seen[f];
                            }
                        }
                        recs[g].w[3 + q] = sw;
                        if (sw & SRC_PLANE || sw & SRC_FAR) recs[f].w[0] |= RF_SPILL;
                    }
                    for (uint32_t q = kInlineFanins; q < nl->nfi[g]; q++) {  // read from edges[] at run time
                        const uint32_t f = edges[eoff[g] + q];
                        if (f < lo) recs[f].w[0] |= RF_SPILL;
                    }
                }
                for (uint32_t f : list) seen[f] = 0xFFFFFFFFu;
                worst = std::max<uint32_t>(worst, (uint32_t)list.size());
                p.far_off = (uint32_t)far_ids.size();
                p.far_n = (uint32_t)list.size();
                far_ids.insert(far_ids.end(), list.begin(), list.end());
                // lists start on 16-byte boundaries: the kernel stages the next
                // piece's list by a bulk copy located from this piece's fields
                while (far_ids.size() & 3) far_ids.push_back(0);
            }
            for (size_t i = 0; i < pieces.size(); i++) pieces[i].nfar_n = i + 1 < pieces.size() ? pieces[i + 1].far_n : 0;
            return worst;
        };
        // Shared memory of k_forward: 2 record buffers; one region holding the
        // reverse pass's 2 edge buffers or the forward pass's 2 far buffers;
        // bitmap; piece bits; barriers; the ring.  The ring: the largest power of
        // two (>= cap, <= 2 * n_gates) that leaves room for far lists of 64
        // entries; the far lists then get the rest of the budget.
        const size_t rec_bytes = al(2 * (size_t)c->cap * sizeof(GateRec));
        const size_t bm_bytes = (size_t)bm_words * 4 <= 16384 ? al((size_t)bm_words * 4) : 0;
        const size_t fixed = rec_bytes + bm_bytes + al(((size_t)c->n_pieces + 31) / 32 * 4) + 128;
        const size_t edge_bytes = 2 * (size_t)c->ecap * 4;
        const size_t far_entry = (size_t)2 * 3 * c->bw * 4;  // one far slot in both buffers, 3 planes
        uint32_t rmin = 32;
        while (rmin < c->cap) rmin *= 2;
        uint32_t rmax = rmin;
        while ((uint64_t)rmax < 2 * (uint64_t)G && fixed + (size_t)rmax * 2 * c->bw * 12 <= budget) rmax *= 2;
        // the ring's memory also holds the reverse pass's row staging buffers
        const size_t rows_bytes = (size_t)2 * c->cap * 2 * c->bw * 4;
        auto ring_bytes = [&](size_t R) { return std::max(R * c->bw * 12, rows_bytes); };
        // The largest ring that fits wins: a smaller ring with longer far lists
        // was measured slower (1M gates, 5,000-gate levels: 116.8 against 109.9
        // ms) although it leaves fewer fan-ins to plane-row reads.
        // far region (far rows of two pieces, or the reverse pass's edges) and
        // the two staged far-id lists, for lists of n entries
        auto far_bytes = [&](size_t n) { return al(std::max(edge_bytes, n * far_entry)) + al(2 * n * 4); };
        uint32_t ring = 0;
        for (uint32_t R = rmax; R >= rmin && !ring; R /= 2)
            if (fixed + far_bytes(64) + ring_bytes(R) <= budget) ring = R;
        if (!ring) {
            delete c;
            return PDF_ENOTSUP;
        }
        const size_t far_room = budget - fixed - ring_bytes(ring);
        uint32_t far_limit = (uint32_t)std::min<size_t>(kMaxFar, far_room / (far_entry + 8)) & ~3u;
        while (far_limit > 64 && far_bytes(far_limit) > far_room) far_limit -= 4;
        const uint32_t farcap = std::max<uint32_t>(4, (far_lists(ring, far_limit) + 3) & ~3u);
        while (far_ids.size() < 4) far_ids.push_back(0);
        c->ring = ring;
        c->farcap = farcap;
        size_t off = 0;
        c->off_rec = (uint32_t)off;
        off += rec_bytes;
        c->off_edge = (uint32_t)off;
        off += al(std::max(edge_bytes, farcap * far_entry));
        c->off_fid = (uint32_t)off;
        off += al(2 * (size_t)farcap * 4);
        c->bm_shared = bm_bytes ? 1u : 0u;
        c->off_bm = (uint32_t)off;
        off += bm_bytes;
        c->off_pbits = (uint32_t)off;
        off += al(((size_t)c->n_pieces + 31) / 32 * 4);
        c->off_mbar = (uint32_t)off;
        off += 128;
        c->off_ring = (uint32_t)off;
        // reverse pass: ring2 and the row staging buffers [2][cap][2][bw] share
        // the ring's memory
        uint32_t ring2 = 0;
        for (uint32_t r = 1; (size_t)r * c->bw * 4 + rows_bytes <= ring_bytes(ring); r *= 2) ring2 = r;
        c->ring2 = ring2;
        c->fwd_smem = off + ring_bytes(ring);
        c->chain = c->n_pieces;
    }
    // nets one pair may mark in the cover: as many as its shared memory holds
    c->hash_cap = 4096;
    while (c->hash_cap > 256 && cover_smem_bytes(c->hash_cap) > (size_t)prop.sharedMemPerBlockOptin) c->hash_cap -= 256;
    c->cover_threads = 256;
    c->cover_grid = (uint32_t)prop.multiProcessorCount;

    auto fail = [&](pdf_status st2) {
        c->segs.release();
        c->seg_off.release();
        c->rec.release();
        c->edges.release();
        c->level_off.release();
        c->pieces.release();
        c->far.release();
        c->err.release();
        delete c;
        return st2;
    };
    if (c->rec.ensure(sizeof(GateRec) * G) != cudaSuccess ||
        c->edges.ensure(sizeof(uint32_t) * edges.size()) != cudaSuccess ||
        c->level_off.ensure(sizeof(uint32_t) * (L + 1)) != cudaSuccess ||
        c->pieces.ensure(sizeof(Piece) * pieces.size()) != cudaSuccess ||
        c->far.ensure(sizeof(uint32_t) * far_ids.size()) != cudaSuccess || c->err.ensure(16) != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(PDF_ENOMEM);
    }
    if (cudaMemcpy(c->rec.p, recs.data(), sizeof(GateRec) * G, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->edges.p, edges.data(), sizeof(uint32_t) * edges.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->level_off.p, nl->level_offsets, sizeof(uint32_t) * (L + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->pieces.p, pieces.data(), sizeof(Piece) * pieces.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(c->far.p, far_ids.data(), sizeof(uint32_t) * far_ids.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemset(c->err.p, 0, 16) != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(PDF_ECUDA);
    }
    c->dc.rec = c->rec.as<GateRec>();
    c->dc.edges = c->edges.as<uint32_t>();
    c->dc.level_off = c->level_off.as<uint32_t>();
    c->dc.n_gates = G;
    c->dc.n_levels = L;
    c->dc.n_pi = inf.n_pi;
    inf.tile_words = c->bw;
    inf.threads = c->threads;
    inf.max_pairs = o.max_pairs ? o.max_pairs : 65536;
    if (o.seg_len > 1) {
        const pdf_status sst = build_segments(c, nl, o.seg_len);
        if (sst != PDF_OK) {
            (void)cudaGetLastError();
            return fail(sst);
        }
    }
    inf.seg_len = c->seg_len;
    inf.n_segments = c->n_first();
    inf.device_bytes = c->rec.bytes + c->edges.bytes + c->level_off.bytes + c->pieces.bytes + c->far.bytes +
                       c->segs.bytes + c->seg_off.bytes;
    *out = c;
    return PDF_OK;
}

extern "C" pdf_status pdf_circuit_segments(const pdf_circuit *c, uint32_t *gates) {
    if (!c || !gates) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    if (c->seg_len <= 1) {
        for (uint32_t g = 0; g < c->info.n_gates; g++) gates[g] = g;
        return PDF_OK;
    }
    PDF_CUDA(cudaMemcpy(gates, c->segs.p, (size_t)c->n_segs * c->seg_len * 4, cudaMemcpyDeviceToHost));
    return PDF_OK;
}

extern "C" void pdf_circuit_destroy(pdf_circuit *c) {
    if (!c) return;
    DeviceGuard dg(c->device);
    c->stage.release();
    c->rec.release();
    c->edges.release();
    c->level_off.release();
    c->pieces.release();
    c->far.release();
    c->err.release();
    c->segs.release();
    c->seg_off.release();
    delete c;
}

extern "C" pdf_status pdf_circuit_query(const pdf_circuit *c, pdf_circuit_info *info) {
    if (!c || !info) return PDF_EINVAL;
    *info = c->info;
    return PDF_OK;
}

// ---------------------------------------------------------------------------

extern "C" pdf_status pdf_state_create(pdf_circuit *c, pdf_state **out) {
    if (!c || !out) return PDF_EINVAL;
    *out = nullptr;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    pdf_state *s = new (std::nothrow) pdf_state();
    if (!s) return PDF_ENOMEM;
    s->c = c;
    s->device = c->device;
    const size_t G = c->n_first();  // first-detect entries: nets, or segments
    if (s->first_x.ensure(4 * G) != cudaSuccess || s->first_y.ensure(4 * G) != cudaSuccess ||
        s->acc.ensure(sizeof(DevAcc)) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&s->host_acc), sizeof(DevAcc), cudaHostAllocDefault) != cudaSuccess) {
        s->host_acc = nullptr;
        (void)cudaGetLastError();
        pdf_state_destroy(s);
        return PDF_ENOMEM;
    }
    std::memset(s->host_acc, 0, sizeof(DevAcc));
    // cleared on a stream of its own: a device-wide sync here would wait for
    // every other circuit's work in flight (a server creates states while it
    // grades)
    cudaStream_t cs = nullptr;
    const bool ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaMemsetAsync(s->first_x.p, 0xFF, 4 * G, cs) == cudaSuccess &&
                    cudaMemsetAsync(s->first_y.p, 0xFF, 4 * G, cs) == cudaSuccess &&
                    cudaMemsetAsync(s->acc.p, 0, sizeof(DevAcc), cs) == cudaSuccess &&
                    cudaStreamSynchronize(cs) == cudaSuccess;
    if (cs) cudaStreamDestroy(cs);
    if (!ok) {
        note_cuda_error(cudaGetLastError(), "pdf_state_create: clearing the state", __LINE__);
        pdf_state_destroy(s);
        return PDF_ECUDA;
    }
    *out = s;
    return PDF_OK;
}

extern "C" void pdf_state_destroy(pdf_state *s) {
    if (!s) return;
    DeviceGuard dg(s->device);
    prof_release(s->prof);
    prof_release(s->pool);
    s->ws.release();
    s->first_x.release();
    s->first_y.release();
    s->acc.release();
    if (s->host_acc && cudaFreeHost(s->host_acc) != cudaSuccess) (void)cudaGetLastError();
    delete s;
}

extern "C" pdf_status pdf_state_reset(pdf_state *s) {
    if (!s) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    const size_t G = s->c->n_first();
    PDF_CUDA(cudaDeviceSynchronize());
    PDF_CUDA(cudaMemset(s->first_x.p, 0xFF, 4 * G));
    PDF_CUDA(cudaMemset(s->first_y.p, 0xFF, 4 * G));
    PDF_CUDA(cudaMemset(s->acc.p, 0, sizeof(DevAcc)));
    PDF_CUDA(cudaDeviceSynchronize());
    return PDF_OK;
}

extern "C" pdf_status pdf_state_reset_async(pdf_state *s, void *stream) {
    if (!s) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const size_t G = s->c->n_first();
    PDF_CUDA(cudaMemsetAsync(s->first_x.p, 0xFF, 4 * G, cs));
    PDF_CUDA(cudaMemsetAsync(s->first_y.p, 0xFF, 4 * G, cs));
    PDF_CUDA(cudaMemsetAsync(s->acc.p, 0, sizeof(DevAcc), cs));
    return PDF_OK;
}

extern "C" pdf_status pdf_state_profile(pdf_state *s, int enable) {
    if (!s) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    std::lock_guard<std::mutex> lk(s->mu);
    PDF_CUDA(cudaDeviceSynchronize());
    for (auto &p : s->prof) s->pool.push_back(p);
    s->prof.clear();
    s->profiling = enable != 0;
    return PDF_OK;
}

extern "C" pdf_status pdf_state_profile_read(pdf_state *s, double *ms, uint32_t *calls) {
    if (!s || !ms) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    std::lock_guard<std::mutex> lk(s->mu);
    ms[0] = ms[1] = ms[2] = 0;
    for (auto &p : s->prof) {
        PDF_CUDA(cudaEventSynchronize(p.ev[3]));
        float a = 0, b = 0, c = 0;
        PDF_CUDA(cudaEventElapsedTime(&a, p.ev[0], p.ev[1]));
        PDF_CUDA(cudaEventElapsedTime(&b, p.ev[2], p.ev[3]));
        PDF_CUDA(cudaEventElapsedTime(&c, p.ev[0], p.ev[3]));
        ms[0] += a;
        ms[1] += b;
        ms[2] += c;
    }
    if (calls) *calls = (uint32_t)s->prof.size();
    return PDF_OK;
}

extern "C" pdf_status pdf_state_snapshot(pdf_state *s, uint32_t *first_x, uint32_t *first_y,
                                         pdf_totals *tot) {
    if (!s) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    const size_t G = s->c->n_first();
    PDF_CUDA(cudaDeviceSynchronize());
    if (first_x) PDF_CUDA(cudaMemcpy(first_x, s->first_x.p, 4 * G, cudaMemcpyDeviceToHost));
    if (first_y) PDF_CUDA(cudaMemcpy(first_y, s->first_y.p, 4 * G, cudaMemcpyDeviceToHost));
    DevAcc h{};
    PDF_CUDA(cudaMemcpy(&h, s->acc.p, sizeof h, cudaMemcpyDeviceToHost));
    if (tot) {
        tot->lo = h.total_lo;
        tot->hi = h.total_hi;
        tot->pairs = h.pairs;
        tot->flags = h.flags;
        tot->reserved = 0;
    }
    return err_status(h.err);
}

extern "C" pdf_status pdf_state_snapshot_on(pdf_state *s, uint32_t *first_x, uint32_t *first_y, pdf_totals *tot,
                                            void *stream) {
    if (!s) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    const size_t G = s->c->n_first();
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if (first_x) PDF_CUDA(cudaMemcpyAsync(first_x, s->first_x.p, 4 * G, cudaMemcpyDeviceToHost, cs));
    if (first_y) PDF_CUDA(cudaMemcpyAsync(first_y, s->first_y.p, 4 * G, cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaMemcpyAsync(s->host_acc, s->acc.p, sizeof(DevAcc), cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    const DevAcc &h = *s->host_acc;
    if (tot) {
        tot->lo = h.total_lo;
        tot->hi = h.total_hi;
        tot->pairs = h.pairs;
        tot->flags = h.flags;
        tot->reserved = 0;
    }
    return err_status(h.err);
}

extern "C" pdf_status pdf_state_restore(pdf_state *s, const uint32_t *first_x,
                                        const uint32_t *first_y, const pdf_totals *tot) {
    if (!s || !first_x || !first_y || !tot) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    const size_t G = s->c->n_first();
    PDF_CUDA(cudaDeviceSynchronize());
    PDF_CUDA(cudaMemcpy(s->first_x.p, first_x, 4 * G, cudaMemcpyHostToDevice));
    PDF_CUDA(cudaMemcpy(s->first_y.p, first_y, 4 * G, cudaMemcpyHostToDevice));
    DevAcc h{};
    h.total_lo = tot->lo;
    h.total_hi = tot->hi;
    h.pairs = tot->pairs;
    h.flags = tot->flags;
    PDF_CUDA(cudaMemcpy(s->acc.p, &h, sizeof h, cudaMemcpyHostToDevice));
    PDF_CUDA(cudaDeviceSynchronize());
    return PDF_OK;
}

// ---------------------------------------------------------------------------

namespace {

pdf_status check_pairs(const pdf_circuit *c, const pdf_pairs *pr, uint64_t pair_base) {
    if (!pr || !pr->v || !pr->t) return PDF_EINVAL;
    if (pr->n_pairs == 0) return PDF_EINVAL;
    if (pr->ld < (pr->n_pairs + 31) / 32) return PDF_EINVAL;
    if (pair_base + pr->n_pairs > 0xFFFFFFFFull) return PDF_EINVAL;  // pair ids are uint32, ~0 = none
    (void)c;
    return PDF_OK;
}

// Sizes the workspace for W words of pairs.
pdf_status ensure_ws(pdf_circuit *c, Workspace &ws, uint64_t W, bool need_planes) {
    const uint64_t n_blocks = (W + c->bw - 1) / c->bw;
    const uint64_t bm_words = (c->info.n_gates + 31) / 32;
    PDF_CUDA(ws.nzb.ensure(n_blocks * bm_words * 4));
    PDF_CUDA(ws.maxlvl.ensure(n_blocks * 4));
    if (lane_tile(c->bw)) {  // the cover's bitmaps per kLaneCoverWords words of a column block
        const uint64_t nf = c->bw / kLaneCoverWords;
        PDF_CUDA(ws.nzb_fine.ensure(nf * n_blocks * bm_words * 4));
        PDF_CUDA(ws.maxlvl_fine.ensure(nf * n_blocks * 4));
    }
    // active bitmap [W], then the count; the list holds <= 2 pairs per gate
    PDF_CUDA(ws.active.ensure(W * 4 + 16));
    const uint64_t list = std::min<uint64_t>(W * 32, 2 * std::max<uint64_t>(c->n_first(), c->info.n_gates));
    PDF_CUDA(ws.active_list.ensure(list * 4));
    // A pair can mark more nets than the cover's table holds only when the
    // circuit has more gates than that; its count then goes through the
    // spill cover, whose slots of 2 x n_gates u128 take up to 16 MiB (at
    // least one slot).
    if (c->info.n_gates > c->hash_cap) {
        const uint64_t slot = 2 * (uint64_t)c->info.n_gates * 16;
        const uint32_t slots = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(16, (16ull << 20) / slot));
        PDF_CUDA(ws.over_list.ensure(list * 4));
        PDF_CUDA(ws.spill.ensure(slots * slot));
        ws.spill_slots = slots;
    }
    if (c->seg_len > 1) {
        // (net, pair) entries: at most N per first pair of a segment, two per
        // segment, and one per (net, pair); a table at least twice that
        const uint64_t most = std::min<uint64_t>(2 * c->n_segs * c->seg_len, (uint64_t)c->info.n_gates * W * 32);
        uint64_t cap = 1024;
        while (cap < 2 * most && cap < (1ull << 27)) cap <<= 1;
        if (ws.seg_first_mask + 1 < cap) {
            PDF_CUDA(ws.seg_first.ensure(cap * 8));
            ws.seg_first_mask = cap - 1;
        }
    }
    if (need_planes) {
        const uint64_t ld = n_blocks * c->bw;
        if (ws.plane_ld < ld || !ws.planes.p) {
            PDF_CUDA(ws.planes.ensure(3 * (uint64_t)c->info.n_gates * ld * 4));
            ws.plane_ld = ld;
        }
    }
    return PDF_OK;
}

FwdArgs base_fwd(pdf_circuit *c, uint64_t n_pairs) {
    FwdArgs a{};
    a.c = c->dc;
    a.pieces = c->pieces.as<Piece>();
    a.n_pieces = c->n_pieces;
    a.cap = c->cap;
    a.ecap = c->ecap;
    a.n_pairs = n_pairs;
    a.W = (uint32_t)((n_pairs + 31) / 32);
    a.store_all = 1;
    a.bm_words = (c->info.n_gates + 31) / 32;
    a.bm_shared = c->bm_shared;
    a.far_ids = c->far.as<uint32_t>();
    a.farcap = c->farcap;
    a.ring_gates = c->ring;
    a.ring2_gates = c->ring2;
    a.off_ring = c->off_ring;
    a.off_rec = c->off_rec;
    a.off_edge = c->off_edge;
    a.off_fid = c->off_fid;
    a.off_bm = c->off_bm;
    a.off_pbits = c->off_pbits;
    a.off_mbar = c->off_mbar;
    a.err = c->err.as<uint32_t>();
    a.wait_polls = c->wait_polls;
    return a;
}

// The device error word of the circuit's stage calls (pdf_sim, pdf_mark):
// read after the call's work is done, then cleared, so that an expired wait
// is reported by the call that met it and by no later one.
pdf_status take_circuit_err(pdf_circuit *c, cudaStream_t cs) {
    unsigned int e = 0;
    PDF_CUDA(cudaMemcpyAsync(&e, c->err.p, sizeof e, cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    if (e) {
        PDF_CUDA(cudaMemsetAsync(c->err.p, 0, sizeof e, cs));
        PDF_CUDA(cudaStreamSynchronize(cs));
    }
    return err_status(e);
}

CoverArgs base_cover(pdf_circuit *c, Workspace &ws, const uint32_t *M, uint64_t ld, uint64_t n_pairs,
                     uint32_t pair_base, const uint32_t *fx, const uint32_t *fy, DevAcc *acc) {
    CoverArgs a{};
    a.c = c->dc;
    a.M = M;
    a.ld = ld;
    // a lane circuit's cover reads bitmaps per 8 words of its column blocks
    // (fewer candidate nets per pair than the whole block's)
    const bool fine = lane_tile(c->bw);
    a.nzb = fine ? ws.nzb_fine.as<uint32_t>() : ws.nzb.as<uint32_t>();
    a.blk_maxlvl = fine ? ws.maxlvl_fine.as<uint32_t>() : ws.maxlvl.as<uint32_t>();
    a.bm_words = (c->info.n_gates + 31) / 32;
    a.bw = fine ? kLaneCoverWords : c->bw;
    a.first_x = fx;
    a.first_y = fy;
    a.n_pairs = n_pairs;
    a.pair_base = pair_base;
    a.active = ws.active.as<uint32_t>();
    a.active_count = a.active + (n_pairs + 31) / 32;
    a.active_list = ws.active_list.as<uint32_t>();
    a.acc = acc;
    a.hash_cap = c->hash_cap;
    a.over_list = ws.over_list.as<uint32_t>();
    a.spill = ws.spill.as<unsigned char>();
    a.spill_slots = ws.spill_slots;
    a.seg = c->seg_args();
    if (c->seg_len > 1) {
        a.seg_first = ws.seg_first.as<unsigned long long>();
        a.seg_first_mask = ws.seg_first_mask;
    }
    return a;
}

// Device pointers of the pairs (staging host pairs through the workspace).
// True when (ptr, ld) can be used by the kernels directly: rows of ld words,
// ld a multiple of the tile width and below 2^30 (row pitches in bytes fit
// 32 bits), every row long enough for whole tiles, and 16-byte aligned base
// addresses.
bool planes_fit(const pdf_circuit *c, uint64_t W, uint64_t ld, std::initializer_list<const void *> ptrs) {
    const uint64_t Wp = (W + c->bw - 1) / c->bw * c->bw;
    if (ld < Wp || ld % c->bw || ld >= (1ull << 30)) return false;
    for (const void *p : ptrs)
        if (!p || (reinterpret_cast<uintptr_t>(p) & 15)) return false;
    return true;
}

// Device pointers of the pairs, staging them through the workspace when
// they are host memory or not in the kernels' layout.
pdf_status stage_pairs(pdf_circuit *c, Workspace &ws, const pdf_pairs *pr, const uint32_t **v,
                       const uint32_t **t, uint64_t *ld, cudaStream_t st) {
    const uint64_t W = (pr->n_pairs + 31) / 32, npi = c->info.n_pi;
    if (pr->on_device && planes_fit(c, W, pr->ld, {pr->v, pr->t})) {
        *v = pr->v;
        *t = pr->t;
        *ld = pr->ld;
        return PDF_OK;
    }
    const uint64_t Wp = (W + c->bw - 1) / c->bw * c->bw;
    PDF_CUDA(ws.pi.ensure(2 * npi * Wp * 4));
    uint32_t *dv = ws.pi.as<uint32_t>(), *dt = dv + npi * Wp;
    const cudaMemcpyKind k = pr->on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (pr->ld == Wp) {  // rows already at the device pitch: one contiguous copy per plane
        PDF_CUDA(cudaMemcpyAsync(dv, pr->v, npi * Wp * 4, k, st));
        PDF_CUDA(cudaMemcpyAsync(dt, pr->t, npi * Wp * 4, k, st));
    } else {
        PDF_CUDA(cudaMemcpy2DAsync(dv, Wp * 4, pr->v, pr->ld * 4, W * 4, npi, k, st));
        PDF_CUDA(cudaMemcpy2DAsync(dt, Wp * 4, pr->t, pr->ld * 4, W * 4, npi, k, st));
    }
    *v = dv;
    *t = dt;
    *ld = Wp;
    return PDF_OK;
}

pdf_status copy_plane_out(uint32_t *dst, uint64_t dst_ld, int dst_dev, const uint32_t *src,
                          uint64_t src_ld, uint64_t W, uint64_t G, cudaStream_t st) {
    if (!dst) return PDF_OK;
    if (dst_ld < W) return PDF_EINVAL;
    PDF_CUDA(cudaMemcpy2DAsync(dst, dst_ld * 4, src, src_ld * 4, W * 4, G,
                               dst_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    return PDF_OK;
}

}  // namespace

namespace {

// First half of a grading call: sim, mark, prune and merge into the state.
// Records what the second half needs in the state.
pdf_status grade_mark_locked(pdf_circuit *c, pdf_state *s, const pdf_pairs *pr, uint64_t pair_base,
                             const pdf_outputs *out, cudaStream_t cs) {
    const uint64_t n = pr->n_pairs, W = (n + 31) / 32, G = c->info.n_gates;
    const bool direct = out && out->on_device && planes_fit(c, W, out->ld, {out->sim_v, out->sim_t, out->mark});
    pdf_status st = ensure_ws(c, s->ws, W, !direct);
    if (st != PDF_OK) return st;
    const uint32_t *pv, *pt;
    uint64_t pld;
    st = stage_pairs(c, s->ws, pr, &pv, &pt, &pld, cs);
    if (st != PDF_OK) return st;

    FwdArgs a = base_fwd(c, n);
    a.pi_v = pv;
    a.pi_t = pt;
    a.pi_ld = pld;
    // with no plane asked for, only the rows read back are written
    a.store_all = out && (out->sim_v || out->sim_t || out->mark) ? 1u : 0u;
    if (direct) {
        a.V = out->sim_v;
        a.T = out->sim_t;
        a.M = out->mark;
        a.ld = out->ld;
    } else {
        a.ld = s->ws.plane_ld;
        a.V = s->ws.planes.as<uint32_t>();
        a.T = a.V + G * a.ld;
        a.M = a.T + G * a.ld;
    }
    a.nzb = s->ws.nzb.as<uint32_t>();
    a.blk_maxlvl = s->ws.maxlvl.as<uint32_t>();
    a.nzb_fine = s->ws.nzb_fine.as<uint32_t>();
    a.maxlvl_fine = s->ws.maxlvl_fine.as<uint32_t>();
    // with segments the state holds per-segment ids, merged after the kernel
    a.first_x = c->seg_len > 1 ? nullptr : s->first_x.as<uint32_t>();
    a.first_y = c->seg_len > 1 ? nullptr : s->first_y.as<uint32_t>();
    a.pair_base = (uint32_t)pair_base;
    DevAcc *acc = s->acc.as<DevAcc>();
    a.err = &acc->err;
    s->pe = nullptr;
    if (s->profiling) {
        ProfEvents p{};
        if (!s->pool.empty()) {
            p = s->pool.back();
            s->pool.pop_back();
        } else {
            for (auto &e : p.ev) PDF_CUDA(cudaEventCreate(&e));
        }
        s->prof.push_back(p);
        s->pe = &s->prof.back();
        PDF_CUDA(cudaEventRecord(s->pe->ev[0], cs));
    }
    // the forward kernel also clears the batch count and the cover's active pairs
    a.acc = acc;
    a.active = s->ws.active.as<uint32_t>();
    PDF_CUDA(launch_forward(a, FWD_FUSED, c->mark_mode, c->bw, c->threads, c->fwd_smem, cs));
    if (c->seg_len > 1) {
        SegMergeArgs sm{};
        sm.seg = c->seg_args();
        sm.V = a.V;
        sm.M = a.M;
        sm.ld = a.ld;
        sm.nzb = a.nzb;
        sm.bm_words = a.bm_words;
        sm.bw = c->bw;
        sm.W = (uint32_t)W;
        sm.pair_base = (uint32_t)pair_base;
        sm.first_x = s->first_x.as<uint32_t>();
        sm.first_y = s->first_y.as<uint32_t>();
        PDF_CUDA(launch_seg_merge(sm, (uint32_t)((W + c->bw - 1) / c->bw), cs));
    }
    if (s->pe) PDF_CUDA(cudaEventRecord(s->pe->ev[1], cs));
    if (out && !direct) {
        st = copy_plane_out(out->sim_v, out->ld, out->on_device, a.V, a.ld, W, G, cs);
        if (st == PDF_OK) st = copy_plane_out(out->sim_t, out->ld, out->on_device, a.T, a.ld, W, G, cs);
        if (st == PDF_OK) st = copy_plane_out(out->mark, out->ld, out->on_device, a.M, a.ld, W, G, cs);
        if (st != PDF_OK) return st;
    }
    s->pend_M = a.M;
    s->pend_ld = a.ld;
    s->pend_n = n;
    s->pend_base = pair_base;
    s->pending = true;
    return PDF_OK;
}

// Second half: count the covered paths of the marked batch against the
// state's first-detect ids and add them to the total.
pdf_status grade_cover_locked(pdf_circuit *c, pdf_state *s, cudaStream_t cs) {
    if (!s->pending) return PDF_EINVAL;
    s->pending = false;
    DevAcc *acc = s->acc.as<DevAcc>();
    const uint32_t base = (uint32_t)s->pend_base;
    CoverArgs ca = base_cover(c, s->ws, s->pend_M, s->pend_ld, s->pend_n, base, s->first_x.as<uint32_t>(),
                              s->first_y.as<uint32_t>(), acc);
    if (s->pe) PDF_CUDA(cudaEventRecord(s->pe->ev[2], cs));  // cover starts (after any exchange)
    PDF_CUDA(launch_cover(ca, c->cover_grid, c->cover_threads, false, cs));  // closes the batch
    if (s->pe) {
        PDF_CUDA(cudaEventRecord(s->pe->ev[3], cs));
        s->pe = nullptr;
    }
    return PDF_OK;
}

}  // namespace

extern "C" pdf_status pdf_grade_mark_async(pdf_circuit *c, pdf_state *s, const pdf_pairs *pr,
                                           uint64_t pair_base, const pdf_outputs *out, void *stream) {
    if (!c || !s || s->c != c) return PDF_EINVAL;
    pdf_status st = check_pairs(c, pr, pair_base);
    if (st != PDF_OK) return st;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    std::lock_guard<std::mutex> lk(s->mu);
    return grade_mark_locked(c, s, pr, pair_base, out, static_cast<cudaStream_t>(stream));
}

extern "C" pdf_status pdf_grade_cover_async(pdf_circuit *c, pdf_state *s, void *stream) {
    if (!c || !s || s->c != c) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    std::lock_guard<std::mutex> lk(s->mu);
    return grade_cover_locked(c, s, static_cast<cudaStream_t>(stream));
}

extern "C" pdf_status pdf_grade_async(pdf_circuit *c, pdf_state *s, const pdf_pairs *pr,
                                      uint64_t pair_base, const pdf_outputs *out, void *stream) {
    if (!c || !s || s->c != c) return PDF_EINVAL;
    pdf_status st = check_pairs(c, pr, pair_base);
    if (st != PDF_OK) return st;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(s->mu);
    st = grade_mark_locked(c, s, pr, pair_base, out, cs);
    if (st != PDF_OK) return st;
    return grade_cover_locked(c, s, cs);
}

extern "C" pdf_status pdf_state_first_copy(pdf_state *s, uint32_t *first_x, uint32_t *first_y, int to_state,
                                           void *stream) {
    if (!s || !first_x || !first_y) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const size_t bytes = 4 * (size_t)s->c->n_first();
    if (to_state) {
        PDF_CUDA(cudaMemcpyAsync(s->first_x.p, first_x, bytes, cudaMemcpyDeviceToDevice, cs));
        PDF_CUDA(cudaMemcpyAsync(s->first_y.p, first_y, bytes, cudaMemcpyDeviceToDevice, cs));
    } else {
        PDF_CUDA(cudaMemcpyAsync(first_x, s->first_x.p, bytes, cudaMemcpyDeviceToDevice, cs));
        PDF_CUDA(cudaMemcpyAsync(first_y, s->first_y.p, bytes, cudaMemcpyDeviceToDevice, cs));
    }
    return PDF_OK;
}

extern "C" pdf_status pdf_grade(pdf_circuit *c, pdf_state *s, const pdf_pairs *pr, uint64_t pair_base,
                                const pdf_outputs *out, pdf_totals *batch, void *stream) {
    pdf_status st = pdf_grade_async(c, s, pr, pair_base, out, stream);
    if (st != PDF_OK) return st;
    DeviceGuard dg(c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    PDF_CUDA(cudaMemcpyAsync(s->host_acc, s->acc.p, sizeof(DevAcc), cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    const DevAcc &h = *s->host_acc;
    if (batch) {
        batch->lo = h.batch_lo;
        batch->hi = h.batch_hi;
        batch->pairs = pr->n_pairs;
        batch->flags = h.batch_flags;
        batch->reserved = 0;
    }
    return err_status(h.err);
}

// ---- stage calls ----------------------------------------------------------

extern "C" pdf_status pdf_sim(pdf_circuit *c, const pdf_pairs *pr, uint32_t *sim_v, uint32_t *sim_t,
                              uint64_t ld, void *stream) {
    if (!c || !sim_v || !sim_t) return PDF_EINVAL;
    pdf_status st = check_pairs(c, pr, 0);
    if (st != PDF_OK) return st;
    const uint64_t W = (pr->n_pairs + 31) / 32, G = c->info.n_gates;
    if (ld < W) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(c->mu);
    const bool direct = planes_fit(c, W, ld, {sim_v, sim_t});
    st = ensure_ws(c, c->stage, W, !direct);
    if (st != PDF_OK) return st;
    const uint32_t *pv, *pt;
    uint64_t pld;
    st = stage_pairs(c, c->stage, pr, &pv, &pt, &pld, cs);
    if (st != PDF_OK) return st;
    FwdArgs a = base_fwd(c, pr->n_pairs);
    a.pi_v = pv;
    a.pi_t = pt;
    a.pi_ld = pld;
    if (direct) {
        a.V = sim_v;
        a.T = sim_t;
        a.ld = ld;
    } else {
        a.ld = c->stage.plane_ld;
        a.V = c->stage.planes.as<uint32_t>();
        a.T = a.V + G * a.ld;
    }
    PDF_CUDA(launch_forward(a, FWD_SIM, c->mark_mode, c->bw, c->threads, c->fwd_smem, cs));
    if (!direct) {
        PDF_CUDA(cudaMemcpy2DAsync(sim_v, ld * 4, a.V, a.ld * 4, W * 4, G, cudaMemcpyDeviceToDevice, cs));
        PDF_CUDA(cudaMemcpy2DAsync(sim_t, ld * 4, a.T, a.ld * 4, W * 4, G, cudaMemcpyDeviceToDevice, cs));
    }
    PDF_CUDA(cudaStreamSynchronize(cs));  // the stage scratch is reused by the next stage call
    return take_circuit_err(c, cs);
}

namespace {

pdf_status mark_planes(pdf_circuit *c, const uint32_t *sim_v, const uint32_t *sim_t, uint32_t *mark,
                       uint64_t n_pairs, uint64_t ld, void *stream, bool prune) {
    if (!c || !sim_v || !sim_t || !mark || n_pairs == 0 || ld < (n_pairs + 31) / 32) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lk(c->mu);
    const uint64_t W = (n_pairs + 31) / 32, G = c->info.n_gates;
    const bool direct = planes_fit(c, W, ld, {sim_v, sim_t, mark});
    pdf_status st = ensure_ws(c, c->stage, W, !direct);
    if (st != PDF_OK) return st;
    FwdArgs a = base_fwd(c, n_pairs);
    if (direct) {
        a.V = const_cast<uint32_t *>(sim_v);
        a.T = const_cast<uint32_t *>(sim_t);
        a.M = mark;
        a.ld = ld;
    } else {
        a.ld = c->stage.plane_ld;
        a.V = c->stage.planes.as<uint32_t>();
        a.T = a.V + G * a.ld;
        a.M = a.T + G * a.ld;
        PDF_CUDA(cudaMemcpy2DAsync(a.V, a.ld * 4, sim_v, ld * 4, W * 4, G, cudaMemcpyDeviceToDevice, cs));
        PDF_CUDA(cudaMemcpy2DAsync(a.T, a.ld * 4, sim_t, ld * 4, W * 4, G, cudaMemcpyDeviceToDevice, cs));
    }
    a.nzb = c->stage.nzb.as<uint32_t>();
    a.blk_maxlvl = c->stage.maxlvl.as<uint32_t>();
    a.no_prune = prune ? 0u : 1u;
    PDF_CUDA(launch_forward(a, FWD_MARK, c->mark_mode, c->bw, c->threads, c->fwd_smem, cs));
    if (!direct)
        PDF_CUDA(cudaMemcpy2DAsync(mark, ld * 4, a.M, a.ld * 4, W * 4, G, cudaMemcpyDeviceToDevice, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    return take_circuit_err(c, cs);
}

}  // namespace

extern "C" pdf_status pdf_mark(pdf_circuit *c, const uint32_t *sim_v, const uint32_t *sim_t,
                               uint32_t *mark, uint64_t n_pairs, uint64_t ld, void *stream) {
    return mark_planes(c, sim_v, sim_t, mark, n_pairs, ld, stream, true);
}

extern "C" pdf_status pdf_mark_forward(pdf_circuit *c, const uint32_t *sim_v, const uint32_t *sim_t,
                                       uint32_t *mark, uint64_t n_pairs, uint64_t ld, void *stream) {
    return mark_planes(c, sim_v, sim_t, mark, n_pairs, ld, stream, false);
}

extern "C" pdf_status pdf_merge(pdf_circuit *c, pdf_state *s, const uint32_t *sim_v, const uint32_t *mark,
                                uint64_t n_pairs, uint64_t ld, uint64_t pair_base, void *stream) {
    if (!c || !s || s->c != c || !sim_v || !mark || n_pairs == 0 || ld < (n_pairs + 31) / 32)
        return PDF_EINVAL;
    if (pair_base + n_pairs > 0xFFFFFFFFull) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if (c->seg_len > 1)
        PDF_CUDA(launch_seg_merge_dense(c->seg_args(), sim_v, mark, ld, n_pairs, (uint32_t)pair_base,
                                        s->first_x.as<uint32_t>(), s->first_y.as<uint32_t>(), cs));
    else
        PDF_CUDA(launch_merge_dense(c->dc, sim_v, mark, ld, n_pairs, (uint32_t)pair_base,
                                    s->first_x.as<uint32_t>(), s->first_y.as<uint32_t>(), cs));
    return PDF_OK;
}

namespace {

// pdf_cover, and with `counts` (host) the paths each primary input credits to
// each pair of the chunk.
pdf_status cover_chunk(pdf_circuit *c, pdf_state *s, const uint32_t *mark, uint64_t n_pairs, uint64_t ld,
                       uint64_t pair_base, uint64_t *counts, pdf_totals *chunk, cudaStream_t cs) {
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t W = (n_pairs + 31) / 32;
    pdf_status st = ensure_ws(c, s->ws, W, false);
    if (st != PDF_OK) return st;
    const size_t count_bytes = (size_t)c->info.n_pi * n_pairs * 16;
    if (counts) {
        PDF_CUDA(s->ws.pi_counts.ensure(count_bytes));
        PDF_CUDA(cudaMemsetAsync(s->ws.pi_counts.p, 0, count_bytes, cs));
    }
    DevAcc *acc = s->acc.as<DevAcc>();
    PDF_CUDA(launch_batch_begin(acc, cs));
    CoverArgs ca = base_cover(c, s->ws, mark, ld, n_pairs, (uint32_t)pair_base, s->first_x.as<uint32_t>(),
                              s->first_y.as<uint32_t>(), acc);
    // the bitmaps the cover reads, at its granularity, from the given marks
    PDF_CUDA(launch_bitmap_from_marks(c->dc, mark, ld, n_pairs, ca.bw, const_cast<uint32_t *>(ca.nzb),
                                      const_cast<uint32_t *>(ca.blk_maxlvl), ca.bm_words, cs));
    if (counts) ca.pi_counts = s->ws.pi_counts.as<unsigned long long>();
    PDF_CUDA(launch_cover(ca, c->cover_grid, c->cover_threads, true, cs));  // closes the batch
    PDF_CUDA(cudaMemcpyAsync(s->host_acc, s->acc.p, sizeof(DevAcc), cudaMemcpyDeviceToHost, cs));
    if (counts) PDF_CUDA(cudaMemcpyAsync(counts, s->ws.pi_counts.p, count_bytes, cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    const DevAcc &h = *s->host_acc;
    if (chunk) {
        chunk->lo = h.batch_lo;
        chunk->hi = h.batch_hi;
        chunk->pairs = n_pairs;
        chunk->flags = h.batch_flags;
        chunk->reserved = 0;
    }
    return err_status(h.err);
}

}  // namespace

extern "C" pdf_status pdf_cover(pdf_circuit *c, pdf_state *s, const uint32_t *mark, uint64_t n_pairs,
                                uint64_t ld, uint64_t pair_base, pdf_totals *chunk, void *stream) {
    if (!c || !s || s->c != c || !mark || n_pairs == 0 || ld < (n_pairs + 31) / 32) return PDF_EINVAL;
    if (pair_base + n_pairs > 0xFFFFFFFFull) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    return cover_chunk(c, s, mark, n_pairs, ld, pair_base, nullptr, chunk, static_cast<cudaStream_t>(stream));
}

extern "C" pdf_status pdf_cover_counts(pdf_circuit *c, pdf_state *s, const uint32_t *mark, uint64_t n_pairs,
                                       uint64_t ld, uint64_t pair_base, uint64_t *counts, pdf_totals *chunk,
                                       void *stream) {
    if (!c || !s || s->c != c || !mark || !counts || n_pairs == 0 || ld < (n_pairs + 31) / 32) return PDF_EINVAL;
    if (pair_base + n_pairs > 0xFFFFFFFFull) return PDF_EINVAL;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    return cover_chunk(c, s, mark, n_pairs, ld, pair_base, counts, chunk, static_cast<cudaStream_t>(stream));
}

// Allocation-free variant of pdf_cover: the same kernels, with their scratch
// carved from the fixed array g_cover_scratch (pdf_kernels.cu) instead of a
// workspace.  Allocates nothing, frees nothing.  The first call on a device
// looks the array's address up (noalloc_scratch).
extern "C" pdf_status pdf_cover_noalloc(pdf_circuit *c, const uint32_t *mark, uint64_t n_pairs, uint64_t ld,
                                        uint64_t pair_base, const uint32_t *first_x, const uint32_t *first_y,
                                        pdf_totals *chunk_total, void *stream) {
    if (!c || !mark || !first_x || !first_y || !chunk_total || n_pairs == 0 || ld < (n_pairs + 31) / 32)
        return PDF_EINVAL;
    if (c->seg_len > 1) return PDF_ENOTSUP;  // its fixed scratch holds no (net, pair) set
    if (pair_base + n_pairs > 0xFFFFFFFFull) return PDF_EINVAL;
    const uint64_t W = (n_pairs + 31) / 32, n_blocks = (W + c->bw - 1) / c->bw;
    const uint64_t bm_words = (c->info.n_gates + 31) / 32;
    auto a256 = [](uint64_t x) { return (x + 255) & ~(uint64_t)255; };
    const uint64_t o_maxlvl = a256(n_blocks * bm_words * 4);
    const uint64_t o_active = o_maxlvl + a256(n_blocks * 4);
    const uint64_t o_list = o_active + a256(W * 4 + 16);
    const uint64_t o_acc = o_list + a256(std::min<uint64_t>(W * 32, 2 * (uint64_t)c->info.n_gates) * 4);
    const uint64_t need = o_acc + a256(sizeof(DevAcc));
    if (need > kNoAllocScratchBytes) return PDF_ELIMIT;
    DeviceGuard dg(c->device);
    if (!dg.ok) return PDF_ECUDA;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    unsigned char *base = nullptr;
    PDF_CUDA(noalloc_scratch(c->device, &base));
    uint32_t *nzb = reinterpret_cast<uint32_t *>(base);
    uint32_t *maxlvl = reinterpret_cast<uint32_t *>(base + o_maxlvl);
    uint32_t *active = reinterpret_cast<uint32_t *>(base + o_active);
    uint32_t *active_list = reinterpret_cast<uint32_t *>(base + o_list);
    DevAcc *acc = reinterpret_cast<DevAcc *>(base + o_acc);
    // the array keeps the previous call's contents: clear the accumulator
    PDF_CUDA(cudaMemsetAsync(acc, 0, sizeof(DevAcc), cs));
    PDF_CUDA(launch_batch_begin(acc, cs));
    PDF_CUDA(launch_bitmap_from_marks(c->dc, mark, ld, n_pairs, c->bw, nzb, maxlvl, (uint32_t)bm_words, cs));
    CoverArgs ca{};
    ca.c = c->dc;
    ca.M = mark;
    ca.ld = ld;
    ca.nzb = nzb;
    ca.blk_maxlvl = maxlvl;
    ca.bm_words = (uint32_t)bm_words;
    ca.bw = c->bw;
    ca.first_x = first_x;
    ca.first_y = first_y;
    ca.n_pairs = n_pairs;
    ca.pair_base = (uint32_t)pair_base;
    ca.active = active;
    ca.active_count = active + W;
    ca.active_list = active_list;
    ca.acc = acc;
    ca.hash_cap = c->hash_cap;
    PDF_CUDA(launch_cover(ca, c->cover_grid, c->cover_threads, true, cs));  // closes the batch
    DevAcc h{};
    PDF_CUDA(cudaMemcpyAsync(&h, acc, sizeof h, cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    chunk_total->lo = h.batch_lo;
    chunk_total->hi = h.batch_hi;
    chunk_total->pairs = n_pairs;
    chunk_total->flags = h.batch_flags;
    chunk_total->reserved = 0;
    return err_status(h.err);
}

// ---------------------------------------------------------------------------
// Batched grading.
// ---------------------------------------------------------------------------

struct pdf_batch {
    int device = 0;
    uint32_t small_cap = 0, small_per_sm = 0;  // the small-table cover: nets per pair, CTAs per SM
    std::vector<pdf_circuit *> circuits;
    std::vector<pdf_state *> states;
    BatchLaunch L{};
    DevBuf ctl;  // control word, arguments, prefixes and items in one block
    uint64_t gate_evals = 0, bytes = 0;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_graph = true;
    // side streams and fork/join events of the forward launches per class
    cudaStream_t side[kMaxBatchClasses - 1] = {};
    cudaEvent_t fork = nullptr, join[kMaxBatchClasses - 1] = {};
    cudaStream_t up = nullptr;  // uploads of the control block
    unsigned char *host_ctl = nullptr;  // mapped pinned staging of the control block
    size_t host_bytes = 0;
    cudaEvent_t prof[3] = {};  // pdf_batch_profile: pass start, forward joined, pass end
    bool profiling = false;
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void release() {
        for (auto &x : prof)
            if (x) cudaEventDestroy(x);
        for (auto &x : prof) x = nullptr;
        if (host_ctl) cudaFreeHost(host_ctl);
        host_ctl = nullptr;
        host_bytes = 0;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (up) cudaStreamDestroy(up);
        up = nullptr;
        for (auto &x : side)
            if (x) cudaStreamDestroy(x);
        for (auto &x : join)
            if (x) cudaEventDestroy(x);
        if (fork) cudaEventDestroy(fork);
        exec = nullptr;
        graph = nullptr;
        cap_stream = nullptr;
        for (auto &x : side) x = nullptr;
        for (auto &x : join) x = nullptr;
        fork = nullptr;
        ctl.release();
    }
};

namespace {

// (Re)build batch b for these jobs: per-circuit arguments and prefixes in
// one device block, which is reused when it is large enough.
// up: the stream that uploads the control block, in order before the next
// pass on it (the caller then must not rebind or destroy the batch before
// that pass is done); null: uploaded and waited for here.
pdf_status batch_build(pdf_batch *b, const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags,
                       cudaStream_t up = nullptr) {
    if (!jobs || !n_jobs || (flags & ~(uint32_t)(PDF_BATCH_APPEND | PDF_BATCH_NO_GRAPH))) return PDF_EINVAL;
    pdf_circuit *c0 = jobs[0].circuit;
    if (!c0) return PDF_EINVAL;
    for (uint32_t i = 0; i < n_jobs; i++) {
        const pdf_batch_job &j = jobs[i];
        if (!j.circuit || !j.state || j.state->c != j.circuit || j.circuit->device != c0->device ||
            j.circuit->mark_mode != c0->mark_mode)
            return PDF_EINVAL;
        if (j.circuit->seg_len > 1) return PDF_ENOTSUP;  // batches grade segments of one net
        const uint64_t n = j.pairs.n_pairs, W = (n + 31) / 32;
        if (n == 0 || !j.pairs.on_device || j.pair_base + n > 0xFFFFFFFFull ||
            !planes_fit(j.circuit, W, j.pairs.ld, {j.pairs.v, j.pairs.t}))
            return PDF_EINVAL;
    }
    b->drop_graph();
    b->device = c0->device;
    b->circuits.clear();
    b->states.clear();
    b->gate_evals = 0;
    std::vector<FwdArgs> fa(n_jobs);
    std::vector<CoverArgs> ca(n_jobs);
    std::vector<uint32_t> bp(n_jobs + 1, 0), gp(n_jobs + 1, 0);
    uint64_t items = 0;
    BatchLaunch &L = b->L;
    L = BatchLaunch{};
    L.sem = (uint32_t)c0->mark_mode;
    L.hash_cap = c0->hash_cap;
    // Jobs in classes of equal tile width and CTAs per SM (1, 2, 4), each
    // class one forward launch (its kernel, block size and shared memory
    // sized for its members), so the CTAs of narrow circuits share SMs
    // instead of holding the shared memory of the widest member; within a
    // class the longest CTA walks go first.
    std::vector<uint32_t> order(n_jobs);
    for (uint32_t i = 0; i < n_jobs; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
        const pdf_circuit *cx = jobs[x].circuit, *cy = jobs[y].circuit;
        if (cx->bw != cy->bw) return cx->bw > cy->bw;
        if (cx->occ != cy->occ) return cx->occ < cy->occ;
        return cx->chain > cy->chain;
    });
    for (uint32_t k = 0; k < n_jobs; k++) {
        const pdf_batch_job &j = jobs[order[k]];
        const uint32_t i = k;
        pdf_circuit *c = j.circuit;
        pdf_state *s = j.state;
        const uint64_t n = j.pairs.n_pairs, W = (n + 31) / 32, G = c->info.n_gates;
        if (ensure_ws(c, s->ws, W, true) != PDF_OK) return PDF_ENOMEM;
        FwdArgs a = base_fwd(c, n);
        a.pi_v = j.pairs.v;
        a.pi_t = j.pairs.t;
        a.pi_ld = j.pairs.ld;
        a.store_all = 0;
        a.ld = s->ws.plane_ld;
        a.V = s->ws.planes.as<uint32_t>();
        a.T = a.V + G * a.ld;
        a.M = a.T + G * a.ld;
        a.nzb = s->ws.nzb.as<uint32_t>();
        a.blk_maxlvl = s->ws.maxlvl.as<uint32_t>();
        a.nzb_fine = s->ws.nzb_fine.as<uint32_t>();
        a.maxlvl_fine = s->ws.maxlvl_fine.as<uint32_t>();
        a.first_x = s->first_x.as<uint32_t>();
        a.first_y = s->first_y.as<uint32_t>();
        a.pair_base = (uint32_t)j.pair_base;
        DevAcc *acc = s->acc.as<DevAcc>();
        a.err = &acc->err;
        a.acc = acc;
        a.active = s->ws.active.as<uint32_t>();
        fa[i] = a;
        ca[i] = base_cover(c, s->ws, a.M, a.ld, n, (uint32_t)j.pair_base, a.first_x, a.first_y, acc);
        const uint64_t blocks = (W + c->bw - 1) / c->bw;
        if (bp[i] + blocks > 0x7FFFFFFFull || gp[i] + G > 0xFFFFFFFFull) return PDF_ENOTSUP;
        bp[i + 1] = bp[i] + (uint32_t)blocks;
        gp[i + 1] = gp[i] + (uint32_t)G;
        items += std::min<uint64_t>(W * 32, 2 * G);
        L.threads = std::max(L.threads, c->threads);
        L.fwd_smem = std::max(L.fwd_smem, c->fwd_smem);
        L.cover_grid = std::max(L.cover_grid, c->cover_grid);
        if (!L.n_class || L.cls[L.n_class - 1].occ != c->occ || L.cls[L.n_class - 1].bw != c->bw) {
            if (L.n_class == kMaxBatchClasses) return PDF_ENOTSUP;
            BatchClass &k2 = L.cls[L.n_class++];
            k2.bw = c->bw;
            k2.occ = c->occ;
            k2.blk0 = bp[i];
        }
        BatchClass &cl = L.cls[L.n_class - 1];
        cl.threads = std::max(cl.threads, c->threads);
        cl.smem = std::max(cl.smem, c->fwd_smem);
        b->gate_evals += G * n;
        b->circuits.push_back(c);
        b->states.push_back(s);
    }
    // one side stream and join event per class after the first
    if (!b->fork) PDF_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (uint32_t k = 1; k < L.n_class; k++) {
        if (!b->side[k - 1]) PDF_CUDA(cudaStreamCreateWithFlags(&b->side[k - 1], cudaStreamNonBlocking));
        if (!b->join[k - 1]) PDF_CUDA(cudaEventCreateWithFlags(&b->join[k - 1], cudaEventDisableTiming));
    }
    for (uint32_t k = 0; k + 1 < kMaxBatchClasses; k++) {
        L.side[k] = b->side[k];
        L.join[k] = b->join[k];
    }
    L.fork = b->fork;
    b->use_graph = !(flags & PDF_BATCH_NO_GRAPH);
    // inside a captured graph the events are external nodes; run directly, plain records
    for (uint32_t k = 0; k < 3; k++) L.prof[k] = b->profiling ? b->prof[k] : nullptr;
    L.prof_external = b->use_graph ? 1u : 0u;
    L.n = n_jobs;
    L.total_blocks = bp[n_jobs];
    for (uint32_t k = 0; k < L.n_class; k++)
        L.cls[k].blocks = (k + 1 < L.n_class ? L.cls[k + 1].blk0 : L.total_blocks) - L.cls[k].blk0;
    L.total_gates = gp[n_jobs];
    L.append = (flags & PDF_BATCH_APPEND) ? 1u : 0u;
    // the small-table cover that runs first (several CTAs per SM)
    if (!b->small_cap) {  // once per batch (its device does not change)
        b->small_cap = cover_small_cap(b->device, &b->small_per_sm);
        if (!b->small_cap) return PDF_ECUDA;
    }
    L.small_cap = std::min(b->small_cap, L.hash_cap);
    L.small_grid = L.cover_grid * b->small_per_sm;
    // one device block: control word, circuit arguments, prefixes, then the
    // item lists (all items; those passed to the large table; those queued
    // for the spill cover)
    auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t list = a256(sizeof(uint2) * std::max<uint64_t>(items, 1));
    const size_t o_f = a256(sizeof(BatchCtl)), o_c = o_f + a256(sizeof(FwdArgs) * n_jobs),
                 o_b = o_c + a256(sizeof(CoverArgs) * n_jobs), o_g = o_b + a256(4 * (n_jobs + 1)),
                 o_i = o_g + a256(4 * (n_jobs + 1)), o_m = o_i + list, o_o = o_m + list, total = o_o + list;
    // the spill cover: as many CTAs as the spilling circuit with the fewest
    // slots has (circuits without slots cannot spill)
    L.spill_grid = 0;
    for (uint32_t i = 0; i < n_jobs; i++)
        if (ca[i].spill_slots) L.spill_grid = L.spill_grid ? std::min(L.spill_grid, ca[i].spill_slots) : ca[i].spill_slots;
    // The block is written into mapped pinned host memory and pulled to the
    // device by a small kernel on the batch's own stream: a copy-engine
    // transfer would queue behind other host threads' bulk uploads (a
    // server's arriving jobs), which held passes up for hundreds of ms.
    if (b->host_bytes < o_i) {
        const size_t want = std::max<size_t>({o_i, 2 * b->host_bytes, (size_t)256 << 10});
        if (b->host_ctl) cudaFreeHost(b->host_ctl);
        b->host_ctl = nullptr;
        b->host_bytes = 0;
        if (cudaHostAlloc(reinterpret_cast<void **>(&b->host_ctl), want, cudaHostAllocMapped) != cudaSuccess)
            return PDF_ENOMEM;
        b->host_bytes = want;
    }
    unsigned char *hbuf = b->host_ctl;
    std::memset(hbuf, 0, o_i);
    std::memcpy(hbuf + o_f, fa.data(), sizeof(FwdArgs) * n_jobs);
    std::memcpy(hbuf + o_c, ca.data(), sizeof(CoverArgs) * n_jobs);
    std::memcpy(hbuf + o_b, bp.data(), 4 * (n_jobs + 1));
    std::memcpy(hbuf + o_g, gp.data(), 4 * (n_jobs + 1));
    // grown geometrically: freeing the old block waits for the whole device
    if (total > b->ctl.bytes && b->ctl.ensure(std::max<size_t>({total, 2 * b->ctl.bytes, (size_t)1 << 20})) != cudaSuccess)
        return PDF_ENOMEM;
    void *src = nullptr;
    if (!up && !b->up) PDF_CUDA(cudaStreamCreateWithFlags(&b->up, cudaStreamNonBlocking));
    PDF_CUDA(cudaHostGetDevicePointer(&src, hbuf, 0));
    // the launch below is checked with cudaGetLastError, which would also
    // report an unchecked failure left on this thread by an earlier call
    // (this library's or the caller's); start from a clean slate
    (void)cudaGetLastError();
    PDF_CUDA(launch_copy_from_host(b->ctl.p, src, o_i / 16, up ? up : b->up));
    if (!up) PDF_CUDA(cudaStreamSynchronize(b->up));
    unsigned char *base = b->ctl.as<unsigned char>();
    L.ctl = reinterpret_cast<BatchCtl *>(base);
    L.fargs = reinterpret_cast<FwdArgs *>(base + o_f);
    L.cargs = reinterpret_cast<CoverArgs *>(base + o_c);
    L.bpref = reinterpret_cast<const uint32_t *>(base + o_b);
    L.gpref = reinterpret_cast<const uint32_t *>(base + o_g);
    L.items = reinterpret_cast<uint2 *>(base + o_i);
    L.mid_items = reinterpret_cast<uint2 *>(base + o_m);
    L.over_items = reinterpret_cast<uint2 *>(base + o_o);
    b->bytes = b->ctl.bytes;
    PDF_CUDA(prepare_batch(L));
    if (b->use_graph && !b->cap_stream &&
        cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
        return PDF_ECUDA;
    return PDF_OK;
}

}  // namespace

extern "C" pdf_status pdf_batch_create(const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags, pdf_batch **out) {
    if (!out) return PDF_EINVAL;
    *out = nullptr;
    if (!jobs || !n_jobs || !jobs[0].circuit) return PDF_EINVAL;
    DeviceGuard dg(jobs[0].circuit->device);
    if (!dg.ok) return PDF_ECUDA;
    pdf_batch *b = new (std::nothrow) pdf_batch();
    if (!b) return PDF_ENOMEM;
    const pdf_status st = batch_build(b, jobs, n_jobs, flags);
    if (st != PDF_OK) {
        b->release();
        delete b;
        (void)cudaGetLastError();
        return st;
    }
    *out = b;
    return PDF_OK;
}

extern "C" pdf_status pdf_batch_rebind(pdf_batch *b, const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags) {
    if (!b || !jobs || !n_jobs || !jobs[0].circuit || jobs[0].circuit->device != b->device) return PDF_EINVAL;
    DeviceGuard dg(b->device);
    if (!dg.ok) return PDF_ECUDA;
    const pdf_status st = batch_build(b, jobs, n_jobs, flags);
    if (st != PDF_OK) (void)cudaGetLastError();
    return st;
}

extern "C" void pdf_batch_destroy(pdf_batch *b) {
    if (!b) return;
    DeviceGuard dg(b->device);
    b->release();
    delete b;
}

extern "C" pdf_status pdf_batch_query(const pdf_batch *b, pdf_batch_info *info) {
    if (!b || !info) return PDF_EINVAL;
    info->n_jobs = b->L.n;
    info->tile_words = b->L.n_class ? b->L.cls[0].bw : 0;  // of the first forward class
    info->threads = b->L.threads;
    info->ctas = b->L.total_blocks;
    info->gate_evals = b->gate_evals;
    info->device_bytes = b->bytes;
    info->forward_launches = 0;
    for (uint32_t k = 0; k < b->L.n_class; k++) info->forward_launches += b->L.cls[k].blocks ? 1u : 0u;
    info->launches = info->forward_launches + (b->L.spill_grid ? 4 : 3);
    return PDF_OK;
}

extern "C" pdf_status pdf_batch_run_async(pdf_batch *b, void *stream) {
    if (!b) return PDF_EINVAL;
    DeviceGuard dg(b->device);
    if (!dg.ok) return PDF_ECUDA;
    (void)cudaGetLastError();  // an unchecked failure of an earlier call is not this run's
    if (!b->use_graph) {
        PDF_CUDA(launch_batch(b->L, static_cast<cudaStream_t>(stream)));
        return PDF_OK;
    }
    if (!b->exec) {  // capture the three launches once
        PDF_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t le = launch_batch(b->L, b->cap_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
            return PDF_ECUDA;
        }
        b->graph = g;
        PDF_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    PDF_CUDA(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
    return PDF_OK;
}

extern "C" pdf_status pdf_batch_profile(pdf_batch *b, int enable) {
    if (!b) return PDF_EINVAL;
    DeviceGuard dg(b->device);
    if (!dg.ok) return PDF_ECUDA;
    if (enable && !b->prof[0])
        for (auto &e : b->prof) PDF_CUDA(cudaEventCreate(&e));
    b->profiling = enable != 0;
    for (uint32_t k = 0; k < 3; k++) b->L.prof[k] = b->profiling ? b->prof[k] : nullptr;
    b->drop_graph();  // captured again at the next run, with or without the events
    return PDF_OK;
}

extern "C" pdf_status pdf_batch_profile_read(pdf_batch *b, double *ms) {
    if (!b || !ms || !b->profiling) return PDF_EINVAL;
    DeviceGuard dg(b->device);
    if (!dg.ok) return PDF_ECUDA;
    float f = 0.0f, c = 0.0f;
    PDF_CUDA(cudaEventSynchronize(b->prof[2]));
    PDF_CUDA(cudaEventElapsedTime(&f, b->prof[0], b->prof[1]));
    PDF_CUDA(cudaEventElapsedTime(&c, b->prof[1], b->prof[2]));
    ms[0] = f;
    ms[1] = c;
    return PDF_OK;
}

pdf_status batch_rebind_on(pdf_batch *b, const pdf_batch_job *jobs, uint32_t n_jobs, uint32_t flags,
                           cudaStream_t stream) {
    if (!b || !jobs || !n_jobs || !jobs[0].circuit || jobs[0].circuit->device != b->device || !stream)
        return PDF_EINVAL;
    DeviceGuard dg(b->device);
    if (!dg.ok) return PDF_ECUDA;
    const pdf_status st = batch_build(b, jobs, n_jobs, flags, stream);
    if (st != PDF_OK) (void)cudaGetLastError();
    return st;
}

pdf_status batch_pass_async(pdf_batch *b, cudaStream_t stream) {
    pdf_status st = pdf_batch_run_async(b, stream);
    if (st != PDF_OK) return st;
    DeviceGuard dg(b->device);
    PDF_CUDA(cudaMemcpyAsync(b->host_ctl, b->ctl.p, sizeof(BatchCtl), cudaMemcpyDeviceToHost, stream));
    return PDF_OK;
}

pdf_status batch_pass_status(const pdf_batch *b) {
    return err_status(reinterpret_cast<const BatchCtl *>(b->host_ctl)->err);
}

extern "C" pdf_status pdf_batch_run(pdf_batch *b, void *stream) {
    pdf_status st = pdf_batch_run_async(b, stream);
    if (st != PDF_OK) return st;
    DeviceGuard dg(b->device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    // read back into the pinned staging of the control block (its image is
    // rewritten at the next rebind): a DMA, not a staged pageable copy
    BatchCtl *h = reinterpret_cast<BatchCtl *>(b->host_ctl);
    PDF_CUDA(cudaMemcpyAsync(h, b->ctl.p, sizeof(BatchCtl), cudaMemcpyDeviceToHost, cs));
    PDF_CUDA(cudaStreamSynchronize(cs));
    return err_status(h->err);
}

// Autotuner of the batch tile width: times the whole batch at each candidate.
extern "C" pdf_status pdf_batch_autotune(const pdf_netlist *const *netlists, const uint64_t *n_pairs, uint32_t n,
                                         const pdf_circuit_opts *base, uint32_t reps, pdf_circuit_opts *best,
                                         float *best_ms) {
    if (!netlists || !n_pairs || !n || !best || reps == 0) return PDF_EINVAL;
    const pdf_circuit_opts b0 = base ? *base : pdf_circuit_opts{};
    DeviceGuard dg(b0.device);
    if (!dg.ok) return PDF_ECUDA;
    float best_t = 0.0f;
    uint32_t best_w = 0, best_threads = 0;
    pdf_status last = PDF_OK;
    // candidates: tile width x block size (the default, piece capacity + 64,
    // or 256 threads: pieces of 192 gates and more CTAs per SM), unless the
    // caller fixed the block size
    std::vector<std::pair<uint32_t, uint32_t>> cand;
    for (uint32_t tw : {2u, 4u, 8u})
        for (uint32_t th : {0u, 256u})
            if (!b0.threads || th == 0) cand.push_back({tw, b0.threads ? b0.threads : th});
    if (!b0.threads) {  // the lane tiles
        cand.push_back({kLaneWords, 0u});
        cand.push_back({kLaneWords2, 0u});
        cand.push_back({kLaneWords4, 0u});
    }
    for (const auto &cw : cand) {
        const uint32_t tw = cw.first;
        pdf_circuit_opts o = b0;
        o.tile_words = tw;
        o.threads = cw.second;
        std::vector<pdf_circuit *> cs(n, nullptr);
        std::vector<pdf_state *> ss(n, nullptr);
        std::vector<void *> bufs(n, nullptr);
        std::vector<pdf_batch_job> jobs(n);
        pdf_batch *b = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        pdf_status st = PDF_OK;
        for (uint32_t i = 0; i < n && st == PDF_OK; i++) {
            st = pdf_circuit_create(netlists[i], &o, &cs[i]);
            if (st == PDF_OK) st = pdf_state_create(cs[i], &ss[i]);
            if (st != PDF_OK) break;
            const uint64_t np = n_pairs[i], W = (np + 31) / 32, ld = (W + tw - 1) / tw * tw;
            const uint32_t npi = cs[i]->info.n_pi;
            std::vector<uint32_t> v(npi * ld), t(npi * ld);
            st = pdf_gen_pairs(0x7A11u + i, npi, np, ld, v.data(), t.data());
            if (st != PDF_OK) break;
            if (cudaMalloc(&bufs[i], 2 * npi * ld * 4) != cudaSuccess) {
                st = PDF_ENOMEM;
                break;
            }
            uint32_t *dv = static_cast<uint32_t *>(bufs[i]), *dt = dv + npi * ld;
            if (cudaMemcpy(dv, v.data(), npi * ld * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(dt, t.data(), npi * ld * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
                st = PDF_ECUDA;
                break;
            }
            jobs[i] = pdf_batch_job{cs[i], ss[i], pdf_pairs{dv, dt, np, ld, 1}, 0};
        }
        if (st == PDF_OK) st = pdf_batch_create(jobs.data(), n, 0, &b);
        if (st == PDF_OK) st = pdf_batch_run(b, nullptr);  // warm-up (captures the graph)
        float ms = 0.0f;
        if (st == PDF_OK) {
            if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
                cudaEventRecord(e0, nullptr) != cudaSuccess)
                st = PDF_ECUDA;
            for (uint32_t r = 0; r < reps && st == PDF_OK; r++) st = pdf_batch_run_async(b, nullptr);
            if (st == PDF_OK && (cudaEventRecord(e1, nullptr) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                                 cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
                st = PDF_ECUDA;
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        pdf_batch_destroy(b);
        for (uint32_t i = 0; i < n; i++) {
            pdf_state_destroy(ss[i]);
            pdf_circuit_destroy(cs[i]);
            if (bufs[i]) cudaFree(bufs[i]);
        }
        (void)cudaGetLastError();
        if (st != PDF_OK) {  // a tile that does not fit is skipped
            last = st;
            continue;
        }
        ms /= (float)reps;
        if (!best_w || ms < best_t) {
            best_t = ms;
            best_w = tw;
            best_threads = cw.second;
        }
    }
    if (!best_w) return last;
    *best = b0;
    best->tile_words = best_w;
    best->threads = best_threads;
    if (best_ms) *best_ms = best_t;
    return PDF_OK;
}

extern "C" pdf_status pdf_state_reserve(pdf_state *s, uint64_t n_pairs) {
    if (!s || !n_pairs) return PDF_EINVAL;
    DeviceGuard dg(s->c->device);
    if (!dg.ok) return PDF_ECUDA;
    std::lock_guard<std::mutex> lk(s->mu);
    return ensure_ws(s->c, s->ws, (n_pairs + 31) / 32, true);
}
