// pdf_server.cpp -- serving loop: continuous batching of grading jobs over
// the public C ABI (circuits, states and pdf_batch_*).
//
// A job owns a device circuit, a coverage state with its workspace and its
// vector pairs (uploaded once).  Worker threads prepare queued jobs in
// arrival order while the estimated device footprint fits the budget (host
// plan, device upload), so that work overlaps the grading; a retired job's
// memory is freed when the next admission needs it or when the server runs
// out of work (cudaFree waits for the whole device).  Each step admits the
// prepared jobs, points every active job at its next batch of pairs (a view
// of the uploaded pairs, or a device-to-device copy into a batch buffer when
// their pitch does not allow a view), grades all of them in one append-mode
// batched pass and retires the jobs whose pairs are done.  The pass is
// rebuilt when its job list or a view changes; it launches its kernels
// directly (no graph capture while workers call into CUDA).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "pdf.h"
#include "pdf_internal.h"
#include "pdf_inject.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
    uint64_t id = 0;
    pdf_netbuf *net = nullptr;  // copy of the netlist until the job retires
    pdf_netlist view{};
    const uint32_t *hv = nullptr, *ht = nullptr;  // caller's host planes
    uint64_t hld = 0, n_pairs = 0, done = 0;
    uint64_t bytes = 0;  // footprint estimate
    pdf_circuit *c = nullptr;
    pdf_state *s = nullptr;
    uint32_t *dv = nullptr;  // [2][n_pi][ld] one batch of pairs
    uint64_t ld = 0, cur = 0;  // words per row, pairs of the batch in flight
    bool in_place = false;     // the batch bound last is read from dall directly
    bool in_flight = false;    // a batch of the job is in the pass in flight
    uint64_t graded = 0;       // pairs of that batch
    uint32_t *dall = nullptr;  // [2][n_pi][hld] all the job's pairs, on the device while active
    pdf_status prep = PDF_OK;  // outcome of the preparation
    double t_ready = 0.0;
};

struct Result {
    pdf_totals total{};
    std::vector<uint32_t> fx, fy;
    pdf_status status = PDF_OK;
};

}  // namespace

struct pdf_server {
    pdf_server_opts o{};
    uint64_t next_id = 1;
    std::vector<Job *> active;
    std::map<uint64_t, Result> results;
    // two batches, used by alternate passes: one is bound for the next pass
    // while the other's pass is in flight
    pdf_batch *batch[2] = {nullptr, nullptr};
    int cur = 0;                   // the batch of the next pass
    bool pending = false;          // a pass is in flight (on `stream`, batch pend_b)
    int pend_b = 0;
    std::vector<Job *> inflight;   // the jobs it grades
    cudaEvent_t done_ev[2] = {nullptr, nullptr};  // recorded after each batch's last pass
    cudaStream_t rstream = nullptr;               // read-back of retiring jobs
    cudaStream_t stream = nullptr;
    pdf_server_stats st{};
    std::vector<double> lat_ms;
    // pinned staging of a retiring job's first-detect ids: read back by DMA,
    // not through the driver's staging of pageable copies (which the workers'
    // uploads keep busy)
    uint32_t *pin = nullptr;
    size_t pin_words = 0;
    // shared with the worker (under mu)
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job *> queue;     // submitted, not yet prepared
    std::deque<Job *> ready;     // prepared, not yet active
    std::deque<Job *> retired;   // results taken, device memory still to free (by a worker)
    uint64_t used = 0;           // footprint of prepared + active jobs
    uint64_t n_active = 0;       // jobs prepared or active (retired ones until freed)
    uint64_t preparing = 0;      // jobs a worker is preparing now
    bool stop = false;
    std::vector<std::thread> workers;
};

namespace {

// Device bytes of an active job: netlist, plan, state, workspace and pair
// buffer (an upper estimate from the netlist and the batch size).
uint64_t footprint(const pdf_netlist &nl, uint64_t batch_pairs, uint32_t bw) {
    const uint64_t G = nl.n_gates, W = (batch_pairs + 31) / 32, ld = (W + bw - 1) / bw * bw;
    const uint64_t npi = nl.level_offsets[1];
    return 64 * G + 24 * nl.n_edges       // records, edges, fan-out lists, far lists
           + 8 * G                        // first-detect ids
           + 12 * G * ld                  // V, T, M planes of one batch
           + (ld / bw) * ((G + 31) / 32) * 4 + 8 * ld * 32 + 4 * ld  // bitmaps, active pairs
           + 8 * npi * ld                 // pair buffer
           + (1u << 20);
}

// The job's pairs, uploaded once at admission.
uint64_t pairs_bytes(const pdf_netlist &nl, uint64_t hld) { return 8 * (uint64_t)nl.level_offsets[1] * hld; }

void free_job(Job *j) {
    if (j->dv) cudaFree(j->dv);
    if (j->dall) cudaFree(j->dall);
    pdf_state_destroy(j->s);
    pdf_circuit_destroy(j->c);
    pdf_netbuf_free(j->net);
    delete j;
}

}  // namespace

namespace {

// A worker's pinned staging: host-to-device copies from the caller's
// pageable planes go through two pinned halves, so a copy engine reads them
// directly; a pageable source would go through the driver's own staging,
// which the serving step's small copies would then queue behind.
struct Stage {
    unsigned char *buf[2] = {};
    cudaEvent_t ev[2] = {};
    size_t cap = 0;  // bytes per half
};

bool upload(void *dst, const void *src, size_t bytes, cudaStream_t up, Stage &sg) {
    if (!sg.buf[0] || !sg.buf[1]) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, up) == cudaSuccess;
    int k = 0;
    for (size_t off = 0; off < bytes; off += sg.cap, k ^= 1) {
        const size_t n = std::min(sg.cap, bytes - off);
        if (cudaEventSynchronize(sg.ev[k]) != cudaSuccess) return false;  // this half's last copy is done
        std::memcpy(sg.buf[k], static_cast<const unsigned char *>(src) + off, n);
        if (cudaMemcpyAsync(static_cast<unsigned char *>(dst) + off, sg.buf[k], n, cudaMemcpyHostToDevice, up) !=
                cudaSuccess ||
            cudaEventRecord(sg.ev[k], up) != cudaSuccess)
            return false;
    }
    return true;
}

// Circuit, state with its workspace, pair buffers and the job's pairs on the
// device.  On failure nothing stays allocated and j->prep holds the status.
void prepare(const pdf_server_opts &o, Job *j, cudaStream_t up, Stage &sg) {
    pdf_circuit_opts co{};
    co.device = o.device;
    co.mark_mode = o.mark_mode;
    co.tile_words = o.tile_words;
    co.max_pairs = o.batch_pairs;
    const uint64_t W = o.batch_pairs / 32, npi = j->view.level_offsets[1];
    j->ld = (W + o.tile_words - 1) / o.tile_words * o.tile_words;
    const size_t hb = (size_t)npi * j->hld * 4;
    pdf_status st = pdf_circuit_create(&j->view, &co, &j->c);
    if (st == PDF_OK) st = pdf_state_create(j->c, &j->s);
    if (st == PDF_OK) st = pdf_state_reserve(j->s, o.batch_pairs);
    if (st == PDF_OK && (cudaMalloc(&j->dv, 2 * npi * j->ld * 4) != cudaSuccess ||
                         cudaMalloc(&j->dall, pairs_bytes(j->view, j->hld)) != cudaSuccess))
        st = PDF_ENOMEM;
    if (st == PDF_OK && (cudaMemsetAsync(j->dv, 0, 2 * npi * j->ld * 4, up) != cudaSuccess ||
                         !upload(j->dall, j->hv, hb, up, sg) || !upload(j->dall + npi * j->hld, j->ht, hb, up, sg) ||
                         cudaStreamSynchronize(up) != cudaSuccess))
        st = PDF_ECUDA;
    if (st != PDF_OK) {
        if (j->dv) cudaFree(j->dv);
        if (j->dall) cudaFree(j->dall);
        pdf_state_destroy(j->s);
        pdf_circuit_destroy(j->c);
        j->dv = nullptr;
        j->dall = nullptr;
        j->s = nullptr;
        j->c = nullptr;
        (void)cudaGetLastError();
    }
    j->prep = st;
}

// Worker (several run): takes queued jobs in arrival order while they fit the
// budget and prepares them.
void work(pdf_server *srv) {
    cudaSetDevice(srv->o.device);
    cudaStream_t up = nullptr;
    cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
    Stage sg;  // without it (allocation failed) uploads go straight from the caller's planes
    sg.cap = 4u << 20;
    for (int k = 0; k < 2; k++) {
        if (cudaHostAlloc(reinterpret_cast<void **>(&sg.buf[k]), sg.cap, cudaHostAllocDefault) != cudaSuccess) {
            sg.buf[k] = nullptr;
            (void)cudaGetLastError();
        }
        if (cudaEventCreateWithFlags(&sg.ev[k], cudaEventDisableTiming) != cudaSuccess) {
            sg.ev[k] = nullptr;
            (void)cudaGetLastError();
        }
    }
    if (!sg.buf[0] || !sg.buf[1] || !sg.ev[0] || !sg.ev[1]) {  // upload() then copies directly
        for (int k = 0; k < 2; k++)
            if (sg.buf[k]) {
                cudaFreeHost(sg.buf[k]);
                sg.buf[k] = nullptr;
            }
    }
    std::unique_lock<std::mutex> lk(srv->mu);
    // cudaFree waits for the whole device, the passes in flight included, so
    // retired jobs are freed only when their memory is needed to admit the
    // next queued job, or when nothing else is left (every job that is
    // prepared or active has retired)
    auto need_free = [&] {
        if (srv->retired.empty()) return false;
        if (srv->queue.empty()) return srv->n_active == srv->retired.size();
        return srv->n_active >= srv->o.max_jobs || srv->used + srv->queue.front()->bytes > srv->o.hbm_budget;
    };
    for (;;) {
        srv->cv.wait(lk, [&] {
            if (srv->stop || need_free()) return true;
            if (srv->queue.empty() || srv->n_active >= srv->o.max_jobs) return false;
            return srv->n_active == 0 || srv->used + srv->queue.front()->bytes <= srv->o.hbm_budget;
        });
        if (srv->stop) break;
        if (need_free()) {  // freeing synchronises the device: keep it off the step
            Job *r = srv->retired.front();
            srv->retired.pop_front();
            const uint64_t bytes = r->bytes;
            lk.unlock();
            free_job(r);
            lk.lock();
            srv->used -= bytes;
            srv->n_active--;
            srv->cv.notify_all();
            continue;
        }
        Job *j = srv->queue.front();
        srv->queue.pop_front();
        srv->used += j->bytes;
        srv->n_active++;
        srv->preparing++;
        lk.unlock();
        prepare(srv->o, j, up, sg);
        lk.lock();
        srv->preparing--;
        srv->ready.push_back(j);
        srv->cv.notify_all();
    }
    lk.unlock();
    if (up) cudaStreamDestroy(up);
    for (int k = 0; k < 2; k++) {
        if (sg.buf[k]) cudaFreeHost(sg.buf[k]);
        if (sg.ev[k]) cudaEventDestroy(sg.ev[k]);
    }
}

}  // namespace

extern "C" pdf_status pdf_server_create(const pdf_server_opts *opts, pdf_server **out) {
    if (!out) return PDF_EINVAL;
    *out = nullptr;
    pdf_server_opts o = opts ? *opts : pdf_server_opts{};
    if (!o.tile_words) o.tile_words = 4;
    if (!o.batch_pairs) o.batch_pairs = 4096;
    if (!o.max_jobs) o.max_jobs = 1024;
    const bool tile_ok = o.tile_words == 1 || o.tile_words == 2 || o.tile_words == 4 || o.tile_words == 8 ||
                         o.tile_words == 32 || o.tile_words == 64 || o.tile_words == 128;
    if (o.batch_pairs % 32 || !tile_ok ||
        o.mark_mode < PDF_MARK_DEFAULT || o.mark_mode > PDF_MARK_FIXED_NONROBUST)
        return PDF_EINVAL;
    if (cudaSetDevice(o.device) != cudaSuccess) return PDF_ENODEV;
    if (!o.hbm_budget) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return PDF_ECUDA;
        o.hbm_budget = fr / 2;
    }
    pdf_server *srv = new (std::nothrow) pdf_server();
    if (!srv) return PDF_ENOMEM;
    srv->o = o;
    if (cudaStreamCreateWithFlags(&srv->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete srv;
        return PDF_ECUDA;
    }
    // the retiring jobs' staging, sized up front for circuits of 256k gates
    // (pinning memory while the loop runs contends with the workers' calls)
    if (host_alloc(reinterpret_cast<void **>(&srv->pin), 2 * (size_t)(256u << 10) * 4) ==
        cudaSuccess)
        srv->pin_words = 2 * (size_t)(256u << 10);
    else {
        srv->pin = nullptr;
        (void)cudaGetLastError();
    }
    for (uint32_t k = 0; k < (o.workers ? o.workers : 4); k++) srv->workers.emplace_back(work, srv);
    *out = srv;
    return PDF_OK;
}

extern "C" void pdf_server_destroy(pdf_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv.notify_all();
    for (std::thread &w : srv->workers) w.join();
    cudaSetDevice(srv->o.device);
    cudaStreamSynchronize(srv->stream);
    for (pdf_batch *b : srv->batch) pdf_batch_destroy(b);
    for (cudaEvent_t e : srv->done_ev)
        if (e) cudaEventDestroy(e);
    if (srv->rstream) cudaStreamDestroy(srv->rstream);
    for (Job *j : srv->active) free_job(j);
    for (Job *j : srv->ready) free_job(j);
    for (Job *j : srv->retired) free_job(j);
    for (Job *j : srv->queue) free_job(j);
    cudaStreamDestroy(srv->stream);
    if (srv->pin) cudaFreeHost(srv->pin);
    delete srv;
}

extern "C" pdf_status pdf_server_submit(pdf_server *srv, const pdf_netlist *nl, const uint32_t *v, const uint32_t *t,
                                        uint64_t ld, uint64_t n_pairs, uint64_t *job_id) {
    if (!srv || !nl || !v || !t || !n_pairs || ld < (n_pairs + 31) / 32 || n_pairs > 0xFFFFFFFFull)
        return PDF_EINVAL;
    // the netlist is checked where the job is prepared (pdf_circuit_create);
    // a job that fails there reports the status from pdf_server_result
    if (!nl->n_gates || !nl->n_levels || !nl->level_offsets) return PDF_EINVAL;
    pdf_status st = PDF_OK;
    Job *j = new (std::nothrow) Job();
    if (!j) return PDF_ENOMEM;
    if ((st = pdf_netbuf_from(nl, &j->net)) != PDF_OK) {
        delete j;
        return st;
    }
    pdf_netbuf_view(j->net, &j->view);
    j->id = srv->next_id++;
    j->hv = v;
    j->ht = t;
    j->hld = ld;
    j->n_pairs = n_pairs;
    j->bytes = footprint(j->view, srv->o.batch_pairs, srv->o.tile_words) + pairs_bytes(j->view, ld);
    j->t_ready = now_s();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->queue.push_back(j);
    }
    srv->cv.notify_one();
    if (job_id) *job_id = j->id;
    return PDF_OK;
}

// One step keeps one batched pass in flight: it admits ready jobs, binds the
// next batch of every job with pairs left to one of two batches, enqueues
// that pass on the server's stream, and only then waits for the pass the
// previous step enqueued, accounts for it and retires the jobs it finished.
// So the host's work of a step (admission, binding, read-back of retiring
// jobs) runs while the device grades, and a job's batches still follow one
// another in stream order.
extern "C" pdf_status pdf_server_step(pdf_server *srv, uint32_t *retired) {
    if (!srv) return PDF_EINVAL;
    if (retired) *retired = 0;
    if (cudaSetDevice(srv->o.device) != cudaSuccess) return PDF_ECUDA;
    const double t0 = now_s();
    pdf_status st = PDF_OK;
    // admission: the jobs the worker has prepared (in arrival order); with
    // none active and no pass in flight, wait (up to a second) for the first
    // one queued or in preparation
    {
        std::unique_lock<std::mutex> lk(srv->mu);
        if (srv->active.empty() && !srv->pending && srv->ready.empty() &&
            (srv->preparing > 0 || !srv->queue.empty()))
            srv->cv.wait_for(lk, std::chrono::seconds(1), [&] {
                return !srv->ready.empty() || (srv->preparing == 0 && srv->queue.empty());
            });
        while (!srv->ready.empty()) {
            Job *j = srv->ready.front();
            srv->ready.pop_front();
            if (j->prep != PDF_OK) {  // could not be prepared: its result reports why
                Result r;
                r.total.flags = 0;
                r.status = j->prep;
                srv->results[j->id] = std::move(r);
                srv->used -= j->bytes;
                srv->n_active--;
                free_job(j);
                srv->st.jobs_done++;
                continue;
            }
            srv->active.push_back(j);
        }
    }
    if (srv->active.empty() && !srv->pending) return PDF_OK;
    if (!srv->done_ev[0]) {
        for (int k = 0; k < 2; k++)
            if (cudaEventCreateWithFlags(&srv->done_ev[k], cudaEventDisableTiming) != cudaSuccess) {
                (void)cudaGetLastError();
                return PDF_ECUDA;
            }
        if (cudaStreamCreateWithFlags(&srv->rstream, cudaStreamNonBlocking) != cudaSuccess) {
            (void)cudaGetLastError();
            return PDF_ECUDA;
        }
    }
    // ---- the next pass: every active job with pairs left that is not in
    // the pass in flight's last batch (a job's pairs are all accounted for
    // when its last batch is enqueued).  Its next batch is read in place
    // from the job's pairs (rows of words done/32 .. on) when their pitch
    // keeps the kernels' alignment, else copied into the job's batch buffer
    // (device to device, ordered after the pass in flight, which may read it)
    const uint64_t tw = srv->o.tile_words;
    std::vector<Job *> grading;
    for (Job *j : srv->active) {
        if (j->done >= j->n_pairs) continue;
        grading.push_back(j);
        const uint64_t n = std::min<uint64_t>(srv->o.batch_pairs, j->n_pairs - j->done);
        j->cur = n;
        const uint64_t npi = j->view.level_offsets[1], w0 = j->done / 32, W = (n + 31) / 32;
        j->in_place = j->hld % tw == 0 && (npi * j->hld) % 4 == 0 && w0 % 4 == 0 && w0 % tw == 0 &&
                      w0 + (W + tw - 1) / tw * tw <= j->hld;
        if (j->in_place) continue;
        uint32_t *dv = j->dv, *dt = j->dv + npi * j->ld;
        const uint32_t *sv = j->dall + w0, *stp = j->dall + npi * j->hld + w0;
        if (cudaMemcpy2DAsync(dv, j->ld * 4, sv, j->hld * 4, W * 4, npi, cudaMemcpyDeviceToDevice, srv->stream) !=
                cudaSuccess ||
            cudaMemcpy2DAsync(dt, j->ld * 4, stp, j->hld * 4, W * 4, npi, cudaMemcpyDeviceToDevice, srv->stream) !=
                cudaSuccess) {
            (void)cudaGetLastError();
            return PDF_ECUDA;
        }
    }
    bool enqueued = false;
    const int b_now = srv->cur;
    if (!grading.empty()) {
        // the batch last used two passes ago (done: the previous step waited
        // for it); its control block is uploaded in order on the stream
        std::vector<pdf_batch_job> jobs;
        for (Job *j : grading) {
            const uint64_t npi = j->view.level_offsets[1], w0 = j->done / 32;
            const pdf_pairs p = j->in_place ? pdf_pairs{j->dall + w0, j->dall + npi * j->hld + w0, j->cur, j->hld, 1}
                                            : pdf_pairs{j->dv, j->dv + npi * j->ld, j->cur, j->ld, 1};
            jobs.push_back(pdf_batch_job{j->c, j->s, p, j->done});
        }
        const uint32_t fl = PDF_BATCH_APPEND | PDF_BATCH_NO_GRAPH;
        pdf_batch *&b = srv->batch[b_now];
        if (!b) {
            if ((st = pdf_batch_create(jobs.data(), (uint32_t)jobs.size(), fl, &b)) != PDF_OK) return st;
            // events around each pass's forward launches and cover: its device time
            if ((st = pdf_batch_profile(b, 1)) != PDF_OK) return st;
        }
        if ((st = batch_rebind_on(b, jobs.data(), (uint32_t)jobs.size(), fl, srv->stream)) != PDF_OK) return st;
        if ((st = batch_pass_async(b, srv->stream)) != PDF_OK) return st;
        // the pass is on the stream: the jobs' pairs of this batch are
        // accounted for now (the next step binds their following batch)
        for (Job *j : grading) j->done += j->cur;
        enqueued = true;
        pdf_batch_info bi{};
        if (pdf_batch_query(b, &bi) == PDF_OK) srv->st.launches += bi.launches;
        if (cudaEventRecord(srv->done_ev[b_now], srv->stream) != cudaSuccess) {
            // without its event the next step could not wait for this pass:
            // wait for it here, and report the failure once it is recorded
            (void)cudaGetLastError();
            (void)cudaStreamSynchronize(srv->stream);
            (void)cudaGetLastError();
            st = PDF_ECUDA;
        }
    }
    // ---- the pass the previous step enqueued: wait for it, account for it
    if (srv->pending) {
        const int pb = srv->pend_b;
        if (cudaEventSynchronize(srv->done_ev[pb]) != cudaSuccess) {
            // an error left by the device itself: every later read-back
            // fails too, so no job can retire with a result read early
            (void)cudaGetLastError();
            return PDF_ECUDA;
        }
        const pdf_status ps = batch_pass_status(srv->batch[pb]);
        double ms[2] = {0.0, 0.0};
        if (pdf_batch_profile_read(srv->batch[pb], ms) == PDF_OK) srv->st.gpu_s += (ms[0] + ms[1]) / 1e3;
        const double t1 = now_s();
        srv->st.steps++;
        for (Job *j : srv->inflight) {
            srv->lat_ms.push_back(1e3 * (t1 - j->t_ready));
            j->t_ready = t1;
            srv->st.batches++;
            srv->st.gate_evals += (uint64_t)j->view.n_gates * j->graded;
            j->in_flight = false;
        }
        srv->pending = false;
        srv->inflight.clear();
        if (ps != PDF_OK && st == PDF_OK) st = ps;  // reported after the pass enqueued above is recorded
    }
    if (enqueued) {
        srv->pending = true;
        srv->pend_b = b_now;
        srv->cur ^= 1;
        srv->inflight = grading;
        for (Job *j : grading) {  // after the previous pass's jobs were cleared above
            j->in_flight = true;
            j->graded = j->cur;
        }
    }
    if (st != PDF_OK) return st;
    // ---- retire the jobs whose pairs are all graded and whose last pass is
    // done.  No job is handed to the workers (who free retired jobs) or
    // leaves the active list until every read-back of this step has
    // succeeded; after a failure here those jobs stay active and retire at
    // a later step.  Read back on a stream of its own: the server's stream
    // holds the pass just enqueued.  First the pinned staging of their
    // first-detect ids, grown geometrically (freeing pinned memory waits for
    // the device).
    size_t gmax = 0;
    for (Job *j : srv->active)
        if (j->done >= j->n_pairs && !j->in_flight) gmax = std::max<size_t>(gmax, j->view.n_gates);
    if (srv->pin_words < 2 * gmax) {
        const size_t want = std::max(2 * gmax, 2 * srv->pin_words);
        if (srv->pin) cudaFreeHost(srv->pin);
        srv->pin = nullptr;
        srv->pin_words = 0;
        if (host_alloc(reinterpret_cast<void **>(&srv->pin), want * 4) != cudaSuccess) {
            srv->pin = nullptr;
            (void)cudaGetLastError();
            return PDF_ENOMEM;
        }
        srv->pin_words = want;
    }
    std::vector<Job *> keep, gone;
    std::vector<Result> res;
    for (Job *j : srv->active) {
        if (j->done < j->n_pairs || j->in_flight) {
            keep.push_back(j);
            continue;
        }
        Result r;
        const size_t G = j->view.n_gates;
        r.fx.resize(G);
        r.fy.resize(G);
        if ((st = pdf_state_snapshot_on(j->s, srv->pin, srv->pin + G, &r.total, srv->rstream)) != PDF_OK) return st;
        std::memcpy(r.fx.data(), srv->pin, 4 * G);
        std::memcpy(r.fy.data(), srv->pin + G, 4 * G);
        res.push_back(std::move(r));
        gone.push_back(j);
    }
    for (size_t k = 0; k < gone.size(); k++) srv->results[gone[k]->id] = std::move(res[k]);
    if (!gone.empty()) {
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            for (Job *j : gone) srv->retired.push_back(j);
        }
        srv->cv.notify_all();
        srv->st.jobs_done += gone.size();
        if (retired) *retired = (uint32_t)gone.size();
    }
    srv->active.swap(keep);
    srv->st.busy_s += now_s() - t0;
    return PDF_OK;
}

extern "C" pdf_status pdf_server_result(pdf_server *srv, uint64_t job_id, pdf_totals *total, uint32_t *first_x,
                                        uint32_t *first_y) {
    if (!srv) return PDF_EINVAL;
    auto it = srv->results.find(job_id);
    if (it == srv->results.end()) return PDF_EINVAL;
    if (it->second.status != PDF_OK) return it->second.status;
    if (total) *total = it->second.total;
    if (first_x) std::memcpy(first_x, it->second.fx.data(), it->second.fx.size() * 4);
    if (first_y) std::memcpy(first_y, it->second.fy.data(), it->second.fy.size() * 4);
    return PDF_OK;
}

extern "C" pdf_status pdf_server_query(const pdf_server *srv, pdf_server_stats *stats) {
    if (!srv || !stats) return PDF_EINVAL;
    *stats = srv->st;
    pdf_server *m = const_cast<pdf_server *>(srv);
    {
        std::lock_guard<std::mutex> lk(m->mu);
        stats->jobs_active = srv->active.size() + srv->ready.size();
        stats->jobs_queued = srv->queue.size();
        stats->bytes_in_use = srv->used;
    }
    std::vector<double> l = srv->lat_ms;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)(f * (l.size() - 1) + 0.5))]; };
        stats->lat_p50_ms = q(0.50);
        stats->lat_p99_ms = q(0.99);
        stats->lat_max_ms = l.back();
    }
    return PDF_OK;
}
